"""CPU checks of the learned-proposal oracle (no GPU): its backward pass
against central finite differences, its bfloat16 rounding against known
answers, and its features against a hand-computed graph."""
import numpy as np
import pytest

import mlp_oracle as mo


def _case(seed, rows):
    rng = np.random.default_rng(seed)
    d = mo.unpack(mo.init_params(seed).copy())
    d["b1"][:] = rng.normal(0, 0.1, mo.HID)
    d["b2"][:] = rng.normal(0, 0.1, mo.HID)
    d["b3"][:] = 0.3
    p = mo.pack(d)
    x = rng.normal(size=(rows, mo.IN))
    t = rng.normal(size=rows)
    return p, x, t


@pytest.mark.parametrize("seed,rows", [(0, 5), (1, 17), (2, 64)])
def test_backward_matches_finite_differences(seed, rows):
    p, x, t = _case(seed, rows)
    _, g = mo.forward_backward(p, x, t, bf16_path=False)
    rng = np.random.default_rng(seed + 100)
    # random coordinates of every parameter block, the last bias included
    offs = np.cumsum([0] + [int(np.prod(s)) for _, s in mo.SIZES])
    idx = np.concatenate([rng.choice(np.arange(offs[i], offs[i + 1]), min(12, offs[i + 1] - offs[i]), replace=False)
                          for i in range(len(mo.SIZES))])
    fd = mo.finite_difference(p, x, t, idx)
    np.testing.assert_allclose(g[idx], fd, rtol=1e-5, atol=1e-8)


def test_forward_matches_loss():
    p, x, t = _case(3, 9)
    y = mo.forward(p, x, bf16_path=False)
    loss, _ = mo.forward_backward(p, x, t, bf16_path=False)
    assert loss == pytest.approx(np.mean((y - t) ** 2), rel=1e-12)


def test_bf16_rounding_known_answers():
    vals = np.array([1.0, 1 + 2 ** -8, 1 + 2 ** -8 + 2 ** -20, 1 + 3 * 2 ** -8, -2.5, 0.0, 3.0e38, 1e-40],
                    np.float32)
    got = mo.bf16(vals)
    # halfway cases go to the even neighbour: 1 + 2^-8 -> 1, 1 + 3*2^-8 -> 1 + 2^-6
    want = np.array([1.0, 1.0, 1.0 + 2 ** -7, 1.0 + 2 ** -6, -2.5, 0.0], np.float32)
    np.testing.assert_array_equal(got[:6], want)
    assert np.isfinite(got[6]) and abs(got[6] - 3.0e38) / 3.0e38 < 2 ** -8
    assert got[7] == pytest.approx(1e-40, rel=2 ** -7)
    assert np.isnan(mo.bf16(np.array([np.nan], np.float32))[0])
    # every output is representable in bf16: the low 16 bits are zero
    r = mo.bf16(np.random.default_rng(0).normal(size=1000).astype(np.float32))
    assert not np.any(r.view(np.uint32) & 0xFFFF)


def test_bf16_path_is_the_same_function():
    p, x, t = _case(4, 200)
    l64, g64 = mo.forward_backward(p, x, t, bf16_path=False)
    l16, g16 = mo.forward_backward(p.astype(np.float32), x.astype(np.float32), t.astype(np.float32), True)
    assert l16 == pytest.approx(l64, rel=2e-2)
    assert np.linalg.norm(g16 - g64) / np.linalg.norm(g64) < 3e-2


def test_features_hand_computed():
    # G1: 1->2 (w3), 1->2 (w2, parallel), 2->3 (w5), 3->3 (self, w4), 3->1 (w0, dropped)
    # G2: 1->2 (w1), 1->2 (w6, last wins), 2->3 (w2), 3->3 (w7)
    n = 3
    s1, d1, w1 = [1, 1, 2, 3, 3], [2, 2, 3, 3, 1], [3, 2, 5, 4, 0]
    s2, d2, w2 = [1, 1, 2, 3], [2, 2, 3, 3], [1, 6, 2, 7]
    m = np.array([0, 1, 2, 3], np.int32)
    F1, F2 = mo.vertex_features(n, s1, d1, w1, s2, d2, w2, m)
    L = np.log1p
    # G1 lists (self-loop apart): 0->1 twice (3, 2), 1->2 (5)
    np.testing.assert_allclose(F1[:, 0], L([2, 1, 0]), rtol=1e-6)        # out-degree
    np.testing.assert_allclose(F1[:, 1], L([0, 2, 1]), rtol=1e-6)        # in-degree
    np.testing.assert_allclose(F1[:, 2], L([5, 5, 0]), rtol=1e-6)        # out-weight
    np.testing.assert_allclose(F1[:, 4], L([2, 0, 0]), rtol=1e-6)        # 2-hop out: out-degree of 1, twice
    np.testing.assert_allclose(F1[:, 5], L([0, 0, 2]), rtol=1e-6)        # 2-hop in: in-degree of 1 for 2
    np.testing.assert_allclose(F1[:, 6], L([3, 5, 0]), rtol=1e-6)        # max out weight
    np.testing.assert_allclose(F1[:, 8], L([0, 0, 4]), rtol=1e-6)        # self-loop
    # contributions: min(3,6)+min(2,6) on 0-1, min(5,2) on 1-2, self min(4,7)
    c = np.array([5.0, 5.0 + 2.0, 2.0 + 4.0])
    np.testing.assert_allclose(F1[:, 9], L(c), rtol=1e-6)
    np.testing.assert_allclose(F1[:, 10], c / (np.array([5, 10, 5]) + 1), rtol=1e-6)
    # G2 lists keep the self-loop: 0->1 (6), 1->2 (2), 2->2 (7)
    np.testing.assert_allclose(F2[:, 0], L([1, 1, 1]), rtol=1e-6)
    np.testing.assert_allclose(F2[:, 1], L([0, 1, 2]), rtol=1e-6)
    np.testing.assert_allclose(F2[:, 3], L([0, 6, 9]), rtol=1e-6)
    np.testing.assert_allclose(F2[:, 9], L(c), rtol=1e-6)               # identity matching
    assert not F1[:, 11:].any() and not F2[:, 11:].any()
    N1, N2 = mo.normalise(F1, F2)
    np.testing.assert_allclose(N1.mean(0), 0, atol=1e-6)
    assert not N1[:, 11:].any() and not N2[:, 11:].any()
