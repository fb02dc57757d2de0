"""GPU parity tests: the CUDA engine through its C ABI against the oracle.

Every delta, score, move sequence and final mapping must be bit-identical.
"""
import numpy as np
import pytest

import bm
import oracle
from conftest import GOLDEN_CASES, load_golden

pytestmark = pytest.mark.gpu


def _engine(g, flags=0):
    return bm.Engine(int(g["n"]), g["src1"], g["dst1"], g["w1"], g["src2"], g["dst2"], g["w2"], flags)


def _oracle(g):
    return oracle.Oracle(int(g["n"]), g["src1"], g["dst1"], g["w1"], g["src2"], g["dst2"], g["w2"])


@pytest.mark.parametrize("flags", [0, bm.BM_FLAG_FORCE_I32])
@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_all_deltas_and_score_match_golden(name, flags):
    z = load_golden(name)
    with _engine(z, flags) as E:
        E.set_mapping(z["map0"])
        assert E.score() == int(z["ref_score"])
        d = E.all_deltas()
        O = _oracle(z)
        assert np.array_equal(d, O.all_deltas(z["map0"]))
        # exact deltas = the reference's own score differences
        assert np.array_equal(d[z["pair_idx"]].astype(np.int64), z["ref_score_diff"])
        n = int(z["n"])
        a, b = np.triu_indices(n, 1)
        assert np.array_equal(E.pair_deltas(a + 1, b + 1), d)
        t = z["triples"]
        td = E.triple_deltas(t[:, 0], t[:, 1], t[:, 2])
        ref = (z["ref_local"][:, 1:] - z["ref_local"][:, :1]).astype(np.int32)
        assert np.array_equal(td, ref)


@pytest.mark.parametrize("flags", [0, bm.BM_FLAG_FORCE_I32])
def test_cfg0_all_deltas(cfg0, flags):
    g = cfg0
    with _engine(g, flags) as E:
        info = E.info()
        assert info["entry_bits"] == (32 if flags else 16)
        E.set_mapping(g["map0"])
        O = _oracle(g)
        assert E.score() == O.score(g["map0"])
        assert np.array_equal(E.all_deltas(), O.all_deltas(g["map0"]))


def test_cfg0_hillclimb_identical_move_sequence(cfg0):
    """Sweep + best-non-conflicting commit until no improving swap remains:
    the mapping after every sweep and the final score equal the oracle's."""
    g = cfg0
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g) as E:
        E.set_mapping(m)
        for it in range(200):
            st = E.sweep()
            ost = O.sweep(m)
            assert st["committed"] == ost["committed"], it
            assert st["candidates"] == ost["candidates"]
            assert st["verified"] == ost["verified"]
            assert st["score_after"] - st["score_before"] == ost["total_delta"]
            assert np.array_equal(E.get_mapping(), m), it
            if st["committed"] == 0:
                break
        assert st["committed"] == 0
        assert E.score() == O.score(m) == st["score_after"]
        assert (E.all_deltas() <= 0).all()


@pytest.mark.parametrize("max_candidates,max_verify", [(64, -1), (0, 5), (17, 3)])
def test_sweep_caps_match_oracle(cfg0, max_candidates, max_verify):
    g = cfg0
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g) as E:
        E.set_mapping(m)
        for _ in range(4):
            st = E.sweep(max_candidates, max_verify)
            ost = O.sweep(m, max_candidates, max_verify)
            assert (st["scanned"], st["verified"], st["committed"]) == (ost["scanned"], ost["verified"], ost["committed"])
            assert np.array_equal(E.get_mapping(), m)


def test_first_improvement_matches_reference_order():
    z = load_golden("medium_n150")
    O = _oracle(z)
    m = z["map0"].copy()
    with _engine(z) as E:
        E.set_mapping(m)
        s0 = E.score()
        c, p = E.first_improvement(3)
        oc, op, ods = O.first_improvement(m, 3)
        assert (c, p) == (oc, op)
        assert np.array_equal(E.get_mapping(), m)
        assert E.score() == s0 + ods == O.score(m)


@pytest.mark.parametrize("seed", [1, 99])
def test_triple_round_matches_oracle(cfg0, seed):
    g = cfg0
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g) as E:
        E.set_mapping(m)
        # move off the random start first so rounds see both signs
        E.sweep()
        O.sweep(m)
        for r in range(3):
            st = E.triple_round(partners=64, seed=seed + r)
            ost = O.triple_round(m, partners=64, seed=seed + r)
            assert st["triples"] == ost["triples"]
            assert (st["candidates"], st["scanned"], st["verified"], st["committed"]) == \
                   (ost["candidates"], ost["scanned"], ost["verified"], ost["committed"])
            assert st["best_delta"] == ost["best_delta"]
            assert st["score_after"] - st["score_before"] == ost["total_delta"]
            assert np.array_equal(E.get_mapping(), m)
        assert E.score() == O.score(m)


def test_edge_cases_partial_mapping_self_loops_duplicates():
    rng = np.random.default_rng(5)
    n = 70
    s1 = rng.integers(1, n + 1, 500); d1 = rng.integers(1, n + 1, 500); w1 = rng.integers(0, 9, 500)
    s2 = rng.integers(1, n + 1, 500); d2 = rng.integers(1, n + 1, 500); w2 = rng.integers(0, 9, 500)
    m = np.zeros(n + 1, np.int32)
    perm = rng.permutation(n) + 1
    m[1:] = perm
    m[rng.choice(np.arange(1, n + 1), 10, replace=False)] = 0   # ten unmatched vertices
    g = dict(n=n, src1=s1, dst1=d1, w1=w1, src2=s2, dst2=d2, w2=w2)
    O = _oracle(g)
    with _engine(g) as E:
        E.set_mapping(m)
        assert E.score() == O.score(m)
        d = E.all_deltas()
        assert np.array_equal(d, O.all_deltas(m))
        mm = m.copy()
        for _ in range(5):
            st = E.sweep()
            O.sweep(mm)
            assert np.array_equal(E.get_mapping(), mm)
        assert E.score() == O.score(mm)


def test_tiny_and_empty_graphs():
    g = dict(n=2, src1=[1], dst1=[2], w1=[3], src2=[2], dst2=[1], w2=[5])
    with _engine(g) as E:
        E.set_mapping(np.array([0, 1, 2], np.int32))
        assert E.score() == 0
        assert list(E.all_deltas()) == [3]
        st = E.sweep()
        assert st["committed"] == 1 and E.score() == 3
    g = dict(n=5, src1=[], dst1=[], w1=[], src2=[], dst2=[], w2=[])
    with _engine(g) as E:
        E.set_mapping(np.arange(6, dtype=np.int32))
        assert E.score() == 0 and not E.all_deltas().any()
        assert E.sweep()["committed"] == 0


def test_bad_mapping_and_call_order_errors():
    g = dict(n=4, src1=[1, 2], dst1=[2, 3], w1=[1, 1], src2=[1], dst2=[2], w2=[1])
    with _engine(g) as E:
        with pytest.raises(bm.BMError) as e:
            E.sweep()
        assert e.value.status == bm.BM_E_STATE
        with pytest.raises(bm.BMError) as e:
            E.set_mapping(np.array([0, 1, 1, 2, 3], np.int32))   # f1 used twice
        assert e.value.status == bm.BM_E_INPUT
        E.set_mapping(np.array([0, 1, 2, 3, 4], np.int32))
        with pytest.raises(bm.BMError):
            E.pair_deltas([1], [1])
        with pytest.raises(bm.BMError):
            E.triple_deltas([1], [2], [2])


def test_large_weights_use_int32_path():
    rng = np.random.default_rng(3)
    n = 200
    # both sides above 65535 (so 16-bit entries cannot be exact), loads below the overflow guard
    z = dict(n=n, src1=rng.integers(1, n + 1, 3000), dst1=rng.integers(1, n + 1, 3000),
             w1=rng.integers(65536, 10**6, 3000), src2=rng.integers(1, n + 1, 3000),
             dst2=rng.integers(1, n + 1, 3000), w2=rng.integers(65536, 10**6, 3000))
    m = np.zeros(n + 1, np.int32); m[1:] = rng.permutation(n) + 1
    O = _oracle(z)
    with _engine(z) as E:
        assert E.info()["entry_bits"] == 32
        E.set_mapping(m)
        assert E.score() == O.score(m)
        assert np.array_equal(E.all_deltas(), O.all_deltas(m))


def test_hub_gemm_matches_scatter_path(cfg0):
    """The tensor-core hub term (threshold GEMM + residual) gives the same
    profit rows and deltas as scattering every term."""
    g = cfg0
    with _engine(g) as E, _engine(g, bm.BM_FLAG_NO_HUB_GEMM) as F:
        assert E.info()["hubs"] > 0 and F.info()["hubs"] == 0
        E.set_mapping(g["map0"])
        F.set_mapping(g["map0"])
        for a in (1, 2, 500, 1000):
            assert np.array_equal(E.profit_row(a), F.profit_row(a))
        assert np.array_equal(E.all_deltas(), F.all_deltas())


def test_hub_gemm_heavy_weights_against_oracle():
    """Weights far above the GEMM threshold exercise the sparse residual."""
    g = bm.generate(bm.gen_params(n=1500, e=60000, seed=5, wmax=30000, tail_prob=0.3, geom_p=0.1))
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g) as E:
        assert E.info()["hubs"] > 0
        E.set_mapping(m)
        assert np.array_equal(E.all_deltas(), O.all_deltas(m))
        for _ in range(3):
            E.sweep()
            O.sweep(m)
            assert np.array_equal(E.get_mapping(), m)
        assert E.score() == O.score(m)


def test_sweep_rejects_n_beyond_the_set_commit():
    """n = 40,000 leaves too little shared memory for the one-CTA set commit
    (7 bytes per vertex): the sweep says so instead of failing in a launch,
    while pair deltas and the score still work at that size."""
    n = 40_000
    rng = np.random.default_rng(3)
    s = rng.integers(1, n + 1, 20_000).astype(np.int32)
    d = rng.integers(1, n + 1, 20_000).astype(np.int32)
    w = rng.integers(1, 9, 20_000).astype(np.int32)
    m = np.concatenate([[0], rng.permutation(n) + 1]).astype(np.int32)
    with bm.Engine(n, s, d, w, d, s, w) as E:
        E.set_mapping(m)
        assert E.score() >= 0
        assert len(E.pair_deltas([1, 2], [3, 4])) == 2
        with pytest.raises(bm.BMError) as ei:
            E.sweep()
        assert ei.value.status == bm.BM_E_INPUT and "too large" in str(ei.value)


@pytest.mark.parametrize("flags", [0, bm.BM_FLAG_FORCE_I32])
def test_commit_across_ctas_is_identical(cfg0, flags):
    """The set commit split over 1, 2, 8 or 32 CTAs (list scans divided, the
    same ordered decisions in every CTA) commits exactly the same swaps, with
    and without a re-verification budget, and matches the oracle."""
    orc = oracle.Oracle.from_pair(cfg0)
    for max_verify in (-1, 40):
        maps = []
        for ctas in (1, 2, 8, 32):
            with bm.Engine.from_pair(cfg0, flags) as E:
                E.set_mapping(cfg0["map0"])
                for _ in range(4):
                    E.sweep(max_verify=max_verify, commit_ctas=ctas)
                maps.append(E.get_mapping())
        for m in maps[1:]:
            np.testing.assert_array_equal(m, maps[0])
        m = cfg0["map0"].copy()
        for _ in range(4):
            orc.sweep(m, max_verify=max_verify)
        np.testing.assert_array_equal(maps[0], m)


def test_sweeps_at_n_26000_match_oracle():
    """A pair larger than the benchmark's (n = 26,000, sparse): the set
    commit's per-vertex state still fits one CTA's shared memory, and the
    sweeps make the oracle's moves."""
    g = bm.generate(bm.gen_params(n=26000, e=60000, seed=29))
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g) as E:
        E.set_mapping(m)
        for _ in range(2):
            st = E.sweep()
            ost = O.sweep(m)
            assert st["committed"] == ost["committed"] > 0
            assert np.array_equal(E.get_mapping(), m)
        assert E.score() == O.score(m)
