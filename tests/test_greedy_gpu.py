"""GPU parity of the greedy feature matcher (src/greedy-feature-match.c:
527-712): features and the whole matching bit-identical to the oracle."""
import numpy as np
import pytest

import bm
import oracle

pytestmark = pytest.mark.gpu


def _rand_graph(rng, n, e, wmax=20):
    s = rng.integers(1, n + 1, e).astype(np.int32)
    d = rng.integers(1, n + 1, e).astype(np.int32)
    w = rng.integers(0, wmax, e).astype(np.int32)        # zero weights, self-loops, repeats
    s = np.concatenate([s, s[:7]]); d = np.concatenate([d, d[:7]]); w = np.concatenate([w, w[7:14] + 1])
    return s, d, w


def test_features_match_oracle(cfg0):
    g = cfg0
    n = int(g["n"])
    for k in ("1", "2"):
        mine = bm.greedy_features(n, g["src" + k], g["dst" + k], g["w" + k])
        assert np.array_equal(mine, oracle.greedy_features(n, g["src" + k], g["dst" + k]))
    rng = np.random.default_rng(3)
    s, d, w = _rand_graph(rng, 300, 2000)
    assert np.array_equal(bm.greedy_features(310, s, d, w), oracle.greedy_features(310, s, d))  # isolated ids


def test_match_cfg0_identical(cfg0):
    m, st = bm.greedy_match(cfg0)
    assert np.array_equal(m, oracle.greedy_match(cfg0))
    assert sorted(m[1:]) == list(range(1, int(cfg0["n"]) + 1))
    assert st["ms_match"] > 0


@pytest.mark.parametrize("seed", [1, 2])
def test_match_edge_cases_identical(seed):
    rng = np.random.default_rng(seed)
    n = 257
    s1, d1, w1 = _rand_graph(rng, n - 6, 3000)        # the last ids have no edges in G1
    s2, d2, w2 = _rand_graph(rng, n, 2500)
    g = dict(n=n, src1=s1, dst1=d1, w1=w1, src2=s2, dst2=d2, w2=w2)
    m, _ = bm.greedy_match(g)
    assert np.array_equal(m, oracle.greedy_match(g))


def test_match_tiny_and_empty():
    g = dict(n=1, src1=[], dst1=[], w1=[], src2=[], dst2=[], w2=[])
    m, _ = bm.greedy_match(g)
    assert list(m) == [0, 1]
    g = dict(n=3, src1=[1, 2], dst1=[2, 3], w1=[5, 1], src2=[3, 1], dst2=[1, 2], w2=[4, 9])
    m, _ = bm.greedy_match(g)
    assert np.array_equal(m, oracle.greedy_match(g))
    with pytest.raises(bm.BMError):
        bm.greedy_match(dict(n=3, src1=[1], dst1=[4], w1=[1], src2=[], dst2=[], w2=[]))


def test_match_larger_identical_and_scores():
    g = bm.generate(bm.gen_params(n=4000, e=80000, seed=17))
    m, st = bm.greedy_match(g)
    assert np.array_equal(m, oracle.greedy_match(g))
    with bm.Engine.from_pair(g) as E:
        E.set_mapping(m)
        greedy = E.score()
        E.set_mapping(g["map0"])
        assert greedy > E.score()     # better than a random start
