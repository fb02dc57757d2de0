"""GPU parity of the 4-set permutation moves: exact deltas of given sets and
permutations, and whole rounds (sampling, the 23 permutations of each 4-set
evaluated from the profit matrix, the sequential set commit) bit-identical to
the oracle, in 16- and 32-bit storage and with the re-verification budget."""
import numpy as np
import pytest

import bm
import oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("flags", [0, bm.BM_FLAG_FORCE_I32])
def test_quad_deltas_match_oracle(cfg0, flags):
    O = oracle.Oracle.from_pair(cfg0)
    m = cfg0["map0"]
    sets, perms, want = [], [], []
    for a in range(1, 400, 3):
        s = O.sample_quad(5, a, a % 7)
        if s is None:
            continue
        q = 1 + (a % 23)
        sets.append([a, *s])
        perms.append(q)
        want.append(O.quad_delta(m, a, s[0], s[1], s[2], q))
    with bm.Engine.from_pair(cfg0, flags) as E:
        E.set_mapping(m)
        got = E.quad_deltas(np.array(sets), np.array(perms))
    np.testing.assert_array_equal(got, np.array(want))


@pytest.mark.parametrize("flags,max_verify", [(0, -1), (bm.BM_FLAG_FORCE_I32, -1), (0, 25)])
def test_quad_rounds_match_oracle(cfg0, flags, max_verify):
    O = oracle.Oracle.from_pair(cfg0)
    m = cfg0["map0"].copy()
    with bm.Engine.from_pair(cfg0, flags) as E:
        E.set_mapping(m)
        for r in range(3):
            st = E.quad_round(partners=24, seed=100 + r, max_verify=max_verify)
            ost = O.quad_round(m, partners=24, seed=100 + r, max_verify=max_verify)
            for k in ("committed", "candidates", "scanned", "verified", "best_delta"):
                assert st[k] == ost[k], k
            assert st["quads"] == ost["quads"]
            assert st["score_after"] - st["score_before"] == ost["total_delta"]
            np.testing.assert_array_equal(E.get_mapping(), m)
            assert E.score() == O.score(m)


def test_quad_after_sweeps_improves_a_local_optimum(cfg0):
    """At a local optimum of pairwise swaps, 4-set moves still find exact
    improvements (the oracle agrees on every one)."""
    O = oracle.Oracle.from_pair(cfg0)
    with bm.Engine.from_pair(cfg0) as E:
        E.set_mapping(cfg0["map0"])
        for _ in range(200):
            if E.sweep()["committed"] == 0:
                break
        m = E.get_mapping()
        st = E.quad_round(partners=64, seed=7)
        ost = O.quad_round(m, partners=64, seed=7)
        assert st["committed"] == ost["committed"]
        np.testing.assert_array_equal(E.get_mapping(), m)
        assert st["score_after"] >= st["score_before"]


def test_quad_arguments_are_checked(cfg0):
    with bm.Engine.from_pair(cfg0) as E:
        E.set_mapping(cfg0["map0"])
        with pytest.raises(bm.BMError):
            E.quad_deltas(np.array([[1, 2, 3, 3]]), np.array([1]))
        with pytest.raises(bm.BMError):
            E.quad_deltas(np.array([[1, 2, 3, 4]]), np.array([24]))
        with pytest.raises(bm.BMError):
            E.quad_round(partners=4096)
