"""GPU parity of the exact swap-lookup table: the profit matrix kept exact
across commits by the moved-vertex update (sweeps with incremental=True), its
delta rows, and the best-swap descent (src/best-swap/score-lookup.c:597-640
with an exact table) against the oracle."""
import numpy as np
import pytest

import bm
import oracle

pytestmark = pytest.mark.gpu


def _engine(g, flags=0):
    return bm.Engine(int(g["n"]), g["src1"], g["dst1"], g["w1"], g["src2"], g["dst2"], g["w2"], flags)


def _oracle(g):
    return oracle.Oracle(int(g["n"]), g["src1"], g["dst1"], g["w1"], g["src2"], g["dst2"], g["w2"])


def _table(O, m):
    """Full n x n delta table of the oracle (0 on the diagonal)."""
    n = O.n
    d = O.all_deltas(m)
    t = np.zeros((n, n), np.int32)
    a, b = np.triu_indices(n, 1)
    t[a, b] = d
    t[b, a] = d
    return t


@pytest.mark.parametrize("flags", [0, bm.BM_FLAG_FORCE_I32, bm.BM_FLAG_NO_HUB_GEMM])
def test_incremental_sweeps_identical_to_rebuilt(cfg0, flags):
    """Sweeps that update the profit matrix from the moved vertices give the
    same candidates, commits and mappings as sweeps that rebuild it, and the
    maintained table equals the oracle's deltas at the end."""
    g = cfg0
    modes = []
    with _engine(g, flags) as E, _engine(g, flags) as F:
        E.set_mapping(g["map0"])
        F.set_mapping(g["map0"])
        for it in range(200):
            a = E.sweep(incremental=True)
            b = F.sweep()
            modes.append(a["profit_mode"])
            for k in ("candidates", "best_delta", "committed", "verified", "score_after"):
                assert a[k] == b[k], (it, k)
            assert np.array_equal(E.get_mapping(), F.get_mapping()), it
            if b["committed"] == 0:
                break
        assert 1 in modes, modes            # the update path ran
        assert modes[0] == 0                # the first sweep builds the matrix
        m = E.get_mapping()
        O = _oracle(g)
        assert np.array_equal(E.lookup_rows(1, int(g["n"])), _table(O, m))


def test_incremental_after_other_moves(cfg0):
    """3-cycle rounds and a new mapping between incremental sweeps: the
    matrix follows whatever changed the matching."""
    g = cfg0
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g) as E:
        E.set_mapping(m)
        for _ in range(3):
            E.sweep(incremental=True)
            O.sweep(m)
        E.triple_round(partners=64, seed=3)
        O.triple_round(m, partners=64, seed=3)
        assert np.array_equal(E.get_mapping(), m)
        st = E.sweep(incremental=True)
        O.sweep(m)
        assert np.array_equal(E.get_mapping(), m)
        rng = np.random.default_rng(4)
        m2 = m.copy()
        sel = rng.choice(np.arange(1, int(g["n"]) + 1), 40, replace=False)
        m2[sel] = m2[rng.permutation(sel)]
        E.set_mapping(m2)
        st = E.sweep(incremental=True)
        O.sweep(m2)
        assert np.array_equal(E.get_mapping(), m2)
        assert E.score() == O.score(m2) == st["score_after"]


def test_lookup_rows_match_oracle(cfg0):
    g = cfg0
    n = int(g["n"])
    O = _oracle(g)
    with _engine(g) as E:
        E.set_mapping(g["map0"])
        t = _table(O, g["map0"])
        assert np.array_equal(E.lookup_rows(1, n), t)
        assert np.array_equal(E.lookup_rows(500, 7), t[499:506])
        assert E.lookup_rows(n, 1).shape == (1, n)
        with pytest.raises(bm.BMError):
            E.lookup_rows(n, 2)
        with pytest.raises(bm.BMError):
            E.lookup_rows(0, 1)


@pytest.mark.parametrize("flags", [0, bm.BM_FLAG_FORCE_I32])
def test_best_swap_descent_matches_oracle(flags):
    """Largest-delta-first single swaps on the exact table: the same swaps,
    in the same order, as the oracle's full re-evaluation at every step."""
    g = bm.generate(bm.gen_params(n=300, e=6000, seed=11))
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g, flags) as E:
        E.set_mapping(m)
        st = E.lookup_descent(150)
        pairs, deltas = O.best_swap_descent(m, 150)
        assert st["swaps"] == len(deltas)
        assert st["score_after"] - st["score_before"] == int(deltas.sum())
        assert np.array_equal(E.get_mapping(), m)
        assert E.score() == O.score(m) == st["score_after"]
        # the table after the descent is the oracle's
        assert np.array_equal(E.lookup_rows(1, 300), _table(O, m))


def test_best_swap_descent_to_convergence_with_unmatched_vertices():
    rng = np.random.default_rng(7)
    n = 120
    s1 = rng.integers(1, n + 1, 900); d1 = rng.integers(1, n + 1, 900); w1 = rng.integers(1, 9, 900)
    s2 = rng.integers(1, n + 1, 900); d2 = rng.integers(1, n + 1, 900); w2 = rng.integers(1, 9, 900)
    keep1, keep2 = s1 != d1, s2 != d2
    g = dict(n=n, src1=s1[keep1], dst1=d1[keep1], w1=w1[keep1], src2=s2[keep2], dst2=d2[keep2], w2=w2[keep2])
    m = np.zeros(n + 1, np.int32)
    m[1:] = rng.permutation(n) + 1
    m[rng.choice(np.arange(1, n + 1), 12, replace=False)] = 0
    O = _oracle(g)
    with _engine(g) as E:
        E.set_mapping(m)
        st = E.lookup_descent(100000)
        pairs, deltas = O.best_swap_descent(m, 100000)
        assert st["converged"] == 1
        assert st["swaps"] == len(deltas)
        assert np.array_equal(E.get_mapping(), m)
        assert E.score() == O.score(m)
        # converged: no improving pair remains in the exact table
        assert E.lookup_rows(1, n).max() <= 0
        # a second call has nothing to do
        st2 = E.lookup_descent(10)
        assert st2["swaps"] == 0 and st2["converged"] == 1 and st2["refresh_mode"] == 2


@pytest.mark.parametrize("flags", [0, bm.BM_FLAG_FORCE_I32])
def test_dense_graph_row_path_identical(flags):
    """A dense pair (average degree 100 in each direction, n = 600): the two
    G2 lists of almost every moved vertex cover a quarter of its row, so the
    update sums each edge's terms in shared memory and writes the row whole.
    Sweeps and the best-swap descent must still equal the oracle."""
    g = bm.generate(bm.gen_params(n=600, e=60000, seed=23))
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g, flags) as E:
        E.set_mapping(m)
        modes = []
        for _ in range(60):
            st = E.sweep(incremental=True)
            O.sweep(m)
            modes.append(st["profit_mode"])
            assert np.array_equal(E.get_mapping(), m)
            if st["committed"] == 0:
                break
        assert np.array_equal(E.lookup_rows(1, 600), _table(O, m))
        m2 = g["map0"].copy()
        E.set_mapping(m2)
        st = E.lookup_descent(60)
        O.best_swap_descent(m2, 60)
        assert np.array_equal(E.get_mapping(), m2) and E.score() == O.score(m2) == st["score_after"]
        assert np.array_equal(E.lookup_rows(1, 600), _table(O, m2))


@pytest.mark.parametrize("flags", [0, bm.BM_FLAG_FORCE_I32])
def test_incremental_triple_and_quad_rounds_match_oracle(cfg0, flags):
    """3-cycle and 4-set rounds that update the profit matrix from the
    previous round's moves make the oracle's moves, round after round."""
    g = cfg0
    O = _oracle(g)
    m = g["map0"].copy()
    with _engine(g, flags) as E:
        E.set_mapping(m)
        for _ in range(4):
            E.sweep(incremental=True)
            O.sweep(m)
        modes = []
        for r in range(4):
            st = E.triple_round(partners=64, seed=40 + r, incremental=True)
            ost = O.triple_round(m, partners=64, seed=40 + r)
            assert st["committed"] == ost["committed"]
            assert np.array_equal(E.get_mapping(), m)
            st = E.quad_round(partners=32, seed=80 + r, incremental=True)
            ost = O.quad_round(m, partners=32, seed=80 + r)
            assert st["committed"] == ost["committed"]
            assert np.array_equal(E.get_mapping(), m)
        assert E.score() == O.score(m)
        assert np.array_equal(E.lookup_rows(1, int(g["n"])), _table(O, m))
