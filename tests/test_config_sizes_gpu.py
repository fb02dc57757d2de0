"""GPU parity at the benchmark workloads' own sizes.

* The pairwise sweep on the N=18,524 / 5,000,000-edge pair (the headline
  workload, seed 20261204): per sweep, >= 256 full rows of deltas (the
  heaviest G1 vertices, rows whose G2 lists exceed the profit kernel's
  long-list threshold, seeded random rows) equal the compiled reference's
  calculate_swap_delta (src/graph-alignment-optimized.c:321-408); the
  sweep's set commit equals the oracle's rule run on the engine's own deltas;
  every committed move's delta equals the reference's on the matching it was
  committed to; the score equals the reference's calculate_alignment_score.
  A second context keeps the profit matrix updated from the moved vertices
  and must make the same moves.
* One 3-cycle round with 256 two-hop partners per vertex on that pair.
* The 64-instance batch (N log-uniform in 500..8,000, E = 20 N): every
  instance against a single-instance context, four (the largest included)
  against the oracle's full sweep.

A full CPU evaluation of one N=18,524 sweep (1.7e8 deltas) or triple round
(9.5e6 rotations) takes minutes, so the deltas are checked by sampling and the
oracle's selection rules run on the engine's deltas (orc_sweep_given,
orc_triple_round_given).
"""
import numpy as np
import pytest

import bm
import oracle

pytestmark = pytest.mark.gpu

CFG1 = dict(n=18524, e=5_000_000, wmax=30000, tail_prob=1e-3, seed=20261204)
LONG_LIST = 2048   # the profit kernel scatters G2 lists longer than this with the whole CTA
HUB_T = 8          # the hub GEMM covers in-edge terms up to this weight


@pytest.fixture(scope="module")
def cfg1():
    return bm.generate(bm.gen_params(**CFG1))


@pytest.fixture(scope="module")
def ref(cfg1):
    """The compiled reference over the pair, or None where it was not built
    (the oracle's swap delta, pinned to it by tests/test_oracle.py, stands in)."""
    try:
        R = oracle.RefGAO()
    except OSError:
        yield None
        return
    gm = R.graph(cfg1["src1"], cfg1["dst1"], cfg1["w1"])
    gf = R.graph(cfg1["src2"], cfg1["dst2"], cfg1["w2"])
    yield R, gm, gf
    R.L.refgao_graph_free(gm)
    R.L.refgao_graph_free(gf)


def _ref_deltas(ref, O, m, a, b):
    if ref is None:
        return O.pair_deltas(m, a, b)
    R, gm, gf = ref
    return R.pair_deltas(gm, gf, m, a, b)


def _g2_degrees(g):
    """Out- and in-degree of every G2 vertex as the engine stores G2: one
    entry per (src, dst), the last weight given wins, zero weights dropped."""
    n = int(g["n"])
    s, d, w = (np.asarray(g[k], np.int64) for k in ("src2", "dst2", "w2"))
    key = s * (n + 1) + d
    _, first_rev = np.unique(key[::-1], return_index=True)
    last = len(key) - 1 - first_rev
    keep = last[w[last] > 0]
    return np.bincount(s[keep], minlength=n + 1), np.bincount(d[keep], minlength=n + 1)


def _hubs(g, nh):
    """The G1 vertices (1-based) whose in-edge terms the hub GEMM covers: the
    nh largest out-degrees, ties by id."""
    n = int(g["n"])
    deg = np.bincount(np.asarray(g["src1"]) - 1, minlength=n)
    return np.argsort(-deg, kind="stable")[:nh] + 1


def _long_list_rows(g, m, hub_set, out2, in2):
    """Rows a whose profit row scatters a G2 list longer than LONG_LIST: an
    in-edge u -> a (u no hub) with |out2(m[u])| > LONG_LIST, or an out-edge
    a -> v with |in2(m[v])| > LONG_LIST."""
    s = np.asarray(g["src1"])
    d = np.asarray(g["dst1"])
    lu = out2[m[s]] * (m[s] > 0)
    rows_in = d[(lu > LONG_LIST) & ~np.isin(s, hub_set)]
    lv = in2[m[d]] * (m[d] > 0)
    rows_out = s[lv > LONG_LIST]
    return np.unique(np.concatenate([rows_in, rows_out]))


def _rows_from_condensed(D, n, rows):
    """[len(rows), n-1] deltas of each row against every other vertex,
    partners ascending, from the linear pair order."""
    b = np.arange(1, n + 1, dtype=np.int64)
    out = []
    for a in rows:
        bb = b[b != a]
        lo = np.minimum(a, bb)
        hi = np.maximum(a, bb)
        out.append(D[(lo - 1) * (2 * n - lo) // 2 + (hi - lo - 1)])
    return np.stack(out)


def _best(vals, partners):
    """Per row: the largest delta and its partner (the smallest id among equals)."""
    k = np.argmax(vals, axis=1)
    r = np.arange(len(k))
    return vals[r, k], partners[r, k]


def test_config1_sweeps_bit_exact_against_reference(cfg1, ref):
    g = cfg1
    n = int(g["n"])
    O = oracle.Oracle.from_pair(g)
    out2, in2 = _g2_degrees(g)
    deg = np.bincount(np.asarray(g["src1"]) - 1, minlength=n) + np.bincount(np.asarray(g["dst1"]) - 1, minlength=n)
    heaviest = np.argsort(-deg, kind="stable")[:32] + 1
    rng = np.random.default_rng(20261204)
    m = g["map0"].copy()
    with bm.Engine.from_pair(g) as E, bm.Engine.from_pair(g) as F:
        info = E.info()
        assert info["entry_bits"] == 16 and info["n"] == n
        assert info["hubs"] > 0 and info["hub_k"] == info["hubs"] * HUB_T
        hub_set = _hubs(g, info["hubs"])
        # hub in-edges heavier than the GEMM threshold go through the residual list
        assert (np.isin(g["src1"], hub_set) & (np.asarray(g["w1"]) > HUB_T)).any()
        E.set_mapping(m)
        F.set_mapping(m)
        assert E.score() == O.score(m)
        if ref:
            assert ref[0].score(ref[1], ref[2], m) == O.score(m)
        modes = []
        # (max_candidates, rows checked): three full sweeps, then capped sweeps
        # that move few vertices, so the second context updates S from them
        plans = [(0, 256), (0, 96), (0, 96), (64, 32), (64, 32), (64, 32)]
        for it, (cap, nrows) in enumerate(plans):
            D = E.all_deltas()
            longr = _long_list_rows(g, m, hub_set, out2, in2)
            assert len(longr) >= 8, "the sample must send lists through the long-list queue"
            pick = list(heaviest[:16]) + list(rng.choice(longr, min(16, len(longr)), replace=False))
            rest = np.setdiff1d(np.arange(1, n + 1), pick)
            pick += list(rng.choice(rest, nrows - len(pick), replace=False))
            pick = np.array(pick, np.int64)
            got = _rows_from_condensed(D, n, pick)
            partners = np.stack([np.delete(np.arange(1, n + 1), a - 1) for a in pick])
            want = _ref_deltas(ref, O, m, np.repeat(pick, n - 1), partners.ravel()).reshape(len(pick), n - 1)
            bad = np.argwhere(got != want)
            assert len(bad) == 0, f"sweep {it}: {len(bad)} deltas differ, first in row {pick[bad[0][0]]}"
            gb, gp = _best(got, partners)
            wb, wp = _best(want, partners)
            assert np.array_equal(gb, wb) and np.array_equal(gp, wp)
            # the set commit: the oracle's rule on the engine's deltas
            m_before = m.copy()
            ost = O.sweep_given(m, D, max_candidates=cap)
            st = E.sweep(max_candidates=cap)
            fst = F.sweep(max_candidates=cap, incremental=True)
            modes.append(fst["profit_mode"])
            for s in (st, fst):
                assert (s["candidates"], s["scanned"], s["verified"], s["committed"], s["best_delta"]) == \
                       (ost["candidates"], ost["scanned"], ost["verified"], ost["committed"], ost["best_delta"]), it
                assert s["score_after"] - s["score_before"] == ost["total_delta"]
            assert ost["committed"] > 0
            assert np.array_equal(E.get_mapping(), m), it
            assert np.array_equal(F.get_mapping(), m), it
            # every committed delta, on the matching it was committed to
            r = m_before.copy()
            for lo, hi, d in ost["moves"]:
                assert _ref_deltas(ref, O, r, [lo], [hi])[0] == d, (it, lo, hi)
                r[lo], r[hi] = r[hi], r[lo]
            assert np.array_equal(r, m)
            sc = O.score(m)
            assert E.score() == F.score() == st["score_after"] == sc
            if ref:
                assert ref[0].score(ref[1], ref[2], m) == sc
        assert 1 in modes[3:], modes


def test_config2_triple_round_at_full_size(cfg1):
    """One 3-cycle round, 256 two-hop partners per vertex (4.7e6 triples), on
    the pair after two sweeps: sampled rotation deltas equal the oracle's and
    the reference's local-score differences (src/permutation.c:623-696), and
    the round commits what the oracle's rule commits on the engine's deltas."""
    g = cfg1
    n, P, seed = int(g["n"]), 256, 4242
    O = oracle.Oracle.from_pair(g)
    with bm.Engine.from_pair(g) as E:
        E.set_mapping(g["map0"])
        E.sweep()
        E.sweep()
        m = E.get_mapping()
        bs, cs = O.triple_samples(seed, P)
        valid = bs > 0
        a = np.repeat(np.arange(1, n + 1, dtype=np.int32), P).reshape(n, P)[valid]
        b, c = bs[valid], cs[valid]
        assert len(a) > 4_000_000
        td = E.triple_deltas(a, b, c)
        rng = np.random.default_rng(7)
        deg = np.bincount(np.asarray(g["src1"]) - 1, minlength=n)
        heavy = np.flatnonzero(np.isin(a, np.argsort(-deg)[:16] + 1))
        sample = np.concatenate([rng.choice(len(a), 40_000, replace=False), rng.choice(heavy, 2_000, replace=False)])
        assert np.array_equal(td[sample], O.triple_deltas(m, a[sample], b[sample], c[sample]))
        try:
            RP = oracle.RefPerm()
        except OSError:
            RP = None
        if RP is not None:
            # the reference's local score deduplicates edges by a linear scan
            # (quadratic in the set's degree), so it checks 300 of the triples
            gm = RP.graph(g["src1"], g["dst1"], g["w1"])
            gf = RP.graph(g["src2"], g["dst2"], g["w2"])
            few = sample[:300]
            rd, _ = RP.triples_omp(gm, gf, m, a[few], b[few], c[few])
            assert np.array_equal(rd, td[few])
            RP.free(gm)
            RP.free(gf)
        full = np.zeros((n, P, 2), np.int32)
        full[valid] = td
        ost = O.triple_round_given(m, P, seed, full)
        st = E.triple_round(partners=P, seed=seed)
        assert st["triples"] == ost["triples"]
        assert (st["candidates"], st["scanned"], st["verified"], st["committed"], st["best_delta"]) == \
               (ost["candidates"], ost["scanned"], ost["verified"], ost["committed"], ost["best_delta"])
        assert ost["committed"] > 0
        assert st["score_after"] - st["score_before"] == ost["total_delta"]
        assert np.array_equal(E.get_mapping(), m)
        assert E.score() == O.score(m)


def _batch_pairs(seed=20261207, count=64):
    """The 64-instance batch workload: N log-uniform in [500, 8000], E = 20 N."""
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(500), np.log(8000), count)).astype(int)
    return [bm.generate(bm.gen_params(n=int(k), e=20 * int(k), seed=seed + 1 + i)) for i, k in enumerate(ns)]


def test_config3_batch64_against_single_instances_and_oracle():
    pairs = _batch_pairs()
    ns = [int(p["n"]) for p in pairs]
    big, small = int(np.argmax(ns)), int(np.argmin(ns))
    others = [int(i) for i in np.random.default_rng(11).permutation(64) if i not in (big, small)]
    check = [big, small, others[0], others[1]]
    orcs = {i: oracle.Oracle.from_pair(pairs[i]) for i in check}
    maps = {i: pairs[i]["map0"].copy() for i in check}
    with bm.Batch(pairs) as B:
        assert B.info()["count"] == 64 and B.info()["max_n"] == max(ns)
        B.set_mappings([p["map0"] for p in pairs])
        B.autotune()
        B.set_mappings([p["map0"] for p in pairs])
        singles = [bm.Engine.from_pair(p) for p in pairs]
        try:
            for E, p in zip(singles, pairs):
                E.set_mapping(p["map0"])
            for it in range(3):
                commits, _ = B.sweeps(1)
                got = B.get_mappings()
                for k, E in enumerate(singles):
                    st = E.sweep()
                    assert commits[k] == st["committed"], (it, k)
                    assert np.array_equal(got[k], E.get_mapping()), (it, k)
                for i in check:
                    ost = orcs[i].sweep(maps[i])
                    assert commits[i] == ost["committed"], (it, i)
                    assert np.array_equal(got[i], maps[i]), (it, i)
            sc = B.scores()
            for i in check:
                assert sc[i] == orcs[i].score(maps[i])
        finally:
            for E in singles:
                E.close()
