"""CPU tests of the timed CPU legs' inputs and harnesses: the generator the
CPU legs load (oracle/_ref/libgen.so) makes the engine's workloads bit for bit,
and the reference's own loops driven by oracle/ref_harness_*.c agree with the
oracle restatement they are timed beside."""
import numpy as np
import pytest

import bm
import oracle


@pytest.mark.parametrize("kw", [dict(), dict(n=3000, e=90_000, wmax=30000, tail_prob=1e-3, seed=20261204)])
def test_cpu_generator_equals_engine_generator(kw):
    a = oracle.generate(**kw)
    b = bm.generate(bm.gen_params(**kw))
    assert a.keys() == b.keys()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_reference_first_improvement_equals_oracle(cfg0):
    try:
        R = oracle.RefGAO()
    except OSError:
        pytest.skip("reference not compiled on this machine")
    g = cfg0
    O = oracle.Oracle.from_pair(g)
    gm = R.graph(g["src1"], g["dst1"], g["w1"])
    gf = R.graph(g["src2"], g["dst2"], g["w2"])
    m1, m2 = g["map0"].copy(), g["map0"].copy()
    s0 = O.score(m1)
    score, commits, passes = R.first_improvement(gm, gf, m1, g["n"], 1000)
    oc, op, ods = O.first_improvement(m2, 1000)
    assert (O.all_deltas(m1) <= 0).all()   # the fixed point
    assert (commits, passes) == (oc, op)
    assert np.array_equal(m1, m2)
    assert score == s0 + ods == O.score(m1)
    R.free(gm)
    R.free(gf)


def test_reference_triple_rotations_equal_oracle(cfg0):
    try:
        RP = oracle.RefPerm()
    except OSError:
        pytest.skip("reference not compiled on this machine")
    g = cfg0
    O = oracle.Oracle.from_pair(g)
    gm = RP.graph(g["src1"], g["dst1"], g["w1"])
    gf = RP.graph(g["src2"], g["dst2"], g["w2"])
    bs, cs = O.triple_samples(3, 8)
    valid = bs > 0
    a = np.repeat(np.arange(1, g["n"] + 1, dtype=np.int32), 8).reshape(g["n"], 8)[valid]
    got, nt = RP.triples_omp(gm, gf, g["map0"], a, bs[valid], cs[valid])
    assert nt >= 1
    assert np.array_equal(got, O.triple_deltas(g["map0"], a, bs[valid], cs[valid]))
    RP.free(gm)
    RP.free(gf)


def test_reference_racy_rows_run_and_lose_images(cfg0):
    """The racy tool's loop evaluates every partner of every listed row and
    commits improving swaps.  It reads both images before taking its critical
    section (src/graph-alignment-optimized-parallel.c:549-565), so two commits
    in one row can give one G2 vertex to two G1 vertices: on this workload the
    matching stops being a permutation, which is why it is timed only as an
    upper bound and never used as an oracle."""
    try:
        RQ = oracle.RefPar()
    except OSError:
        pytest.skip("reference not compiled on this machine")
    g = cfg0
    gm = RQ.graph(g["src1"], g["dst1"], g["w1"])
    gf = RQ.graph(g["src2"], g["dst2"], g["w2"])
    m = g["map0"].copy()
    cnt, commits, nt = RQ.rows(gm, gf, m, np.arange(1, 41, dtype=np.int32), g["n"])
    assert cnt == 40 * (g["n"] - 1) and commits > 0 and nt >= 1
    if nt > 1:
        assert len(np.unique(m[1:])) <= g["n"]
    RQ.free(gm)
    RQ.free(gf)
