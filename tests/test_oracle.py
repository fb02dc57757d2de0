"""CPU tests: the oracle pinned against the reference (golden fixtures made by
running the reference's own code, and the compiled reference when present)."""
import numpy as np
import pytest

import oracle
from conftest import GOLDEN_CASES, load_golden


def _pair(z):
    return oracle.Oracle(int(z["n"]), z["src1"], z["dst1"], z["w1"], z["src2"], z["dst2"], z["w2"])


@pytest.mark.parametrize("name", GOLDEN_CASES)
def test_oracle_matches_reference_golden(name):
    z = load_golden(name)
    O = _pair(z)
    m = z["map0"]
    assert O.score(m) == int(z["ref_score"])
    d = O.all_deltas(m)
    n = int(z["n"])
    a, b = np.triu_indices(n, 1)
    exact = d[z["pair_idx"]]
    # every delta equals the reference's score difference (exactness)
    assert np.array_equal(exact.astype(np.int64), z["ref_score_diff"])
    if name == "g1_self_loops_n50":
        # the reference delta double-counts G1 self-loops; the oracle is exact
        loops = set(int(s) for s, t in zip(z["src1"], z["dst1"]) if s == t)
        touched = np.array([(x + 1) in loops or (y + 1) in loops for x, y in zip(a, b)])
        assert np.array_equal(d[~touched], z["ref_deltas"][~touched])
        assert (d[touched] != z["ref_deltas"][touched]).any()
    else:
        assert np.array_equal(d, z["ref_deltas"])
    # 3-cycles: local-score differences of the reference's calculate_permutation_delta
    for t, (x, y, w) in enumerate(z["triples"]):
        for rot in range(2):
            ref = int(z["ref_local"][t, 1 + rot] - z["ref_local"][t, 0])
            assert O.triple_delta(m, int(x), int(y), int(w), rot) == ref


def test_oracle_matches_compiled_reference_cfg0(cfg0):
    try:
        R = oracle.RefGAO()
    except OSError:
        pytest.skip("reference not compiled on this machine")
    g = cfg0
    O = oracle.Oracle.from_pair(g)
    gm = R.graph(g["src1"], g["dst1"], g["w1"])
    gf = R.graph(g["src2"], g["dst2"], g["w2"])
    m = g["map0"]
    assert O.score(m) == R.score(gm, gf, m)
    n = g["n"]
    a, b = np.triu_indices(n, 1)
    assert np.array_equal(O.all_deltas(m), R.pair_deltas(gm, gf, m, a + 1, b + 1))


def test_oracle_sweep_rule_properties(cfg0):
    g = cfg0
    O = oracle.Oracle.from_pair(g)
    m = g["map0"].copy()
    s = O.score(m)
    for _ in range(3):
        st = O.sweep(m, want_moves=True)
        s2 = O.score(m)
        assert s2 == s + st["total_delta"]
        assert st["total_delta"] == int(st["moves"][:, 2].sum())
        assert (st["moves"][:, 2] > 0).all()
        assert sorted(m[1:]) == list(range(1, g["n"] + 1))
        s = s2


def test_oracle_rules_from_supplied_deltas_equal_the_full_rules(cfg0):
    """orc_sweep_given / orc_triple_round_given (used where the CPU cannot
    evaluate every pair or triple) make the same moves as the full rules when
    given the oracle's own deltas; a planted delta changes the outcome, so the
    supplied deltas are what decides.  The bulk delta functions equal the
    one-at-a-time ones."""
    g = cfg0
    O = oracle.Oracle.from_pair(g)
    m1, m2 = g["map0"].copy(), g["map0"].copy()
    for caps in ((0, -1), (64, 5)):
        d = O.all_deltas(m1)
        a = O.sweep(m1, *caps, want_moves=True)
        b = O.sweep_given(m2, d, *caps)
        keys = ("total_delta", "candidates", "scanned", "verified", "committed")
        assert {k: a[k] for k in keys} == {k: b[k] for k in keys}
        assert np.array_equal(a["moves"], b["moves"]) and np.array_equal(m1, m2)
    d = O.all_deltas(m1)
    n = g["n"]
    x, y = np.triu_indices(n, 1)
    assert np.array_equal(O.pair_deltas(m1, x[:5000] + 1, y[:5000] + 1), d[:5000])
    d[int(np.argmin(d))] = 10**9
    assert O.sweep_given(m1.copy(), d)["best_delta"] == 10**9
    # the 3-cycle round
    P, seed = 16, 7
    bs, cs = O.triple_samples(seed, P)
    valid = bs > 0
    a = np.repeat(np.arange(1, n + 1, dtype=np.int32), P).reshape(n, P)[valid]
    td = O.triple_deltas(m1, a, bs[valid], cs[valid])
    for i in range(0, len(a), 97):
        for rot in range(2):
            assert td[i, rot] == O.triple_delta(m1, int(a[i]), int(bs[valid][i]), int(cs[valid][i]), rot)
    full = np.zeros((n, P, 2), np.int32)
    full[valid] = td
    r1, r2 = m1.copy(), m1.copy()
    t1 = O.triple_round(r1, partners=P, seed=seed)
    t2 = O.triple_round_given(r2, P, seed, full)
    assert t1 == t2 and t1["triples"] == int(valid.sum()) and np.array_equal(r1, r2)


def test_oracle_first_improvement_terminates():
    z = load_golden("small_n40")
    O = _pair(z)
    m = z["map0"].copy()
    s0 = O.score(m)
    c, passes, dsum = O.first_improvement(m, 1000)
    assert O.score(m) == s0 + dsum
    assert c > 0
    # at the fixed point no swap improves
    assert (O.all_deltas(m) <= 0).all()


def test_oracle_best_swap_descent_against_reference_deltas():
    """Each step of the best-swap descent takes the largest of the compiled
    reference's deltas over all pairs (first in pair order among equals), and
    the score moves by exactly that delta."""
    try:
        R = oracle.RefGAO()
    except OSError:
        pytest.skip("reference not compiled on this machine")
    z = load_golden("small_n40")
    O = _pair(z)
    gm = R.graph(z["src1"], z["dst1"], z["w1"])
    gf = R.graph(z["src2"], z["dst2"], z["w2"])
    n = int(z["n"])
    a, b = np.triu_indices(n, 1)
    m = z["map0"].copy()
    steps = 0
    while True:
        ref = R.pair_deltas(gm, gf, m, a + 1, b + 1)
        mm = m.copy()
        pairs, deltas = O.best_swap_descent(mm, 1)
        if ref.max() <= 0:
            assert len(deltas) == 0
            break
        i = int(np.argmax(ref))
        assert (pairs[0, 0], pairs[0, 1], deltas[0]) == (a[i] + 1, b[i] + 1, ref[i])
        assert O.score(mm) == O.score(m) + int(deltas[0]) == R.score(gm, gf, mm)
        m = mm
        steps += 1
    assert steps > 5


def _permute4(m, s, q):
    import itertools
    perm = list(itertools.permutations(range(4)))[q]
    m2 = m.copy()
    for i in range(4):
        m2[s[i]] = m[s[perm[i]]]
    return m2


def test_quad_delta_matches_reference_permutation_score(cfg0):
    """4-set permutations: the oracle's delta equals the difference of the
    reference's calculate_permutation_delta local score (src/permutation.c)
    before and after permuting the images, for sampled connected 4-sets and
    all 23 permutations."""
    try:
        R = oracle.RefPerm()
    except OSError:
        pytest.skip("reference not compiled on this machine")
    g = cfg0
    O = oracle.Oracle.from_pair(g)
    gm = R.graph(g["src1"], g["dst1"], g["w1"])
    gf = R.graph(g["src2"], g["dst2"], g["w2"])
    m = g["map0"]
    done = 0
    for a in range(1, 200, 7):
        for j in range(3):
            s = O.sample_quad(11, a, j)
            if s is None:
                continue
            st = [a, *s]
            assert len(set(st)) == 4
            before = R.local_score(gm, gf, m, st)
            for q in range(1, 24):
                ref = R.local_score(gm, gf, _permute4(m, st, q), st) - before
                assert O.quad_delta(m, a, s[0], s[1], s[2], q) == ref
            done += 1
    assert done > 40


def test_oracle_quad_round_rule(cfg0):
    g = cfg0
    O = oracle.Oracle.from_pair(g)
    m = g["map0"].copy()
    s = O.score(m)
    for r in range(2):
        st = O.quad_round(m, partners=16, seed=r)
        assert st["committed"] > 0 and st["quads"] > 0
        s2 = O.score(m)
        assert s2 == s + st["total_delta"]
        assert sorted(m[1:]) == list(range(1, g["n"] + 1))
        s = s2


# ---- greedy feature matcher (src/greedy-feature-match.c:527-712) ----

def _write_csv(path, s, d, w):
    with open(path, "w") as f:
        f.write("from,to,weight\n")
        for a, b, c in zip(s, d, w):
            f.write(f"{int(a)},{int(b)},{int(c)}\n")


def _greedy_graph(rng, n, e, zero_w=False, loops=True):
    """Random graph on ids 1..n in which every id appears (a ring), with
    repeated edges and, optionally, self-loops."""
    s = np.concatenate([np.arange(1, n + 1), rng.integers(1, n + 1, e)])
    d = np.concatenate([np.arange(2, n + 2) % n + 0, rng.integers(1, n + 1, e)])
    d[:n][d[:n] == 0] = n
    if not loops:
        keep = s != d
        s, d = s[keep], d[keep]
    s = np.concatenate([s, s[:5]])            # repeated edges
    d = np.concatenate([d, d[:5]])
    w = np.zeros(len(s), np.int32) if zero_w else rng.integers(1, 20, len(s)).astype(np.int32)
    return s.astype(np.int32), d.astype(np.int32), w


def test_greedy_features_and_distance_match_reference(tmp_path):
    try:
        R = oracle.RefGreedy()
    except OSError:
        pytest.skip("reference not compiled on this machine")
    rng = np.random.default_rng(31)
    n = 60
    s, d, w = _greedy_graph(rng, n, 300)
    p = str(tmp_path / "g.csv")
    _write_csv(p, s, d, w)
    g, nn = R.load(p)
    try:
        assert nn == n and np.array_equal(R.node_ids(g, n), np.arange(1, n + 1))
        ref = R.features(g, n)
    finally:
        R.free(g)
    mine = oracle.greedy_features(n, s, d)
    assert np.array_equal(mine, ref[:, :4])
    assert np.array_equal(mine.sum(1), ref[:, 4])
    for _ in range(300):
        f1 = mine[rng.integers(n)]
        f2 = rng.integers(0, 50, 4).astype(np.int32)
        if f2.sum() == 0:
            continue
        assert oracle.greedy_distance(f1, f2) == R.distance(f1, f2)


@pytest.mark.parametrize("seed,n,e", [(5, 40, 160), (6, 40, 160), (7, 40, 160), (8, 150, 900)])
def test_greedy_match_structural_part_matches_reference(tmp_path, seed, n, e):
    """With every G1 weight 0 the align term vanishes in both: the
    reference's own match_vertices then gives the oracle's matching.  (Equal
    totals keep index order in the reference because this C library's qsort
    is a stable merge sort; the oracle and the engine order them by id.)"""
    try:
        R = oracle.RefGreedy()
    except OSError:
        pytest.skip("reference not compiled on this machine")
    rng = np.random.default_rng(seed)
    s1, d1, w1 = _greedy_graph(rng, n, e, zero_w=True)
    s2, d2, w2 = _greedy_graph(rng, n, e)
    p1, p2 = str(tmp_path / "g1.csv"), str(tmp_path / "g2.csv")
    _write_csv(p1, s1, d1, w1)
    _write_csv(p2, s2, d2, w2)
    g1, _ = R.load(p1)
    g2, _ = R.load(p2)
    try:
        ref = R.match(g1, g2, n)
    finally:
        R.free(g1)
        R.free(g2)
    mine = oracle.greedy_match(dict(n=n, src1=s1, dst1=d1, w1=w1, src2=s2, dst2=d2, w2=w2))
    assert np.array_equal(mine[1:], ref)
    assert sorted(mine[1:]) == list(range(1, n + 1))


def test_greedy_match_against_python_restatement():
    """The oracle's align term and tie rule against a plain-Python loop."""
    rng = np.random.default_rng(9)
    n = 30
    s1, d1, w1 = _greedy_graph(rng, n, 120)
    s2, d2, w2 = _greedy_graph(rng, n, 120)
    w2[3] = 0
    g = dict(n=n, src1=s1, dst1=d1, w1=w1, src2=s2, dst2=d2, w2=w2)
    f1 = oracle.greedy_features(n, s1, d1)
    f2 = oracle.greedy_features(n, s2, d2)
    W2 = {}
    for a, b, c in zip(s2, d2, w2):
        W2[(int(a), int(b))] = int(c)                        # last weight wins
    o1 = sorted(range(1, n + 1), key=lambda v: (-int(f1[v - 1].sum()), v))
    o2 = sorted(range(1, n + 1), key=lambda v: (-int(f2[v - 1].sum()), v))
    m = {}
    for v1 in o1:
        best, bg = -np.inf, None
        for v2 in o2:
            if v2 in m.values():
                continue
            al = 0
            for a, b, c in zip(s1, d1, w1):
                if a == v1 and b in m:
                    al += min(int(c), W2.get((v2, m[b]), 0))
                if b == v1 and a in m:
                    al += min(int(c), W2.get((m[a], v2), 0))
            st = -oracle.greedy_distance(f1[v1 - 1], f2[v2 - 1])
            tot = 0.3 * st + 0.7 * al
            if tot > best:
                best, bg = tot, v2
        m[v1] = bg
    mine = oracle.greedy_match(g)
    assert [mine[v] for v in range(1, n + 1)] == [m[v] for v in range(1, n + 1)]
