"""Generates the golden fixtures in this directory from the REFERENCE itself.

Run here (where the reference tree exists), after `make -C oracle ref`:
    python tests/golden/make_golden.py
Each case is a small graph pair, a matching, and outputs of the reference's
own code compiled in place (oracle/_ref/librefgao.so = reference
src/graph-alignment-optimized.c, oracle/_ref/librefperm.so = reference
src/permutation.c): the alignment score, every swap delta in linear pair
order, and 3-cycle local scores before/after each rotation.  The fixtures are
committed so tests can pin the oracle on machines without the reference.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402


def rand_pair(rng, n, e, wmax, self_loops=0, dup_g2=0):
    """Random directed pair without G1 self-loops/duplicates unless asked."""
    pairs = set()
    s1, d1 = [], []
    while len(s1) < e:
        a, b = int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))
        if a == b or (a, b) in pairs:
            continue
        pairs.add((a, b))
        s1.append(a); d1.append(b)
    w1 = list(rng.integers(1, wmax + 1, size=e))
    for _ in range(self_loops):
        a = int(rng.integers(1, n + 1))
        if (a, a) in pairs:
            continue
        pairs.add((a, a)); s1.append(a); d1.append(a); w1.append(int(rng.integers(1, wmax + 1)))
    pi = rng.permutation(n) + 1
    s2 = [int(pi[a - 1]) for a in s1]
    d2 = [int(pi[b - 1]) for b in d1]
    w2 = [max(1, int(w) + int(rng.integers(-1, 2))) for w in w1]
    keep = rng.random(len(s2)) > 0.15
    s2 = [x for x, k in zip(s2, keep) if k]; d2 = [x for x, k in zip(d2, keep) if k]; w2 = [x for x, k in zip(w2, keep) if k]
    for _ in range(e // 10):
        a, b = int(rng.integers(1, n + 1)), int(rng.integers(1, n + 1))
        s2.append(a); d2.append(b); w2.append(int(rng.integers(1, wmax + 1)))
    for _ in range(dup_g2):   # repeated G2 edges: the reference keeps the last weight
        i = int(rng.integers(0, len(s2)))
        s2.append(s2[i]); d2.append(d2[i]); w2.append(int(rng.integers(1, wmax + 1)))
    m = np.zeros(n + 1, np.int32)
    m[1:] = rng.permutation(n) + 1
    A = lambda x: np.asarray(x, np.int32)
    return dict(n=n, src1=A(s1), dst1=A(d1), w1=A(w1), src2=A(s2), dst2=A(d2), w2=A(w2), map0=m)


def main():
    R = oracle.RefGAO()
    P = oracle.RefPerm()
    cases = [
        ("small_n40", dict(n=40, e=220, wmax=9), 11),
        ("medium_n150", dict(n=150, e=1500, wmax=40), 12),
        ("heavy_weights_n80", dict(n=80, e=600, wmax=30000), 13),
        ("g2_duplicates_n60", dict(n=60, e=400, wmax=12, dup_g2=30), 14),
        ("g1_self_loops_n50", dict(n=50, e=300, wmax=7, self_loops=8), 15),
    ]
    for name, kw, seed in cases:
        rng = np.random.default_rng(seed)
        g = rand_pair(rng, **kw)
        n = g["n"]
        gm = R.graph(g["src1"], g["dst1"], g["w1"])
        gf = R.graph(g["src2"], g["dst2"], g["w2"])
        m = g["map0"]
        a, b = np.triu_indices(n, 1)
        deltas = R.pair_deltas(gm, gf, m, a + 1, b + 1)
        score = R.score(gm, gf, m)
        # exact deltas via the reference's own score: score(after swap) - score(before)
        k = min(300, len(a))
        idx = rng.choice(len(a), size=k, replace=False)
        diff = np.zeros(k, np.int64)
        for t, i in enumerate(idx):
            m2 = m.copy(); x, y = a[i] + 1, b[i] + 1
            m2[x], m2[y] = m2[y], m2[x]
            diff[t] = R.score(gm, gf, m2) - score
        # 3-cycles: reference local scores before / after each rotation
        pm = P.graph(g["src1"], g["dst1"], g["w1"])
        pf = P.graph(g["src2"], g["dst2"], g["w2"])
        trip = np.zeros((60, 3), np.int32)
        loc = np.zeros((60, 3), np.int64)
        for t in range(60):
            v = rng.choice(n, size=3, replace=False) + 1
            trip[t] = v
            loc[t, 0] = P.local_score(pm, pf, m, v)
            for rot in range(2):
                m2 = m.copy(); fa, fb, fc = m[v[0]], m[v[1]], m[v[2]]
                if rot == 0: m2[v[0]], m2[v[1]], m2[v[2]] = fb, fc, fa
                else:        m2[v[0]], m2[v[1]], m2[v[2]] = fc, fa, fb
                loc[t, 1 + rot] = P.local_score(pm, pf, m2, v)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), n=n, src1=g["src1"], dst1=g["dst1"], w1=g["w1"],
                            src2=g["src2"], dst2=g["dst2"], w2=g["w2"], map0=m, ref_deltas=deltas,
                            ref_score=score, pair_idx=idx, ref_score_diff=diff, triples=trip, ref_local=loc)
        print(name, "n", n, "score", score, "pos deltas", int((deltas > 0).sum()))


if __name__ == "__main__":
    main()
