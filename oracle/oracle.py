"""ctypes binding of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loads oracle/_ref/liboracle.so (the C restatement, bm_oracle.c),
oracle/_ref/libgen.so (the seeded workload generator, host C, so the CPU legs
make their inputs without the engine library) and, when they were built, the
reference's own code compiled in place: oracle/_ref/librefgao.so
(src/graph-alignment-optimized.c), librefpar.so
(src/graph-alignment-optimized-parallel.c), librefperm.so (src/permutation.c)
and librefgreedy.so (src/greedy-feature-match.c).  Only tests/, smoke() and
bench.py's CPU-baseline leg import this module, as the checker.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


def _load(name):
    path = os.path.join(REF_DIR, name)
    return C.CDLL(path) if os.path.exists(path) else None


vp, i32, i64, u64 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64
_orc = None


def orc_lib():
    global _orc
    if _orc is None:
        L = C.CDLL(os.path.join(REF_DIR, "liboracle.so"))
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i32, i64, vp, vp, vp, i64, vp, vp, vp]
        L.orc_free.argtypes = [vp]
        L.orc_free.restype = None
        L.orc_score.restype = i64
        L.orc_score.argtypes = [vp, vp]
        L.orc_swap_delta.argtypes = [vp, vp, i32, i32]
        L.orc_all_deltas.argtypes = [vp, vp, vp]
        L.orc_all_deltas.restype = None
        L.orc_sweep.argtypes = [vp, vp, i32, i32, vp, vp]
        L.orc_sweep_given.argtypes = [vp, vp, vp, i32, i32, vp, vp]
        L.orc_pair_deltas.argtypes = [vp, vp, i64, vp, vp, vp]
        L.orc_pair_deltas.restype = None
        L.orc_triple_deltas.argtypes = [vp, vp, i64, vp, vp, vp, vp]
        L.orc_triple_deltas.restype = None
        L.orc_triple_samples.restype = i64
        L.orc_triple_samples.argtypes = [vp, u64, i32, vp, vp]
        L.orc_triple_round_given.argtypes = [vp, vp, i32, u64, vp, i32, i32, vp]
        L.orc_first_improvement.restype = i64
        L.orc_first_improvement.argtypes = [vp, vp, i32, C.POINTER(i32), C.POINTER(i64)]
        L.orc_local_score.restype = i64
        L.orc_local_score.argtypes = [vp, vp, vp, i32]
        L.orc_triple_delta.argtypes = [vp, vp, i32, i32, i32, i32]
        L.orc_sample_triple.argtypes = [vp, u64, i32, i32, C.POINTER(i32), C.POINTER(i32)]
        L.orc_triple_round.argtypes = [vp, vp, i32, u64, i32, i32, vp]
        L.orc_quad_delta.argtypes = [vp, vp, i32, i32, i32, i32, i32]
        L.orc_sample_quad.argtypes = [vp, u64, i32, i32, C.POINTER(i32), C.POINTER(i32), C.POINTER(i32)]
        L.orc_quad_round.argtypes = [vp, vp, i32, u64, i32, i32, vp]
        L.orc_best_swap_descent.argtypes = [vp, vp, i32, vp, vp]
        L.orc_greedy_features.argtypes = [i32, i64, vp, vp, vp]
        L.orc_greedy_features.restype = None
        L.orc_greedy_distance.argtypes = [vp, vp]
        L.orc_greedy_match.argtypes = [i32, i64, vp, vp, vp, i64, vp, vp, vp, vp]
        L.orc_greedy_match.restype = None
        _orc = L
    return _orc


class GenParams(C.Structure):
    """bm_gen_params of include/bm.h."""
    _fields_ = [("n", C.c_int32), ("wmax", C.c_int32), ("e", C.c_int64), ("seed", C.c_uint64),
                ("alpha", C.c_double), ("geom_p", C.c_double), ("tail_prob", C.c_double),
                ("tail_alpha", C.c_double), ("tail_scale", C.c_double), ("del_frac", C.c_double),
                ("add_frac", C.c_double), ("jitter", C.c_int32), ("reserved", C.c_int32)]


_gen = None


def generate(n=1000, e=20000, seed=20261203, wmax=5000, tail_prob=0.0, **kw):
    """The seeded graph pair of bm_generate (the same source, compiled into
    oracle/_ref/libgen.so): dict of int32 arrays, 1-based ids."""
    global _gen
    if _gen is None:
        L = C.CDLL(os.path.join(REF_DIR, "libgen.so"))
        L.bm_gen_defaults.argtypes = [C.POINTER(GenParams)]
        L.bm_gen_defaults.restype = None
        L.bm_generate.argtypes = [C.POINTER(GenParams), vp, vp, vp, C.POINTER(i64), vp, vp, vp, vp, vp]
        _gen = L
    p = GenParams()
    _gen.bm_gen_defaults(C.byref(p))
    p.n, p.e, p.seed, p.wmax, p.tail_prob = n, e, seed, wmax, tail_prob
    for k, v in kw.items():
        setattr(p, k, v)
    cap = e + int(np.ceil(p.add_frac * e)) + 1
    s1, d1, w1 = (np.zeros(e, np.int32) for _ in range(3))
    s2, d2, w2 = (np.zeros(cap, np.int32) for _ in range(3))
    pi = np.zeros(n + 1, np.int32)
    m0 = np.zeros(n + 1, np.int32)
    e2 = i64()
    st = _gen.bm_generate(C.byref(p), _p(s1), _p(d1), _p(w1), C.byref(e2), _p(s2), _p(d2), _p(w2), _p(pi),
                          _p(m0))
    if st != 0:
        raise ValueError(f"bm_generate failed with status {st}")
    k = e2.value
    return dict(n=n, src1=s1, dst1=d1, w1=w1, src2=s2[:k].copy(), dst2=d2[:k].copy(), w2=w2[:k].copy(), pi=pi,
                map0=m0)


class Oracle:
    """The C restatement (bm_oracle.c) over one graph pair (1-based ids)."""

    def __init__(self, n, src1, dst1, w1, src2, dst2, w2):
        self._keep = [np.ascontiguousarray(x, np.int32) for x in (src1, dst1, w1, src2, dst2, w2)]
        a = self._keep
        self.n = int(n)
        self.h = orc_lib().orc_create(self.n, len(a[0]), _p(a[0]), _p(a[1]), _p(a[2]),
                                      len(a[3]), _p(a[3]), _p(a[4]), _p(a[5]))

    @classmethod
    def from_pair(cls, g):
        return cls(g["n"], g["src1"], g["dst1"], g["w1"], g["src2"], g["dst2"], g["w2"])

    def __del__(self):
        if getattr(self, "h", None):
            orc_lib().orc_free(self.h)
            self.h = None

    def score(self, m):
        m = np.ascontiguousarray(m, np.int32)
        return orc_lib().orc_score(self.h, _p(m))

    def swap_delta(self, m, a, b):
        m = np.ascontiguousarray(m, np.int32)
        return orc_lib().orc_swap_delta(self.h, _p(m), int(a), int(b))

    def all_deltas(self, m):
        m = np.ascontiguousarray(m, np.int32)
        out = np.zeros(self.n * (self.n - 1) // 2, np.int32)
        orc_lib().orc_all_deltas(self.h, _p(m), _p(out))
        return out

    def pair_deltas(self, m, a, b):
        """Deltas of the pairs (a[i], b[i]) on matching m."""
        m = np.ascontiguousarray(m, np.int32)
        a = np.ascontiguousarray(a, np.int32)
        b = np.ascontiguousarray(b, np.int32)
        out = np.zeros(len(a), np.int32)
        orc_lib().orc_pair_deltas(self.h, _p(m), len(a), _p(a), _p(b), _p(out))
        return out

    def triple_deltas(self, m, a, b, c):
        """Both rotations' deltas of the triples (a[i], b[i], c[i]), [k, 2]."""
        m = np.ascontiguousarray(m, np.int32)
        a, b, c = (np.ascontiguousarray(x, np.int32) for x in (a, b, c))
        out = np.zeros(2 * len(a), np.int32)
        orc_lib().orc_triple_deltas(self.h, _p(m), len(a), _p(a), _p(b), _p(c), _p(out))
        return out.reshape(-1, 2)

    def sweep(self, m, max_candidates=0, max_verify=-1, want_moves=False):
        """Runs one sweep IN PLACE on m (int32 array); returns stats dict."""
        st = np.zeros(8, np.int64)
        mv = np.zeros(3 * (self.n + 1), np.int32) if want_moves else None
        c = orc_lib().orc_sweep(self.h, _p(m), max_candidates, max_verify, _p(st),
                                _p(mv) if mv is not None else None)
        d = dict(total_delta=int(st[0]), candidates=int(st[1]), scanned=int(st[2]), verified=int(st[3]),
                 committed=int(st[4]), best_delta=int(st[5]), deltas=int(st[6]))
        if want_moves:
            d["moves"] = mv[:3 * c].reshape(-1, 3)
        return d

    def sweep_given(self, m, all_deltas, max_candidates=0, max_verify=-1):
        """The sweep's selection and commit IN PLACE on m from supplied deltas
        (the linear pair order of all_deltas); returns stats with the moves
        as [k, 3] rows (lo, hi, delta) in commit order."""
        d = np.ascontiguousarray(all_deltas, np.int32)
        assert d.shape == (self.n * (self.n - 1) // 2,)
        st = np.zeros(8, np.int64)
        mv = np.zeros(3 * (self.n + 1), np.int32)
        c = orc_lib().orc_sweep_given(self.h, _p(m), _p(d), max_candidates, max_verify, _p(st), _p(mv))
        return dict(total_delta=int(st[0]), candidates=int(st[1]), scanned=int(st[2]), verified=int(st[3]),
                    committed=int(st[4]), best_delta=int(st[5]), deltas=int(st[6]),
                    moves=mv[:3 * c].reshape(-1, 3))

    def triple_samples(self, seed, partners):
        """(b, c) of every slot of a 3-cycle round, [n, partners] each, 0 where
        the slot has no valid triple."""
        b = np.zeros(self.n * partners, np.int32)
        c = np.zeros(self.n * partners, np.int32)
        orc_lib().orc_triple_samples(self.h, seed, partners, _p(b), _p(c))
        return b.reshape(self.n, partners), c.reshape(self.n, partners)

    def triple_round_given(self, m, partners, seed, deltas, max_candidates=0, max_verify=-1):
        """A 3-cycle round IN PLACE on m from supplied deltas [n, partners, 2]."""
        d = np.ascontiguousarray(deltas, np.int32)
        assert d.shape == (self.n, partners, 2)
        st = np.zeros(8, np.int64)
        orc_lib().orc_triple_round_given(self.h, _p(m), partners, seed, _p(d), max_candidates, max_verify,
                                         _p(st))
        return dict(total_delta=int(st[0]), candidates=int(st[1]), scanned=int(st[2]), verified=int(st[3]),
                    committed=int(st[4]), best_delta=int(st[5]), triples=int(st[6]))

    def best_swap_descent(self, m, max_swaps):
        """Best-swap descent IN PLACE on m; returns (pairs [k,2], deltas [k])."""
        sw = np.zeros(2 * max(max_swaps, 1), np.int32)
        dl = np.zeros(max(max_swaps, 1), np.int32)
        k = orc_lib().orc_best_swap_descent(self.h, _p(m), int(max_swaps), _p(sw), _p(dl))
        return sw[:2 * k].reshape(-1, 2), dl[:k]

    def first_improvement(self, m, max_passes):
        p, ds = i32(), i64()
        c = orc_lib().orc_first_improvement(self.h, _p(m), max_passes, C.byref(p), C.byref(ds))
        return c, p.value, ds.value

    def triple_delta(self, m, a, b, c, rot):
        m = np.ascontiguousarray(m, np.int32)
        return orc_lib().orc_triple_delta(self.h, _p(m), a, b, c, rot)

    def local_score(self, m, vs):
        m = np.ascontiguousarray(m, np.int32)
        vs = np.ascontiguousarray(vs, np.int32)
        return orc_lib().orc_local_score(self.h, _p(m), _p(vs), len(vs))

    def sample_triple(self, seed, a, j):
        b, c = i32(), i32()
        ok = orc_lib().orc_sample_triple(self.h, seed, a, j, C.byref(b), C.byref(c))
        return (b.value, c.value) if ok else None

    def triple_round(self, m, partners=256, seed=0, max_candidates=0, max_verify=-1):
        st = np.zeros(8, np.int64)
        orc_lib().orc_triple_round(self.h, _p(m), partners, seed, max_candidates, max_verify, _p(st))
        return dict(total_delta=int(st[0]), candidates=int(st[1]), scanned=int(st[2]), verified=int(st[3]),
                    committed=int(st[4]), best_delta=int(st[5]), triples=int(st[6]))

    def quad_delta(self, m, a, b, c, d, q):
        """Exact delta of permutation q (1..23) of the 4-set (a, b, c, d), 1-based."""
        m = np.ascontiguousarray(m, np.int32)
        return orc_lib().orc_quad_delta(self.h, _p(m), a, b, c, d, q)

    def sample_quad(self, seed, a, j):
        b, c, d = C.c_int32(), C.c_int32(), C.c_int32()
        ok = orc_lib().orc_sample_quad(self.h, seed, a, j, C.byref(b), C.byref(c), C.byref(d))
        return (b.value, c.value, d.value) if ok else None

    def quad_round(self, m, partners=64, seed=0, max_candidates=0, max_verify=-1):
        """Runs one 4-set round IN PLACE on m; returns stats dict."""
        st = np.zeros(8, np.int64)
        orc_lib().orc_quad_round(self.h, _p(m), partners, seed, max_candidates, max_verify, _p(st))
        return dict(total_delta=int(st[0]), candidates=int(st[1]), scanned=int(st[2]), verified=int(st[3]),
                    committed=int(st[4]), best_delta=int(st[5]), quads=int(st[6]))


def greedy_features(n, src, dst):
    """[n, 4] int32: in, out, 2-hop out-reach, 2-hop in-reach (bm_oracle.c)."""
    s, d = (np.ascontiguousarray(x, np.int32) for x in (src, dst))
    out = np.zeros((int(n), 4), np.int32)
    orc_lib().orc_greedy_features(int(n), len(s), _p(s), _p(d), _p(out))
    return out


def greedy_distance(f1, f2):
    a, b = (np.ascontiguousarray(x, np.int32) for x in (f1, f2))
    return orc_lib().orc_greedy_distance(_p(a), _p(b))


def greedy_match(g):
    """The greedy feature matcher's matching, 1-based int32[n+1]."""
    n = int(g["n"])
    a = [np.ascontiguousarray(g[k], np.int32) for k in ("src1", "dst1", "w1", "src2", "dst2", "w2")]
    m = np.zeros(n + 1, np.int32)
    orc_lib().orc_greedy_match(n, len(a[0]), _p(a[0]), _p(a[1]), _p(a[2]), len(a[3]), _p(a[3]), _p(a[4]),
                               _p(a[5]), _p(m))
    return m


class RefGreedy:
    """The reference's src/greedy-feature-match.c, compiled in place.  Graphs
    are loaded from CSV files by the reference's own loader."""

    def __init__(self):
        L = _load("librefgreedy.so")
        if L is None:
            raise OSError("oracle/_ref/librefgreedy.so not built")
        L.refgreedy_load.restype = vp
        L.refgreedy_load.argtypes = [C.c_char_p, C.POINTER(i32)]
        L.refgreedy_free.argtypes = [vp]
        L.refgreedy_free.restype = None
        L.refgreedy_node_id.argtypes = [vp, i32]
        L.refgreedy_features.argtypes = [vp, vp]
        L.refgreedy_features.restype = None
        L.refgreedy_distance.argtypes = [vp, vp]
        L.refgreedy_match.argtypes = [vp, vp, vp]
        self.L = L

    def load(self, path):
        n = i32()
        g = self.L.refgreedy_load(path.encode(), C.byref(n))
        if not g:
            raise OSError(f"reference loader failed on {path}")
        return g, n.value

    def node_ids(self, g, n):
        return np.array([self.L.refgreedy_node_id(g, i) for i in range(n)], np.int32)

    def features(self, g, n):
        out = np.zeros((n, 6), np.int32)
        self.L.refgreedy_features(g, _p(out))
        return out

    def distance(self, f1, f2):
        a, b = (np.ascontiguousarray(x, np.int32) for x in (f1, f2))
        return self.L.refgreedy_distance(_p(a), _p(b))

    def match(self, g1, g2, n):
        out = np.zeros(n, np.int32)
        if self.L.refgreedy_match(g1, g2, _p(out)) != 0:
            raise RuntimeError("reference match_vertices failed")
        return out

    def free(self, g):
        self.L.refgreedy_free(g)


class RefGAO:
    """The reference's src/graph-alignment-optimized.c, compiled in place."""

    def __init__(self, lib=None):
        L = lib or _load("librefgao.so")
        if L is None:
            raise OSError("oracle/_ref/librefgao.so not built")
        L.refgao_graph_new.restype = vp
        L.refgao_graph_add_many.argtypes = [vp, i64, vp, vp, vp]
        L.refgao_graph_add_many.restype = None
        L.refgao_graph_free.argtypes = [vp]
        L.refgao_graph_free.restype = None
        L.refgao_score.argtypes = [vp, vp, vp]
        L.refgao_swap_delta.argtypes = [vp, vp, vp, i32, i32]
        L.refgao_pair_deltas.argtypes = [vp, vp, vp, i64, vp, vp, vp]
        L.refgao_pair_deltas.restype = None
        L.refgao_rows_omp.restype = i64
        L.refgao_rows_omp.argtypes = [vp, vp, vp, vp, i32, i32, C.POINTER(i64), C.POINTER(i32)]
        L.refgao_first_improvement.argtypes = [vp, vp, vp, i32, i32, C.POINTER(i64), C.POINTER(i32)]
        self.L = L
        self.NUM_NODES = L.refgao_num_nodes()

    def graph(self, s, d, w):
        g = self.L.refgao_graph_new()
        a = [np.ascontiguousarray(x, np.int32) for x in (s, d, w)]
        self.L.refgao_graph_add_many(g, len(a[0]), _p(a[0]), _p(a[1]), _p(a[2]))
        return g

    def pad(self, m):
        """The reference indexes mappings up to NUM_NODES."""
        out = np.zeros(max(self.NUM_NODES, len(m) - 1) + 1, np.int32)
        out[:len(m)] = m
        return out

    def score(self, gm, gf, m):
        mp = self.pad(m)
        return self.L.refgao_score(gm, gf, _p(mp))

    def pair_deltas(self, gm, gf, m, a, b):
        mp = self.pad(m)
        a = np.ascontiguousarray(a, np.int32)
        b = np.ascontiguousarray(b, np.int32)
        out = np.zeros(len(a), np.int32)
        self.L.refgao_pair_deltas(gm, gf, _p(mp), len(a), _p(a), _p(b), _p(out))
        return out

    def first_improvement(self, gm, gf, m, n, max_passes):
        """The reference's first-improvement loop on m (updated in place)
        until a pass commits nothing; returns (score, commits, passes)."""
        mp = self.pad(m)
        c, p = i64(), i32()
        s = self.L.refgao_first_improvement(gm, gf, _p(mp), int(n), int(max_passes), C.byref(c), C.byref(p))
        m[:] = mp[:len(m)]
        return s, c.value, p.value

    def free(self, g):
        self.L.refgao_graph_free(g)

    def rows_omp(self, gm, gf, m, rows, n):
        mp = self.pad(m)
        rows = np.ascontiguousarray(rows, np.int32)
        cs, nt = i64(), i32()
        cnt = self.L.refgao_rows_omp(gm, gf, _p(mp), _p(rows), len(rows), n, C.byref(cs), C.byref(nt))
        return cnt, cs.value, nt.value


class RefPar:
    """The reference's racy OpenMP tool, src/graph-alignment-optimized-parallel.c,
    compiled in place: its parallel loop over partners driven for given rows."""

    def __init__(self):
        L = _load("librefpar.so")
        if L is None:
            raise OSError("oracle/_ref/librefpar.so not built")
        L.refpar_graph_new.restype = vp
        L.refpar_graph_add_many.argtypes = [vp, i64, vp, vp, vp]
        L.refpar_graph_add_many.restype = None
        L.refpar_graph_free.argtypes = [vp]
        L.refpar_graph_free.restype = None
        L.refpar_rows.restype = i64
        L.refpar_rows.argtypes = [vp, vp, vp, vp, i32, i32, C.POINTER(i64), C.POINTER(i32)]
        self.L = L
        self.NUM_NODES = L.refpar_num_nodes()

    def graph(self, s, d, w):
        g = self.L.refpar_graph_new()
        a = [np.ascontiguousarray(x, np.int32) for x in (s, d, w)]
        self.L.refpar_graph_add_many(g, len(a[0]), _p(a[0]), _p(a[1]), _p(a[2]))
        return g

    def free(self, g):
        self.L.refpar_graph_free(g)

    def rows(self, gm, gf, m, rows, n):
        """Runs the rows on m (updated in place); returns (deltas, commits, threads)."""
        mp = np.zeros(max(self.NUM_NODES, len(m) - 1) + 1, np.int32)
        mp[:len(m)] = m
        rows = np.ascontiguousarray(rows, np.int32)
        c, nt = i64(), i32()
        cnt = self.L.refpar_rows(gm, gf, _p(mp), _p(rows), len(rows), int(n), C.byref(c), C.byref(nt))
        m[:] = mp[:len(m)]
        return cnt, c.value, nt.value


class RefPerm:
    """The reference's src/permutation.c, compiled in place."""

    def __init__(self):
        L = _load("librefperm.so")
        if L is None:
            raise OSError("oracle/_ref/librefperm.so not built")
        L.refperm_graph_new.restype = vp
        L.refperm_graph_add_many.argtypes = [vp, i64, vp, vp, vp]
        L.refperm_graph_add_many.restype = None
        L.refperm_local_score.argtypes = [vp, vp, vp, vp, i32]
        L.refperm_score.argtypes = [vp, vp, vp]
        L.refperm_graph_free.argtypes = [vp]
        L.refperm_graph_free.restype = None
        L.refperm_triples_omp.argtypes = [vp, vp, vp, i64, vp, vp, vp, vp]
        self.L = L

    def graph(self, s, d, w):
        g = self.L.refperm_graph_new()
        a = [np.ascontiguousarray(x, np.int32) for x in (s, d, w)]
        self.L.refperm_graph_add_many(g, len(a[0]), _p(a[0]), _p(a[1]), _p(a[2]))
        return g

    def free(self, g):
        self.L.refperm_graph_free(g)

    def triples_omp(self, gm, gf, m, a, b, c):
        """Both rotations' deltas of the triples by the reference's local score
        under OpenMP, [k, 2]; returns (deltas, threads)."""
        mp = np.zeros(max(18524, len(m) - 1) + 1, np.int32)
        mp[:len(m)] = m
        a, b, c = (np.ascontiguousarray(x, np.int32) for x in (a, b, c))
        out = np.zeros(2 * len(a), np.int32)
        nt = self.L.refperm_triples_omp(gm, gf, _p(mp), len(a), _p(a), _p(b), _p(c), _p(out))
        return out.reshape(-1, 2), nt

    def local_score(self, gm, gf, m, vs):
        mp = np.zeros(max(18524, len(m) - 1) + 1, np.int32)
        mp[:len(m)] = m
        vs = np.ascontiguousarray(vs, np.int32)
        return self.L.refperm_local_score(gm, gf, _p(mp), _p(vs), len(vs))
