"""ctypes binding of the engine's C ABI (include/bm.h) for tests and bench.

The engine itself is libbm.so (CUDA kernels for sm_100a + host C).  This module
only marshals numpy arrays across the C boundary; there is no Python or CPU
fallback for any compute call -- if the library is missing, loading fails.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libbm.so")

BM_OK, BM_E_INPUT, BM_E_CUDA, BM_E_OVERFLOW, BM_E_TIMEOUT, BM_E_NOMEM, BM_E_STATE, BM_E_IO = (
    0, -1, -2, -3, -4, -5, -6, -7)
BM_FLAG_FORCE_I32 = 1
BM_FLAG_NO_HUB_GEMM = 2
BM_STATIC_MAX_PAIRS = 65536
BM_STALL_HUB_GEMM, BM_STALL_COMMIT, BM_STALL_COMBINE, BM_STALL_GREEDY, BM_STALL_MLP_GEMM, BM_STALL_BATCH = (
    1, 2, 3, 4, 5, 6)


class GenParams(C.Structure):
    _fields_ = [("n", C.c_int32), ("wmax", C.c_int32), ("e", C.c_int64), ("seed", C.c_uint64),
                ("alpha", C.c_double), ("geom_p", C.c_double), ("tail_prob", C.c_double),
                ("tail_alpha", C.c_double), ("tail_scale", C.c_double), ("del_frac", C.c_double),
                ("add_frac", C.c_double), ("jitter", C.c_int32), ("reserved", C.c_int32)]


class Info(C.Structure):
    _fields_ = [("n", C.c_int32), ("entry_bits", C.c_int32), ("e1", C.c_int64), ("e2", C.c_int64),
                ("g1_self_loops", C.c_int64), ("device_bytes", C.c_int64), ("device", C.c_int32),
                ("num_sms", C.c_int32), ("hubs", C.c_int32), ("hub_k", C.c_int32)]


class SweepOpts(C.Structure):
    _fields_ = [("max_candidates", C.c_int32), ("max_verify", C.c_int32), ("commit_ctas", C.c_int32),
                ("incremental", C.c_int32), ("reserved", C.c_int32 * 4)]


class SweepStats(C.Structure):
    _fields_ = [("score_before", C.c_int64), ("score_after", C.c_int64), ("deltas_evaluated", C.c_int64),
                ("candidates", C.c_int32), ("scanned", C.c_int32), ("verified", C.c_int32),
                ("committed", C.c_int32), ("best_delta", C.c_int32), ("profit_mode", C.c_int32),
                ("ms_profit", C.c_float), ("ms_combine", C.c_float), ("ms_commit", C.c_float),
                ("ms_total", C.c_float), ("ms_prep", C.c_float), ("ms_hub", C.c_float), ("min_terms", C.c_int64),
                ("commit_entries", C.c_int64), ("commit_steps", C.c_int32), ("commit_carried", C.c_int32)]


class TripleOpts(C.Structure):
    _fields_ = [("partners", C.c_int32), ("max_candidates", C.c_int32), ("max_verify", C.c_int32),
                ("incremental", C.c_int32), ("seed", C.c_uint64), ("reserved", C.c_int32 * 4)]


class TripleStats(C.Structure):
    _fields_ = [("score_before", C.c_int64), ("score_after", C.c_int64), ("triples", C.c_int64),
                ("rotations", C.c_int64), ("candidates", C.c_int32), ("scanned", C.c_int32),
                ("verified", C.c_int32), ("committed", C.c_int32), ("best_delta", C.c_int32),
                ("reserved", C.c_int32), ("ms_sample", C.c_float), ("ms_eval", C.c_float),
                ("ms_commit", C.c_float), ("ms_total", C.c_float)]


class LookupStats(C.Structure):
    _fields_ = [("score_before", C.c_int64), ("score_after", C.c_int64), ("swaps", C.c_int32),
                ("converged", C.c_int32), ("refresh_mode", C.c_int32), ("reserved", C.c_int32),
                ("ms_refresh", C.c_float), ("ms_total", C.c_float)]


class GreedyStats(C.Structure):
    _fields_ = [("ms_features", C.c_float), ("ms_match", C.c_float), ("reserved", C.c_int32 * 2)]


class MlpTrainStats(C.Structure):
    _fields_ = [("samples", C.c_int64), ("steps", C.c_int64), ("first_loss", C.c_float), ("last_loss", C.c_float)]


class LearnedOpts(C.Structure):
    _fields_ = [("pool", C.c_int32), ("per_row", C.c_int32), ("top_fraction", C.c_double), ("seed", C.c_uint64),
                ("retries", C.c_int32), ("reserved", C.c_int32)]


class LearnedRunStats(C.Structure):
    _fields_ = [("sweeps", C.c_int32), ("learned", C.c_int32), ("exhaustive", C.c_int32), ("reached", C.c_int32),
                ("converged", C.c_int32), ("reserved", C.c_int32), ("score_before", C.c_int64),
                ("score_after", C.c_int64), ("committed", C.c_int64), ("ms_total", C.c_float),
                ("ms_learned", C.c_float), ("ms_exhaustive", C.c_float), ("reserved2", C.c_float)]


class QuadOpts(C.Structure):
    _fields_ = [("partners", C.c_int32), ("max_candidates", C.c_int32), ("max_verify", C.c_int32),
                ("incremental", C.c_int32), ("seed", C.c_uint64), ("reserved", C.c_int32 * 4)]


class QuadStats(C.Structure):
    _fields_ = [("score_before", C.c_int64), ("score_after", C.c_int64), ("quads", C.c_int64),
                ("permutations", C.c_int64), ("candidates", C.c_int32), ("scanned", C.c_int32),
                ("verified", C.c_int32), ("committed", C.c_int32), ("best_delta", C.c_int32),
                ("reserved", C.c_int32), ("ms_sample", C.c_float), ("ms_eval", C.c_float),
                ("ms_commit", C.c_float), ("ms_total", C.c_float)]


def _p(a):
    return a.ctypes.data_as(C.c_void_p)


_lib = None


def lib():
    """Loads libbm.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, i32, i64, u32 = C.c_void_p, C.c_int32, C.c_int64, C.c_uint32
        L.bm_status_string.restype = C.c_char_p
        L.bm_status_string.argtypes = [i32]
        L.bm_last_error.restype = C.c_char_p
        L.bm_last_error.argtypes = [vp]
        L.bm_create.argtypes = [C.POINTER(vp), i32, i64, vp, vp, vp, i64, vp, vp, vp, u32]
        L.bm_destroy.argtypes = [vp]
        L.bm_destroy.restype = None
        L.bm_get_info.argtypes = [vp, C.POINTER(Info)]
        for f in ("bm_set_mapping", "bm_get_mapping", "bm_all_deltas"):
            getattr(L, f).argtypes = [vp, vp]
        L.bm_score.argtypes = [vp, C.POINTER(i64)]
        L.bm_pair_deltas.argtypes = [vp, i64, vp, vp, vp]
        L.bm_profit_row.argtypes = [vp, i32, vp]
        L.bm_pair_deltas_static.argtypes = [vp, i64, vp, vp, vp]
        L.bm_sweep.argtypes = [vp, C.POINTER(SweepOpts), C.POINTER(SweepStats)]
        L.bm_hillclimb.argtypes = [vp, i32, C.POINTER(SweepOpts), vp, C.POINTER(i32)]
        L.bm_first_improvement.argtypes = [vp, i32, C.POINTER(i64), C.POINTER(i32)]
        L.bm_triple_deltas.argtypes = [vp, i64, vp, vp, vp, vp]
        L.bm_triple_round.argtypes = [vp, C.POINTER(TripleOpts), C.POINTER(TripleStats)]
        L.bm_lookup_rows.argtypes = [vp, i32, i32, vp]
        L.bm_lookup_descent.argtypes = [vp, i32, C.POINTER(LookupStats)]
        L.bm_greedy_match.argtypes = [i32, i64, vp, vp, vp, i64, vp, vp, vp, vp, C.POINTER(GreedyStats)]
        L.bm_greedy_features.argtypes = [i32, i64, vp, vp, vp, vp]
        L.bm_timer_mark.argtypes = [vp, i32]
        L.bm_timer_elapsed.argtypes = [vp, i32, i32, C.POINTER(C.c_float)]
        L.bm_measure_peaks.argtypes = [i32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.bm_test_stall.argtypes = [i32]
        L.bm_batch_create.argtypes = [C.POINTER(vp), i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, u32]
        L.bm_batch_destroy.argtypes = [vp]
        L.bm_batch_destroy.restype = None
        L.bm_batch_last_error.restype = C.c_char_p
        L.bm_batch_last_error.argtypes = [vp]
        L.bm_batch_set_mappings.argtypes = [vp, vp]
        L.bm_batch_get_mappings.argtypes = [vp, vp]
        L.bm_batch_scores.argtypes = [vp, vp]
        L.bm_batch_autotune.argtypes = [vp, C.POINTER(i32), C.POINTER(i32)]
        L.bm_batch_set_schedule.argtypes = [vp, i32, i32, i32]
        L.bm_batch_sweeps.argtypes = [vp, i32, C.POINTER(SweepOpts), vp, C.POINTER(C.c_float)]
        L.bm_batch_info.argtypes = [vp, C.POINTER(i32), C.POINTER(i32), C.POINTER(i64), C.POINTER(i32), C.POINTER(i32)]
        L.bm_mlp_param_count.restype = i64
        L.bm_mlp_param_count.argtypes = []
        L.bm_mlp_create.argtypes = [C.POINTER(vp), C.c_uint64]
        L.bm_mlp_destroy.argtypes = [vp]
        L.bm_mlp_destroy.restype = None
        L.bm_mlp_last_error.restype = C.c_char_p
        L.bm_mlp_last_error.argtypes = [vp]
        L.bm_mlp_get_params.argtypes = [vp, vp]
        L.bm_mlp_set_params.argtypes = [vp, vp]
        L.bm_mlp_features.argtypes = [vp, vp, vp, vp]
        L.bm_mlp_rank_pairs.argtypes = [vp, vp, i64, vp, vp, vp]
        L.bm_mlp_forward.argtypes = [vp, i64, vp, vp]
        L.bm_mlp_train_step.argtypes = [vp, i64, vp, vp, C.c_float, C.POINTER(C.c_float), vp]
        L.bm_mlp_train_from.argtypes = [vp, vp, i32, i32, i32, C.c_float, C.c_uint64, C.POINTER(MlpTrainStats)]
        L.bm_learned_sweep.argtypes = [vp, vp, C.POINTER(LearnedOpts), C.POINTER(SweepStats), C.POINTER(i32)]
        L.bm_learned_run.argtypes = [vp, vp, C.POINTER(LearnedOpts), i32, i64, i32, C.POINTER(LearnedRunStats),
                                     vp, vp, vp]
        L.bm_quad_deltas.argtypes = [vp, i64, vp, vp, vp]
        L.bm_quad_round.argtypes = [vp, C.POINTER(QuadOpts), C.POINTER(QuadStats)]
        L.bm_free.argtypes = [vp]
        L.bm_free.restype = None
        L.bm_read_graph_csv.argtypes = [C.c_char_p, C.POINTER(i64), C.POINTER(vp), C.POINTER(vp),
                                        C.POINTER(vp), C.POINTER(i32)]
        L.bm_read_mapping_csv.argtypes = [C.c_char_p, i32, vp, C.POINTER(i32)]
        L.bm_write_mapping_csv.argtypes = [C.c_char_p, i32, vp]
        L.bm_write_mapping_csv_numeric.argtypes = [C.c_char_p, i32, vp]
        L.bm_gen_defaults.argtypes = [C.POINTER(GenParams)]
        L.bm_gen_defaults.restype = None
        L.bm_generate.argtypes = [C.POINTER(GenParams), vp, vp, vp, C.POINTER(i64), vp, vp, vp, vp, vp]
        _lib = L
    return _lib


class BMError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{lib().bm_status_string(status).decode()} ({status}): {msg}")
        self.status = status


def _check(st, ctx=None):
    if st != BM_OK:
        raise BMError(st, (lib().bm_last_error(ctx) or b"").decode())


def test_stall(site):
    """bm_test_stall: the next launch at `site` makes one bounded wait run out."""
    _check(lib().bm_test_stall(int(site)))


# ---- generator -------------------------------------------------------------
def gen_params(n=1000, e=20000, seed=20261203, wmax=5000, tail_prob=0.0, **kw):
    p = GenParams()
    lib().bm_gen_defaults(C.byref(p))
    p.n, p.e, p.seed, p.wmax, p.tail_prob = n, e, seed, wmax, tail_prob
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def generate(params):
    """Runs bm_generate; returns dict of int32 numpy arrays (1-based ids)."""
    e = params.e
    cap = e + int(np.ceil(params.add_frac * e)) + 1
    s1, d1, w1 = (np.zeros(e, np.int32) for _ in range(3))
    s2, d2, w2 = (np.zeros(cap, np.int32) for _ in range(3))
    pi = np.zeros(params.n + 1, np.int32)
    m0 = np.zeros(params.n + 1, np.int32)
    e2 = C.c_int64()
    _check(lib().bm_generate(C.byref(params), _p(s1), _p(d1), _p(w1), C.byref(e2), _p(s2), _p(d2),
                             _p(w2), _p(pi), _p(m0)))
    k = e2.value
    return dict(n=params.n, src1=s1, dst1=d1, w1=w1, src2=s2[:k].copy(), dst2=d2[:k].copy(),
                w2=w2[:k].copy(), pi=pi, map0=m0)


# ---- engine ----------------------------------------------------------------
class Engine:
    """One engine context on the current CUDA device."""

    def __init__(self, n, src1, dst1, w1, src2, dst2, w2, flags=0):
        arrs = [np.ascontiguousarray(x, dtype=np.int32) for x in (src1, dst1, w1, src2, dst2, w2)]
        self._keep = arrs
        h = C.c_void_p()
        st = lib().bm_create(C.byref(h), int(n), len(arrs[0]), _p(arrs[0]), _p(arrs[1]), _p(arrs[2]),
                             len(arrs[3]), _p(arrs[3]), _p(arrs[4]), _p(arrs[5]), flags)
        _check(st, None)
        self.h = h
        self.n = int(n)

    @classmethod
    def from_pair(cls, g, flags=0):
        return cls(g["n"], g["src1"], g["dst1"], g["w1"], g["src2"], g["dst2"], g["w2"], flags)

    def close(self):
        if getattr(self, "h", None):
            lib().bm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def info(self):
        i = Info()
        _check(lib().bm_get_info(self.h, C.byref(i)), self.h)
        return {k: getattr(i, k) for k, _ in Info._fields_}

    def set_mapping(self, m):
        m = np.ascontiguousarray(m, dtype=np.int32)
        assert m.shape == (self.n + 1,)
        _check(lib().bm_set_mapping(self.h, _p(m)), self.h)

    def get_mapping(self):
        m = np.zeros(self.n + 1, np.int32)
        _check(lib().bm_get_mapping(self.h, _p(m)), self.h)
        return m

    def score(self):
        s = C.c_int64()
        _check(lib().bm_score(self.h, C.byref(s)), self.h)
        return s.value

    def pair_deltas(self, m1, m2):
        m1 = np.ascontiguousarray(m1, np.int32)
        m2 = np.ascontiguousarray(m2, np.int32)
        out = np.zeros(len(m1), np.int32)
        _check(lib().bm_pair_deltas(self.h, len(m1), _p(m1), _p(m2), _p(out)), self.h)
        return out

    def pair_deltas_static(self, m1, m2):
        """bm_pair_deltas_static: same deltas, staged in the library's fixed array."""
        m1 = np.ascontiguousarray(m1, np.int32)
        m2 = np.ascontiguousarray(m2, np.int32)
        out = np.zeros(len(m1), np.int32)
        _check(lib().bm_pair_deltas_static(self.h, len(m1), _p(m1), _p(m2), _p(out)), self.h)
        return out

    def all_deltas(self):
        out = np.zeros(self.n * (self.n - 1) // 2, np.int32)
        _check(lib().bm_all_deltas(self.h, _p(out)), self.h)
        return out

    def profit_row(self, a):
        out = np.zeros(self.n, np.int32)
        _check(lib().bm_profit_row(self.h, int(a), _p(out)), self.h)
        return out

    def sweep(self, max_candidates=0, max_verify=-1, commit_ctas=0, incremental=False):
        o = SweepOpts(max_candidates, max_verify, commit_ctas, int(bool(incremental)))
        s = SweepStats()
        _check(lib().bm_sweep(self.h, C.byref(o), C.byref(s)), self.h)
        return {k: getattr(s, k) for k, _ in SweepStats._fields_ if k != "reserved"}

    def lookup_rows(self, a0, rows):
        """Rows a0..a0+rows-1 (1-based) of the exact delta table, shape [rows, n]."""
        out = np.zeros((int(rows), self.n), np.int32)
        _check(lib().bm_lookup_rows(self.h, int(a0), int(rows), _p(out)), self.h)
        return out

    def lookup_descent(self, max_swaps):
        s = LookupStats()
        _check(lib().bm_lookup_descent(self.h, int(max_swaps), C.byref(s)), self.h)
        return {k: getattr(s, k) for k, _ in LookupStats._fields_ if k != "reserved"}

    def timer_mark(self, slot):
        _check(lib().bm_timer_mark(self.h, slot), self.h)

    def timer_elapsed(self, a, b):
        ms = C.c_float()
        _check(lib().bm_timer_elapsed(self.h, a, b, C.byref(ms)), self.h)
        return ms.value

    def first_improvement(self, max_passes):
        c, p = C.c_int64(), C.c_int32()
        _check(lib().bm_first_improvement(self.h, int(max_passes), C.byref(c), C.byref(p)), self.h)
        return c.value, p.value

    def triple_deltas(self, a, b, c):
        a, b, c = (np.ascontiguousarray(x, np.int32) for x in (a, b, c))
        out = np.zeros(2 * len(a), np.int32)
        _check(lib().bm_triple_deltas(self.h, len(a), _p(a), _p(b), _p(c), _p(out)), self.h)
        return out.reshape(-1, 2)

    def quad_deltas(self, sets, perms):
        """Exact deltas of permutation perms[i] (1..23) of 1-based 4-sets sets[i]."""
        sets = np.ascontiguousarray(sets, np.int32).reshape(-1, 4)
        perms = np.ascontiguousarray(perms, np.int32)
        out = np.zeros(len(sets), np.int32)
        _check(lib().bm_quad_deltas(self.h, len(sets), _p(sets), _p(perms), _p(out)), self.h)
        return out

    def quad_round(self, partners=64, seed=0, max_candidates=0, max_verify=-1, incremental=False):
        o = QuadOpts(partners, max_candidates, max_verify, int(bool(incremental)), seed)
        s = QuadStats()
        _check(lib().bm_quad_round(self.h, C.byref(o), C.byref(s)), self.h)
        return {k: getattr(s, k) for k, _ in QuadStats._fields_ if k != "reserved"}

    def triple_round(self, partners=256, seed=0, max_candidates=0, max_verify=-1, incremental=False):
        o = TripleOpts()
        o.partners, o.max_candidates, o.max_verify, o.seed = partners, max_candidates, max_verify, seed
        o.incremental = int(bool(incremental))
        s = TripleStats()
        _check(lib().bm_triple_round(self.h, C.byref(o), C.byref(s)), self.h)
        return {k: getattr(s, k) for k, _ in TripleStats._fields_ if k != "reserved"}


def read_graph_csv(path):
    e, s, d, w, mx = C.c_int64(), C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_int32()
    _check(lib().bm_read_graph_csv(path.encode(), C.byref(e), C.byref(s), C.byref(d), C.byref(w),
                                   C.byref(mx)))
    out = []
    for ptr in (s, d, w):
        if e.value:
            arr = np.ctypeslib.as_array(C.cast(ptr, C.POINTER(C.c_int32)), shape=(e.value,)).copy()
        else:
            arr = np.zeros(0, np.int32)
        lib().bm_free(ptr)
        out.append(arr)
    return out[0], out[1], out[2], mx.value


def read_mapping_csv(path, n):
    m = np.zeros(n + 1, np.int32)
    cnt = C.c_int32()
    _check(lib().bm_read_mapping_csv(path.encode(), n, _p(m), C.byref(cnt)))
    return m, cnt.value


def write_mapping_csv(path, m, numeric=False):
    m = np.ascontiguousarray(m, np.int32)
    f = lib().bm_write_mapping_csv_numeric if numeric else lib().bm_write_mapping_csv
    _check(f(path.encode(), len(m) - 1, _p(m)))


def greedy_match(g):
    """Greedy feature matcher (bm_greedy_match): (map int32[n+1], stats dict)."""
    n = int(g["n"])
    a = [np.ascontiguousarray(g[k], np.int32) for k in ("src1", "dst1", "w1", "src2", "dst2", "w2")]
    m = np.zeros(n + 1, np.int32)
    st = GreedyStats()
    _check(lib().bm_greedy_match(n, len(a[0]), _p(a[0]), _p(a[1]), _p(a[2]), len(a[3]), _p(a[3]), _p(a[4]),
                                 _p(a[5]), _p(m), C.byref(st)))
    return m, {"ms_features": st.ms_features, "ms_match": st.ms_match}


def greedy_features(n, src, dst, w):
    """[n, 4] int32: in-degree, out-degree, distinct 2-hop out-reach, 2-hop in-reach."""
    s, d, ww = (np.ascontiguousarray(x, np.int32) for x in (src, dst, w))
    out = np.zeros((int(n), 4), np.int32)
    _check(lib().bm_greedy_features(int(n), len(s), _p(s), _p(d), _p(ww), _p(out)))
    return out


def measure_peaks(n):
    """(shared-memory atomic adds/s, int32 min+add pairs/s) on the current device."""
    r, m = C.c_double(), C.c_double()
    _check(lib().bm_measure_peaks(int(n), C.byref(r), C.byref(m)))
    return r.value, m.value


class Batch:
    """Independent instances swept together (bm_batch_*)."""

    def __init__(self, pairs, flags=0):
        self.pairs = pairs
        k = len(pairs)
        keep = []

        def arr(key):
            xs = [np.ascontiguousarray(g[key], np.int32) for g in pairs]
            keep.extend(xs)
            ptrs = (C.c_void_p * k)(*[x.ctypes.data for x in xs])
            keep.append(ptrs)
            return ptrs
        n = np.array([g["n"] for g in pairs], np.int32)
        e1 = np.array([len(g["src1"]) for g in pairs], np.int64)
        e2 = np.array([len(g["src2"]) for g in pairs], np.int64)
        keep += [n, e1, e2]
        h = C.c_void_p()
        st = lib().bm_batch_create(C.byref(h), k, _p(n), _p(e1), arr("src1"), arr("dst1"), arr("w1"),
                                   _p(e2), arr("src2"), arr("dst2"), arr("w2"), flags)
        if st != BM_OK:
            raise BMError(st, (lib().bm_batch_last_error(None) or b"").decode())
        self.h = h
        self.k = k
        self.ns = [int(g["n"]) for g in pairs]

    def _chk(self, st):
        if st != BM_OK:
            raise BMError(st, (lib().bm_batch_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            lib().bm_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_mappings(self, maps):
        ms = [np.ascontiguousarray(m, np.int32) for m in maps]
        ptrs = (C.c_void_p * self.k)(*[m.ctypes.data for m in ms])
        self._chk(lib().bm_batch_set_mappings(self.h, ptrs))

    def get_mappings(self):
        ms = [np.zeros(n + 1, np.int32) for n in self.ns]
        ptrs = (C.c_void_p * self.k)(*[m.ctypes.data for m in ms])
        self._chk(lib().bm_batch_get_mappings(self.h, ptrs))
        return ms

    def scores(self):
        s = np.zeros(self.k, np.int64)
        self._chk(lib().bm_batch_scores(self.h, _p(s)))
        return s

    def autotune(self):
        a, b = C.c_int32(), C.c_int32()
        self._chk(lib().bm_batch_autotune(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def set_schedule(self, persistent, profit_threads=512, combine_tile=64):
        """persistent: one launch per sweep; else the launch sequence."""
        self._chk(lib().bm_batch_set_schedule(self.h, int(bool(persistent)), int(profit_threads), int(combine_tile)))

    def sweeps(self, k, max_candidates=0, max_verify=-1):
        o = SweepOpts(max_candidates, max_verify)
        c = np.zeros(self.k, np.int64)
        ms = C.c_float()
        self._chk(lib().bm_batch_sweeps(self.h, int(k), C.byref(o), _p(c), C.byref(ms)))
        return c, ms.value

    def info(self):
        vals = [C.c_int32(), C.c_int32(), C.c_int64(), C.c_int32(), C.c_int32()]
        self._chk(lib().bm_batch_info(self.h, *[C.byref(v) for v in vals]))
        return dict(zip(("count", "max_n", "total_pairs", "profit_threads", "combine_tile"), [v.value for v in vals]))


# ---- learned swap proposal ---------------------------------------------------
MLP_IN, MLP_HID = 128, 256


class Mlp:
    """The proposal network (128 -> 256 -> 256 -> 1) on the current CUDA device.

    Parameters are fp32 in the order W1[256][128], b1[256], W2[256][256],
    b2[256], w3[256], b3 (bm_mlp_param_count() values)."""

    def __init__(self, seed=0):
        h = C.c_void_p()
        st = lib().bm_mlp_create(C.byref(h), int(seed))
        if st != BM_OK:
            raise BMError(st, (lib().bm_mlp_last_error(None) or b"").decode())
        self.h = h
        self.count = int(lib().bm_mlp_param_count())

    def _chk(self, st):
        if st != BM_OK:
            raise BMError(st, (lib().bm_mlp_last_error(self.h) or b"").decode())

    def close(self):
        if getattr(self, "h", None):
            lib().bm_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def get_params(self):
        out = np.zeros(self.count, np.float32)
        self._chk(lib().bm_mlp_get_params(self.h, _p(out)))
        return out

    def set_params(self, params):
        params = np.ascontiguousarray(params, np.float32)
        assert params.size == self.count
        self._chk(lib().bm_mlp_set_params(self.h, _p(params)))

    def features(self, engine):
        """(F1, F2): per-vertex features of engine's graphs and current matching."""
        f1 = np.zeros((engine.n, 32), np.float32)
        f2 = np.zeros((engine.n, 32), np.float32)
        self._chk(lib().bm_mlp_features(self.h, engine.h, _p(f1), _p(f2)))
        return f1, f2

    def rank_pairs(self, engine, m1, m2):
        """Network scores of the 1-based pairs (m1[i], m2[i]) on engine's matching."""
        a = np.ascontiguousarray(m1, np.int32)
        b = np.ascontiguousarray(m2, np.int32)
        out = np.zeros(len(a), np.float32)
        self._chk(lib().bm_mlp_rank_pairs(self.h, engine.h, len(a), _p(a), _p(b), _p(out)))
        return out

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_IN)
        out = np.zeros(len(x), np.float32)
        self._chk(lib().bm_mlp_forward(self.h, len(x), _p(x), _p(out)))
        return out

    def train_step(self, x, target, lr=0.0, want_grads=True):
        """One forward/backward pass; returns (loss, grads or None)."""
        x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_IN)
        t = np.ascontiguousarray(target, np.float32)
        assert len(t) == len(x)
        loss = C.c_float()
        g = np.zeros(self.count, np.float32) if want_grads else None
        self._chk(lib().bm_mlp_train_step(self.h, len(x), _p(x), _p(t), float(lr), C.byref(loss),
                                          _p(g) if want_grads else None))
        return loss.value, g

    def train_from(self, engine, sweeps=2, extra_partners=16, epochs=1, lr=1e-2, seed=0):
        st = MlpTrainStats()
        self._chk(lib().bm_mlp_train_from(self.h, engine.h, int(sweeps), int(extra_partners), int(epochs),
                                          float(lr), int(seed), C.byref(st)))
        return dict(samples=st.samples, steps=st.steps, first_loss=st.first_loss, last_loss=st.last_loss)

    def learned_sweep(self, engine, pool=64, top_fraction=0.02, seed=0, per_row=0, retries=0):
        """One learned sweep of engine's matching; returns its stats with 'fell_back'."""
        o = LearnedOpts(int(pool), int(per_row), float(top_fraction), int(seed), int(retries), 0)
        s = SweepStats()
        fb = C.c_int32()
        self._chk(lib().bm_learned_sweep(engine.h, self.h, C.byref(o), C.byref(s), C.byref(fb)))
        d = {k: getattr(s, k) for k, _ in SweepStats._fields_ if k != "reserved"}
        d["fell_back"] = fb.value
        return d

    def learned_run(self, engine, max_sweeps=1000, target_score=0, probe_every=8, pool=64, top_fraction=0.02,
                    seed=0, per_row=0, retries=0, trace=False):
        """The learned-proposal descent (bm_learned_run); returns its stats, and
        with trace=True also per-step arrays score, ms (cumulative) and kind."""
        o = LearnedOpts(int(pool), int(per_row), float(top_fraction), int(seed), int(retries), 0)
        st = LearnedRunStats()
        if trace:
            sc = np.zeros(max(max_sweeps, 1), np.int64)
            ms = np.zeros(max(max_sweeps, 1), np.float32)
            kd = np.zeros(max(max_sweeps, 1), np.int8)
            ptrs = (_p(sc), _p(ms), _p(kd))
        else:
            ptrs = (None, None, None)
        self._chk(lib().bm_learned_run(engine.h, self.h, C.byref(o), int(max_sweeps), int(target_score),
                                       int(probe_every), C.byref(st), *ptrs))
        d = {k: getattr(st, k) for k, _ in LearnedRunStats._fields_ if not k.startswith("reserved")}
        if trace:
            k = st.sweeps
            d.update(trace_score=sc[:k].copy(), trace_ms=ms[:k].copy(), trace_kind=kd[:k].copy())
        return d
