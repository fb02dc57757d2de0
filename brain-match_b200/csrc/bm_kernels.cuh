// bm_kernels.cuh -- sm_100a device code of the swap-delta engine.
//
// Notation (0-based inside the engine; the C ABI is 1-based like the
// reference):  G1 vertices a,b,u,v in [0,n);  G2 vertices f,g in [0,n);
// p: G1 -> G2 (value n = unmatched, "NONE");  pinv: G2 -> G1 (n = NONE).
// W2 is G2's dense (n+1)x(n+1) weight matrix whose row and column n are 0,
// which plays the role of the reference's unused row/column 0.
//
// Profit matrix.  For every ordered pair (a,b) of G1 vertices
//     S[a][b] = sum_{(a,v,w) in out1(a)} min(w, W2[p b][p v])
//             + sum_{(u,a,w) in in1(a)}  min(w, W2[p u][p b])
//             + unary self-loop terms + per-edge corner corrections
// i.e. the score a would earn by taking p(b) while everyone else stays.
// S[a][a] is a's current contribution, and the exact swap delta is
//     delta(a,b) = S[a][b] + S[b][a] - S[a][a] - S[b][b]
// once the corner corrections below are folded into S.  This is the same
// arithmetic as calculate_swap_delta (src/graph-alignment-optimized.c:321-408)
// regrouped by row: the reference skips the partner in each edge list and adds
// the two a<->b edges separately; here those terms are removed or replaced by
// the correction  min(x,W2[pa][pb]) + min(x,W2[pb][pa]) - min(x,W2[pa][pa])
// - min(x,W2[pb][pb])  added to S[a][b] for every G1 edge a->b of weight x.
//
// S is accumulated sparse x sparse: for each out-edge (a,v,w1) of a, every
// G2 in-edge (g -> p(v), w2) contributes min(w1,w2) to S[a][pinv(g)]; for each
// in-edge (u,a,w1), every G2 out-edge (p(u) -> g, w2) contributes to
// S[a][pinv(g)].  Only nonzero min terms are ever touched.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace bm {

// ---- list entries: (id, weight) packed per storage mode ----
template <bool W16> struct Ent;
template <> struct Ent<true> {
    typedef uint32_t T;  // id in bits 0..15, weight in bits 16..31
    static __host__ __device__ __forceinline__ int id(T e) { return (int)(e & 0xFFFFu); }
    static __host__ __device__ __forceinline__ int w(T e) { return (int)(e >> 16); }
    static __host__ __device__ __forceinline__ T make(int i, int w) { return (uint32_t)i | ((uint32_t)w << 16); }
};
template <> struct Ent<false> {
    typedef int2 T;  // x = id, y = weight
    static __host__ __device__ __forceinline__ int id(T e) { return e.x; }
    static __host__ __device__ __forceinline__ int w(T e) { return e.y; }
    static __host__ __device__ __forceinline__ T make(int i, int w) { return make_int2(i, w); }
};
template <bool W16> struct Dense;
template <> struct Dense<true> { typedef uint16_t T; };
template <> struct Dense<false> { typedef int32_t T; };

// Device view of a context.
template <bool W16> struct DevView {
    typedef typename Ent<W16>::T E;
    typedef typename Dense<W16>::T D;
    int n;
    const int* off1o; const E* ent1o;   // G1 out-lists (id = dst)
    const int* off1i; const E* ent1i;   // G1 in-lists  (id = src)
    const int* off2o; const E* ent2o;   // G2 out-lists (id = dst)
    const int* off2i; const E* ent2i;   // G2 in-lists  (id = src)
    const int* offs;  const int* selfw; // G1 self-loops per vertex
    E* ent1oP; E* ent1iP;               // G1 lists with ids mapped through p
    E* ent2oP; E* ent2iP;               // G2 lists with ids mapped through pinv
    const int* off2oH; E* ent2oHP;      // G2 out-entries above the hub threshold, mapped through pinv
    const D* W2;                        // dense (n+1)^2, row/col n zero
    const D* W2T;                       // its transpose (columns of W2 read as rows)
    const int* W2D;                     // its diagonal W2[f][f], f = 0..n
    int* p; int* pinv;                  // n+1 entries, [n] = n
    int* S;                             // n*n profit matrix
    __device__ __forceinline__ int w2(int f, int g) const {
        return (int)W2[(size_t)f * (size_t)(n + 1) + (size_t)g];
    }
    // same value as w2(f, g), read from row g of the transpose
    __device__ __forceinline__ int w2t(int f, int g) const {
        return (int)W2T[(size_t)g * (size_t)(n + 1) + (size_t)f];
    }
    // same value as w2(f, f)
    __device__ __forceinline__ int w2d(int f) const { return W2D[f]; }
};

__device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }

// ---------------------------------------------------------------------------
// Relabel list ids through a map (p for G1 lists, pinv for G2 lists).
template <bool W16>
__global__ void k_relabel(const typename Ent<W16>::T* __restrict__ in,
                          typename Ent<W16>::T* __restrict__ out, long long m,
                          const int* __restrict__ map) {
    typedef Ent<W16> EN;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long stride = (long long)gridDim.x * blockDim.x;
    for (; i < m; i += stride) {
        typename EN::T e = in[i];
        out[i] = EN::make(__ldg(&map[EN::id(e)]), EN::w(e));
    }
}

// Work estimate of a profit row: number of min terms it scatters.
template <bool W16>
__global__ void k_row_work(DevView<W16> g, const unsigned char* __restrict__ is_hub,
                           unsigned long long* __restrict__ key, int* __restrict__ val,
                           unsigned long long* __restrict__ total) {
    typedef Ent<W16> EN;
    const int lane = threadIdx.x & 31;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int a = warp; a < g.n; a += nwarps) {
        long long w = 0;
        for (int i = g.off1o[a] + lane; i < g.off1o[a + 1]; i += 32) {
            int f = EN::id(g.ent1oP[i]);
            w += g.off2i[f + 1] - g.off2i[f];
        }
        for (int i = g.off1i[a] + lane; i < g.off1i[a + 1]; i += 32) {
            if (is_hub && is_hub[EN::id(g.ent1i[i])]) continue;  // tensor-core term
            int f = EN::id(g.ent1iP[i]);
            w += g.off2o[f + 1] - g.off2o[f];
        }
        for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (lane == 0) {
            if (total) atomicAdd(total, (unsigned long long)w);   // min terms the row scatters
            w += (g.off1o[a + 1] - g.off1o[a]) + (g.off1i[a + 1] - g.off1i[a]);
            if (g.offs[a + 1] > g.offs[a]) w += g.n;
            key[a] = (unsigned long long)min(w, 0xffffffffLL);   // 32-bit sort keys
            val[a] = a;
        }
    }
}

// ---------------------------------------------------------------------------
// Profit rows.  Persistent CTAs take rows from `order` (heaviest first) via an
// atomic counter, accumulate the row in shared memory (n+1 ints: slot n
// absorbs terms for unmatched G2 vertices) and write it to S[a][0..n).
// Inside a row, warps take the row's G1 edges round robin and scatter the
// matching G2 list; lists longer than kLongList are queued and then scattered
// by the whole CTA, so a few hub lists cannot hold the row's barrier.
// The queue is small enough (1 KB) that three CTAs of 512 threads with an
// N = 18,524 row each (74 KB) share one SM; a row that queues more scatters
// the rest warp by warp.
constexpr int kLongList = 4096;
constexpr int kLongQueue = 128;

// Scatters min(w1, w2) over list[i0, i1) into acc, lanes striding by `step`.
template <bool W16>
__device__ __forceinline__ void scatter_list(int* acc, const typename Ent<W16>::T* __restrict__ list,
                                             int i0, int i1, int w1, int first, int step) {
    typedef Ent<W16> EN;
    typedef typename EN::T E;
    int i = i0 + first;
    for (; i + 7 * step < i1; i += 8 * step) {  // eight loads in flight per thread
        E x[8];
#pragma unroll
        for (int u = 0; u < 8; u++) x[u] = list[i + u * step];
#pragma unroll
        for (int u = 0; u < 8; u++) atomicAdd(&acc[EN::id(x[u])], imin(w1, EN::w(x[u])));
    }
    for (; i + 3 * step < i1; i += 4 * step) {
        const E x0 = list[i], x1 = list[i + step], x2 = list[i + 2 * step], x3 = list[i + 3 * step];
        atomicAdd(&acc[EN::id(x0)], imin(w1, EN::w(x0)));
        atomicAdd(&acc[EN::id(x1)], imin(w1, EN::w(x1)));
        atomicAdd(&acc[EN::id(x2)], imin(w1, EN::w(x2)));
        atomicAdd(&acc[EN::id(x3)], imin(w1, EN::w(x3)));
    }
    for (; i < i1; i += step) { const E x = list[i]; atomicAdd(&acc[EN::id(x)], imin(w1, EN::w(x))); }
}

// Hub residual: terms of a hub in-edge (u,a,w1) above the threshold T that
// the tensor-core GEMM does not cover, min(w1,w2) - T for w1 > T, over the
// G2 out-entries of p(u) whose weight w2 is above T.
template <bool W16>
__device__ __forceinline__ void scatter_residual(int* acc, const typename Ent<W16>::T* __restrict__ list,
                                                 int i0, int i1, int w1, int thr, int first, int step) {
    typedef Ent<W16> EN;
    for (int i = i0 + first; i < i1; i += step) {
        const typename EN::T x = list[i];
        atomicAdd(&acc[EN::id(x)], imin(w1, EN::w(x)) - thr);
    }
}

// One profit row of S by a group of threads that all call it together: the
// whole block (NT = 0), or the NT threads (a power of two) of the block's
// NT-aligned group; `sync` is a barrier over exactly those threads.  It ends
// with a barrier.  acc holds n+1 ints of shared memory.
// With `work`, the row also records its scheduling key for the next rebuild
// (its scattered min terms + its edges + n if it has self-loops, the
// estimate k_row_work makes) in work[a], and adds its terms to *work_total.
template <bool W16, int NT, typename Sync>
__device__ __forceinline__ void profit_row_on(const DevView<W16>& g, int a, int* acc, int2* s_long, int* s_nlong,
                                              const unsigned char* __restrict__ is_hub, int hub_thr, int* s_terms,
                                              unsigned long long* work, unsigned long long* work_total, Sync sync) {
    static_assert(NT == 0 || (NT & (NT - 1)) == 0, "group size is a power of two");
    typedef Ent<W16> EN;
    typedef typename EN::T E;
    const int n = g.n;
    const int tid = NT ? (int)(threadIdx.x & (NT - 1)) : (int)threadIdx.x;
    const int nthr = NT ? NT : (int)blockDim.x;
    const int lane = tid & 31, wid = tid >> 5, nw = nthr >> 5;
    if (tid == 0) {
        *s_nlong = 0;
        if (work) *s_terms = 0;
    }
    // the row's scattered terms start from zero; with hubs, the tensor-core
    // hub terms already in S are added when the row is written back
    if ((n & 3) == 0) {
        int4* a4 = reinterpret_cast<int4*>(acc);
        for (int i = tid; i < (n >> 2); i += nthr) a4[i] = make_int4(0, 0, 0, 0);
        if (tid == 0) acc[n] = 0;
    } else {
        for (int i = tid; i <= n; i += nthr) acc[i] = 0;
    }
    sync();
    // out-edges of a against G2 in-lists of p(v), then in-edges against out-lists of p(u)
    const int so = g.off1o[a], lo = g.off1o[a + 1] - so;
    const int si = g.off1i[a], li = g.off1i[a + 1] - si;
    // the warp's edges are j = wid + nw * t; lane t loads the set-up of its t-th
    // edge (entry, list extent, kind) so one round of loads serves 32 edges
    const int tot = lo + li;
    for (int base = wid; base < tot; base += nw * 32) {
        const int j = base + nw * lane;
        int f = 0, w1 = 0, b0 = 0, b1 = 0, kind = 0;  // kind: 0 none, 1 out-edge, 2 in-edge, 3 hub residual
        if (j < tot) {
            const bool out = j < lo;
            const E ea = out ? g.ent1oP[so + j] : g.ent1iP[si + (j - lo)];
            f = EN::id(ea);
            w1 = EN::w(ea);
            if (!out && is_hub && is_hub[EN::id(g.ent1i[si + (j - lo)])]) {
                // hub in-edge: the GEMM has its terms up to the threshold
                if (w1 > hub_thr) { kind = 3; b0 = g.off2oH[f]; b1 = g.off2oH[f + 1]; }
            } else {
                kind = out ? 1 : 2;
                const int* off = out ? g.off2i : g.off2o;
                b0 = off[f];
                b1 = off[f + 1];
            }
        }
        if (work) {   // the chunk's scattered terms
            int c = kind ? b1 - b0 : 0;
            for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0 && c) atomicAdd(s_terms, c);
        }
        const int cnt = min(32, (tot - base + nw - 1) / nw);
        for (int t = 0; t < cnt; t++) {
            const int kt = __shfl_sync(0xffffffffu, kind, t);
            const int w1t = __shfl_sync(0xffffffffu, w1, t);
            const int b0t = __shfl_sync(0xffffffffu, b0, t);
            const int b1t = __shfl_sync(0xffffffffu, b1, t);
            const int ft = __shfl_sync(0xffffffffu, f, t);
            if (kt == 0) continue;
            if (kt == 3) {
                scatter_residual<W16>(acc, g.ent2oHP, b0t, b1t, w1t, hub_thr, lane, 32);
                continue;
            }
            const bool out = kt == 1;
            if (b1t - b0t > kLongList) {
                int q = 0;
                if (lane == 0) q = atomicAdd(s_nlong, 1);
                q = __shfl_sync(0xffffffffu, q, 0);
                if (q < kLongQueue) {
                    if (lane == 0) s_long[q] = make_int2(ft, w1t | (out ? 0 : (int)0x80000000));
                    continue;
                }
            }
            scatter_list<W16>(acc, out ? g.ent2iP : g.ent2oP, b0t, b1t, w1t, lane, 32);
        }
    }
    sync();
    // long lists, one at a time, by the whole block
    const int nl = min(*s_nlong, kLongQueue);
    for (int q = 0; q < nl; q++) {
        const int2 e = s_long[q];
        const bool out = e.y >= 0;
        const int w1 = e.y & 0x7fffffff;
        const int* off = out ? g.off2i : g.off2o;
        const E* list = out ? g.ent2iP : g.ent2oP;
        scatter_list<W16>(acc, list, off[e.x], off[e.x + 1], w1, tid, nthr);
    }
    // corner corrections for every G1 edge a->b
    {
        const int pa = g.p[a];
        const int dpa = g.w2d(pa);
        for (int j = tid; j < lo; j += nthr) {
            const int b = EN::id(g.ent1o[so + j]);
            const E ep = g.ent1oP[so + j];
            const int pb = EN::id(ep), x = EN::w(ep);
            const int c = imin(x, g.w2(pa, pb)) + imin(x, g.w2t(pb, pa))
                        - imin(x, dpa) - imin(x, g.w2d(pb));
            if (c) atomicAdd(&acc[b], c);
        }
    }
    // unary terms of G1 self-loops: a taking p(b) earns min(s, W2[p b][p b])
    {
        const int q0 = g.offs[a], q1 = g.offs[a + 1];
        if (q1 > q0) {
            sync();
            for (int b = tid; b < n; b += nthr) {
                const int pb = g.p[b];
                const int d = g.w2d(pb);
                int t = 0;
                for (int q = q0; q < q1; q++) t += imin(g.selfw[q], d);
                acc[b] += t;
            }
        }
    }
    sync();
    if (work && tid == 0) {
        const long long terms = *s_terms;
        atomicAdd(work_total, (unsigned long long)terms);
        long long w = terms + tot + (g.offs[a + 1] > g.offs[a] ? n : 0);
        work[a] = (unsigned long long)min(w, 0xffffffffLL);
    }
    int* row = g.S + (size_t)a * (size_t)n;
    if ((n & 3) == 0) {
        int4* r4 = reinterpret_cast<int4*>(row);
        const int4* a4 = reinterpret_cast<const int4*>(acc);
        if (is_hub) {
            const int n4 = n >> 2;
            int i = tid;
            for (; i + 3 * (int)nthr < n4; i += 4 * nthr) {
                int4 h[4];
#pragma unroll
                for (int u = 0; u < 4; u++) h[u] = r4[i + u * nthr];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int4 v = a4[i + u * nthr];
                    r4[i + u * nthr] = make_int4(h[u].x + v.x, h[u].y + v.y, h[u].z + v.z, h[u].w + v.w);
                }
            }
            for (; i < n4; i += nthr) {
                const int4 h = r4[i], v = a4[i];
                r4[i] = make_int4(h.x + v.x, h.y + v.y, h.z + v.z, h.w + v.w);
            }
        } else {
            for (int i = tid; i < (n >> 2); i += nthr) r4[i] = a4[i];
        }
    } else {
        if (is_hub) for (int i = tid; i < n; i += nthr) row[i] += acc[i];
        else for (int i = tid; i < n; i += nthr) row[i] = acc[i];
    }
    sync();
}

// One profit row of S by the whole block (all threads call it together; it
// ends with a barrier).
template <bool W16>
__device__ __forceinline__ void profit_row(const DevView<W16>& g, int a, int* acc, int2* s_long, int* s_nlong,
                                           const unsigned char* __restrict__ is_hub, int hub_thr,
                                           int* s_terms = nullptr, unsigned long long* work = nullptr,
                                           unsigned long long* work_total = nullptr) {
    profit_row_on<W16, 0>(g, a, acc, s_long, s_nlong, is_hub, hub_thr, s_terms, work, work_total,
                          [] { __syncthreads(); });
}

template <bool W16>
__global__ void __launch_bounds__(512, 3)
k_profit(DevView<W16> g, const int* __restrict__ order, int* __restrict__ counter,
         const unsigned char* __restrict__ is_hub, int hub_thr, unsigned long long* __restrict__ work,
         unsigned long long* __restrict__ work_total) {
    extern __shared__ int acc[];
    __shared__ int s_row, s_nlong, s_terms;
    __shared__ int2 s_long[kLongQueue];  // (G2 vertex, w1 | kind << 31)
    for (;;) {
        if (threadIdx.x == 0) s_row = atomicAdd(counter, 1);
        __syncthreads();
        const int r = s_row;
        if (r >= g.n) break;
        profit_row<W16>(g, order[r], acc, s_long, &s_nlong, is_hub, hub_thr, &s_terms, work, work_total);
    }
}

// ---------------------------------------------------------------------------
// Per-row best partner as a packed key  (delta + 2^31) << 32 | ~b  (larger
// delta, then smaller b, wins).
__device__ __forceinline__ unsigned long long pack_best(int d, int b) {
    return ((unsigned long long)(unsigned)(d + 0x80000000u) << 32) | (unsigned)(~b);
}
__device__ __forceinline__ unsigned long long kmax(unsigned long long x, unsigned long long y) {
    return x > y ? x : y;
}

// Candidate keys: one per row whose best partner improves, deduplicated when
// two rows pick each other.  Sort key: (0x7fffffff - delta) << 32 | lo << 16 | hi
// -> ascending order = delta desc, lo asc, hi asc.  Rows without a candidate
// get ~0.
static __global__ void k_candidates(const unsigned long long* __restrict__ rowbest, int n,
                             unsigned long long* __restrict__ keys, int* __restrict__ ncand,
                             int* __restrict__ best_delta) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const unsigned long long k = rowbest[a];
    unsigned long long out = ~0ull;
    if (k) {
        const int d = (int)((unsigned)(k >> 32) - 0x80000000u);
        const int b = (int)(~(unsigned)(k & 0xffffffffu));
        if (d > 0) {
            atomicMax(best_delta, d);
            const unsigned long long kb = rowbest[b];
            const int bb = (int)(~(unsigned)(kb & 0xffffffffu));
            const bool mutual = (kb != 0) && (bb == a);
            if (!mutual || a < b) {
                const int lo = a < b ? a : b, hi = a < b ? b : a;
                out = ((unsigned long long)(0x7fffffffu - (unsigned)d) << 32) |
                      ((unsigned long long)lo << 16) | (unsigned long long)hi;
                atomicAdd(ncand, 1);
            }
        }
    }
    keys[a] = out;
}

// ---------------------------------------------------------------------------
// Exact swap delta of (a,b) on the current matching, one element of the four
// edge lists per thread of the group, as calculate_swap_delta computes it
// (src/graph-alignment-optimized.c:321-408), plus the exact self-loop terms.
template <bool W16>
__device__ __forceinline__ int swap_delta_part(const DevView<W16>& g, int a, int b, int t, int nt) {
    typedef Ent<W16> EN;
    const int pa = g.p[a], pb = g.p[b];
    int d = 0;
    const int la0 = g.off1o[a], la = g.off1o[a + 1] - la0;
    const int ia0 = g.off1i[a], ia = g.off1i[a + 1] - ia0;
    const int lb0 = g.off1o[b], lb = g.off1o[b + 1] - lb0;
    const int ib0 = g.off1i[b], ib = g.off1i[b + 1] - ib0;
    const int tot = la + ia + lb + ib;
    for (int k = t; k < tot; k += nt) {
        int q = k;
        if (q < la) {  // out-edge a->v
            const typename EN::T e = g.ent1o[la0 + q];
            const int v = EN::id(e), w = EN::w(e);
            if (v == b) d += imin(w, g.w2(pb, pa)) - imin(w, g.w2(pa, pb));
            else { const int pv = g.p[v]; d += imin(w, g.w2(pb, pv)) - imin(w, g.w2(pa, pv)); }
            continue;
        }
        q -= la;
        if (q < ia) {  // in-edge u->a
            const typename EN::T e = g.ent1i[ia0 + q];
            const int u = EN::id(e), w = EN::w(e);
            if (u != b) { const int pu = g.p[u]; d += imin(w, g.w2(pu, pb)) - imin(w, g.w2(pu, pa)); }
            continue;  // the edge b->a is counted once, from b's out-list
        }
        q -= ia;
        if (q < lb) {  // out-edge b->v
            const typename EN::T e = g.ent1o[lb0 + q];
            const int v = EN::id(e), w = EN::w(e);
            if (v == a) d += imin(w, g.w2(pa, pb)) - imin(w, g.w2(pb, pa));
            else { const int pv = g.p[v]; d += imin(w, g.w2(pa, pv)) - imin(w, g.w2(pb, pv)); }
            continue;
        }
        q -= lb;
        {  // in-edge u->b
            const typename EN::T e = g.ent1i[ib0 + q];
            const int u = EN::id(e), w = EN::w(e);
            if (u != a) { const int pu = g.p[u]; d += imin(w, g.w2(pu, pa)) - imin(w, g.w2(pu, pb)); }
        }
    }
    if (t == 0) {
        for (int q = g.offs[a]; q < g.offs[a + 1]; q++)
            d += imin(g.selfw[q], g.w2(pb, pb)) - imin(g.selfw[q], g.w2(pa, pa));
        for (int q = g.offs[b]; q < g.offs[b + 1]; q++)
            d += imin(g.selfw[q], g.w2(pa, pa)) - imin(g.selfw[q], g.w2(pb, pb));
    }
    return d;
}

// One warp per requested pair.
template <bool W16>
__global__ void k_pair_deltas(DevView<W16> g, const int* __restrict__ pa, const int* __restrict__ pb,
                              long long k, int* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (; w < k; w += nw) {
        int d = swap_delta_part<W16>(g, pa[w], pb[w], lane, 32);
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) out[w] = d;
    }
}

// Alignment score (src/graph-alignment-optimized.c:292-307): one warp per row.
template <bool W16>
__global__ void k_score(DevView<W16> g, unsigned long long* __restrict__ out) {
    typedef Ent<W16> EN;
    const int lane = threadIdx.x & 31;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    long long s = 0;
    for (int a = warp; a < g.n; a += nwarps) {
        const int pa = g.p[a];
        for (int i = g.off1o[a] + lane; i < g.off1o[a + 1]; i += 32) {
            const typename EN::T e = g.ent1o[i];
            s += imin(EN::w(e), g.w2(pa, g.p[EN::id(e)]));
        }
        if (lane == 0)
            for (int q = g.offs[a]; q < g.offs[a + 1]; q++) s += imin(g.selfw[q], g.w2(pa, pa));
    }
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0 && s) atomicAdd(out, (unsigned long long)s);
}

// ---------------------------------------------------------------------------
// Counters reported by the commit kernels.
struct CommitStats {
    long long total_delta;
    int scanned, verified, committed, steps;
    long long entries;
    int carried, pad;
};

}  // namespace bm
