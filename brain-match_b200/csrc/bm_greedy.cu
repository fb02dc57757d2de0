// bm_greedy.cu -- the greedy feature matcher (src/greedy-feature-match.c:
// 527-712) on the GPU: an initial matching for the swap search.
//
// Vertex features (compute_vertex_features, :527-566): in- and out-degree
// (every list entry: repeated edges and self-loops count), the number of
// distinct vertices reachable in exactly two out-steps and the number that
// reach the vertex in two in-steps, and their sum ("total").  G1 vertices are
// matched one at a time in order of total (descending; ties by id, where the
// reference's qsort leaves the order unspecified), each to the unmatched G2
// vertex of largest
//     0.3 * -distance + 0.7 * align            (:633-647)
// with distance = (int)(1000 * sum_k |ratio1_k - ratio2_k|) over the four
// feature/total ratios (compute_feature_distance, :575-586) and align the
// edge overlap with the G1 neighbours matched so far:
//     sum_{v1->t, t matched} min(w, W2[v2][m t]) + sum_{s->v1, s matched} min(w, W2[m s][v2])
// (compute_edge_alignment, :297-356, with its evident intent: the reference
// compares G2 ids against G2 indices and tests a G1 vertex against G2 position
// flags).  Among equal scores the first candidate in G2's feature order wins,
// as the reference's strict ">" does.  A vertex without any edge (total 0,
// where the reference divides 0/0) has all ratios 0.  W2 is the last weight
// given for a G2 pair, which is what the reference's prepended lists find first.
//
// The sequential loop runs as one cooperative grid, a CTA per SM: each step
// scatters the align terms through the G2 lists of the matched neighbours'
// images into an L2-resident array (the list entries spread evenly over all
// threads of the grid), every CTA takes the best of its own slice of
// candidates, and every CTA reduces the published slice bests -- one bounded
// grid barrier per step (the scatter of step i+1 runs before step i's decision
// is reduced: only edges to step i's vertex need it, and those are added per
// slice afterwards).
#include <cub/cub.cuh>
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "bm.h"
#include "bm_internal.cuh"

namespace bm {
namespace {

constexpr int kGreedyThreads = 512;
constexpr int kGreedyUnroll = 4;   // list entries a thread has in flight in the align scatter
constexpr int kGreedyMaxFix = 32;  // edges to the previous step's vertex recorded (more: rescanned)
constexpr unsigned kGreedySpinLimit = 1u << 24;  // polls of one grid-barrier wait (~1 s)

struct GreedyBest {
    double score;
    int pos;  // candidate's place in G2's feature order
    int g;    // candidate (0-based), -1 none
};

__device__ __forceinline__ bool better(const GreedyBest& x, const GreedyBest& y) {
    return x.score > y.score || (x.score == y.score && x.pos < y.pos);
}

// Distinct vertices at the end of a two-step walk along the lists (off, id):
// cnt[u] = |{w : u -> v -> w}|.  One CTA per vertex, a bitmap of n bits in
// shared memory.
__global__ void k_two_hop(const int* __restrict__ off, const int* __restrict__ id, int n, int* __restrict__ cnt) {
    extern __shared__ unsigned bits[];
    __shared__ int part[32];
    const int words = (n + 31) >> 5;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int u = blockIdx.x; u < n; u += gridDim.x) {
        for (int i = threadIdx.x; i < words; i += blockDim.x) bits[i] = 0u;
        __syncthreads();
        for (int j = off[u] + wid; j < off[u + 1]; j += nw) {
            const int v = id[j];
            for (int k = off[v] + lane; k < off[v + 1]; k += 32) {
                const int w = id[k];
                atomicOr(&bits[w >> 5], 1u << (w & 31));
            }
        }
        __syncthreads();
        int c = 0;
        for (int i = threadIdx.x; i < words; i += blockDim.x) c += __popc(bits[i]);
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) part[wid] = c;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < nw; w++) t += part[w];
            cnt[u] = t;
        }
        __syncthreads();
    }
}

// Features (in, out, 2-hop out, 2-hop in), the four ratios to their total and
// the sort key (total descending, id ascending).
__global__ void k_features(const int* __restrict__ offo, const int* __restrict__ offi, const int* __restrict__ r2,
                           const int* __restrict__ c2, int n, int4* __restrict__ feat, double4* __restrict__ ratio,
                           unsigned long long* __restrict__ key, int* __restrict__ val) {
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    const int in = offi[v + 1] - offi[v], out = offo[v + 1] - offo[v];
    const int4 f = make_int4(in, out, r2[v], c2[v]);
    const int total = f.x + f.y + f.z + f.w;
    feat[v] = f;
    double4 r = make_double4(0.0, 0.0, 0.0, 0.0);
    if (total > 0) {
        const double t = (double)total;
        r = make_double4(__ddiv_rn((double)f.x, t), __ddiv_rn((double)f.y, t), __ddiv_rn((double)f.z, t),
                         __ddiv_rn((double)f.w, t));
    }
    ratio[v] = r;
    key[v] = ((unsigned long long)(0xffffffffu - (unsigned)total) << 32) | (unsigned)v;
    val[v] = v;
}

__global__ void k_positions(const int* __restrict__ order, int n, int* __restrict__ pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pos[order[i]] = i;
}

struct GreedyArgs {
    int n, slice;
    const int *off1o, *id1o, *w1o, *off1i, *id1i, *w1i;  // G1, every entry
    const int *off2o, *id2o, *w2o, *off2i, *id2i, *w2i;  // G2, one entry per pair (last weight)
    const int* order1;                                    // G1 in feature order
    const int* pos2;                                      // G2 vertex -> place in feature order
    const double4 *ratio1, *ratio2;
    int* acc;                                             // [2][n] align sums by step parity, zero between uses
    GreedyBest* bests;                                    // [2][gridDim.x] per-CTA bests
    unsigned* bar;                                        // [0] arrivals [1] generation [2] error
    int* map;                                             // out: G1 -> G2 (0-based)
    int stall;                                            // test hook: CTA 0 skips the first arrival
};

// Score of candidate g for the G1 vertex with ratios r1: the reference's
// double arithmetic, every operation rounded once (no contraction).
__device__ __forceinline__ double greedy_score(const double4& r1, const double4& r2, int align) {
    double d = fabs(__dsub_rn(r1.x, r2.x));
    d = __dadd_rn(d, fabs(__dsub_rn(r1.y, r2.y)));
    d = __dadd_rn(d, fabs(__dsub_rn(r1.z, r2.z)));
    d = __dadd_rn(d, fabs(__dsub_rn(r1.w, r2.w)));
    const int dist = __double2int_rz(__dmul_rn(d, 1000.0));
    return __dadd_rn(__dmul_rn(0.3, (double)(-dist)), __dmul_rn(0.7, (double)align));
}

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of the co-resident CTAs.  Each wait is bounded: after
// kGreedySpinLimit polls the CTA records the error word and every CTA leaves
// at its next barrier.  Returns false once the error word is set.  With
// `stall` (the bm_test_stall hook) CTA 0 does not arrive and every CTA polls
// only a few thousand times, so the barrier never completes and every CTA
// leaves at it.
__device__ bool grid_barrier(unsigned* bar, bool stall = false) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        const unsigned gen = ld_acquire_u32(&bar[1]);
        const unsigned limit = stall ? (1u << 12) : kGreedySpinLimit;
        if (!(stall && blockIdx.x == 0) && atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            unsigned it = 0;
            while (ld_acquire_u32(&bar[1]) == gen) {
                if (ld_acquire_u32(&bar[2]) || ++it > limit) {
                    atomicExch(&bar[2], 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok && !ld_acquire_u32(&bar[2]);
    }
    __syncthreads();
    return s_ok != 0;
}

// The grid's best of a step, reduced by every CTA from the published slice
// bests (buffer par): v's image in map_s, the candidate taken if it is in this
// CTA's slice [base, base + len), the output by CTA 0.  All threads call it.
__device__ void greedy_decide(const GreedyArgs& a, int par, int v, int* map_s, unsigned char* taken, int base,
                              int len, GreedyBest* wbest) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    GreedyBest best{-1.0 / 0.0, 0x7fffffff, -1};
    for (int r = tid; r < (int)gridDim.x; r += blockDim.x) {
        const GreedyBest* src = a.bests + par * gridDim.x + r;
        const GreedyBest c{__ldcg(&src->score), __ldcg(&src->pos), __ldcg(&src->g)};
        if (better(c, best)) best = c;
    }
    for (int o = 16; o; o >>= 1) {
        GreedyBest y;
        y.score = __shfl_xor_sync(0xffffffffu, best.score, o);
        y.pos = __shfl_xor_sync(0xffffffffu, best.pos, o);
        y.g = __shfl_xor_sync(0xffffffffu, best.g, o);
        if (better(y, best)) best = y;
    }
    if (lane == 0) wbest[wid] = best;
    __syncthreads();
    if (tid == 0) {
        for (int w = 1; w < kGreedyThreads / 32; w++)
            if (better(wbest[w], best)) best = wbest[w];
        map_s[v] = best.g;
        if (best.g >= base && best.g < base + len) taken[best.g - base] = 1;
        if (blockIdx.x == 0) a.map[v] = best.g;
    }
    __syncthreads();
}

// The sequential matching, one CTA per SM (cooperative launch).  Step i:
// the list entries of v1's edges are spread evenly over all threads of the
// grid, which scatter the align terms into acc (global, L2-resident), then
// every CTA takes the best candidate of its own slice of G2, then
// all CTAs reduce the slices' bests, each from the same published array.
__global__ void __launch_bounds__(kGreedyThreads, 1) k_greedy(GreedyArgs a) {
    extern __shared__ double4 gsm4[];
    double4* r2_s = gsm4;                                // slice: ratios of this CTA's candidates
    int* map_s = reinterpret_cast<int*>(r2_s + a.slice); // n: G1 -> G2, -1 unmatched (a copy per CTA)
    int* pos_s = map_s + a.n;                            // slice
    unsigned char* taken = reinterpret_cast<unsigned char*>(pos_s + a.slice);
    __shared__ GreedyBest wbest[kGreedyThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int base = blockIdx.x * a.slice;
    const int len = max(0, min(a.slice, a.n - base));
    for (int i = tid; i < a.n; i += blockDim.x) map_s[i] = -1;
    for (int l = tid; l < a.slice; l += blockDim.x) {
        taken[l] = l < len ? 0 : 1;
        pos_s[l] = l < len ? a.pos2[base + l] : 0x7fffffff;
        r2_s[l] = l < len ? a.ratio2[base + l] : make_double4(0.0, 0.0, 0.0, 0.0);
    }
    __syncthreads();
    typedef cub::BlockScan<int, kGreedyThreads> Scan;
    __shared__ typename Scan::TempStorage scan_tmp;
    __shared__ int s_pre[kGreedyThreads + 1];   // prefix of the chunk's list lengths
    __shared__ int s_beg[kGreedyThreads];       // list start of each edge of the chunk
    __shared__ int s_w[kGreedyThreads];         // its G1 weight, bit 31 set for an in-edge
    const long long gt = (long long)blockIdx.x * kGreedyThreads + tid;
    const long long gthreads = (long long)gridDim.x * kGreedyThreads;
    // the head of a step -- its vertex, edge extents and this thread's edge of
    // the first chunk -- does not depend on the previous decision: it is
    // loaded one step ahead, while the previous step's candidates are scored
    int nv = a.order1[0], no0 = a.off1o[nv], ndout = a.off1o[nv + 1] - no0;
    int ni0 = a.off1i[nv], ndin = a.off1i[nv + 1] - ni0;
    int nt = 0, nwt = 0;
    if (tid < ndout + ndin) {
        nt = tid < ndout ? a.id1o[no0 + tid] : a.id1i[ni0 + tid - ndout];
        nwt = tid < ndout ? a.w1o[no0 + tid] : a.w1i[ni0 + tid - ndout];
    }
    // the edges of a step's vertex to the previous step's vertex (whose image is
    // decided only after this step's scatter): their indices, then their terms
    // added per slice once the image is known
    __shared__ int s_nfix, s_fix[kGreedyMaxFix];
    if (tid == 0) s_nfix = 0;
    __syncthreads();
    int prev = -1;
    for (int step = 0; step < a.n; step++) {
        const int par = step & 1;
        int* acc = a.acc + (size_t)par * a.n;
        const int v1 = nv, o0 = no0, dout = ndout, i0 = ni0, din = ndin;
        // ---- align terms: v1's edges in chunks of one per thread; every CTA
        // computes the chunk's list extents, and the chunk's list entries are
        // spread evenly over all threads of the grid; an edge to the previous
        // step's vertex is recorded and left for later ----
        for (int c0 = 0; c0 < dout + din; c0 += kGreedyThreads) {
            const int j = c0 + tid;
            int beg = 0, len = 0, wv = 0;
            if (j < dout + din) {
                const bool out = j < dout;
                const int t = c0 == 0 ? nt : out ? a.id1o[o0 + j] : a.id1i[i0 + j - dout];
                const int w = c0 == 0 ? nwt : out ? a.w1o[o0 + j] : a.w1i[i0 + j - dout];
                if (t == prev) {
                    const int q = atomicAdd(&s_nfix, 1);
                    if (q < kGreedyMaxFix) s_fix[q] = j;
                }
                const int f = map_s[t];
                if (f >= 0 && w > 0) {
                    const int* off = out ? a.off2i : a.off2o;
                    beg = off[f];
                    len = off[f + 1] - beg;
                    wv = out ? w : (w | (int)0x80000000);
                }
            }
            int pre, total;
            Scan(scan_tmp).ExclusiveSum(len, pre, total);
            s_pre[tid] = pre;
            s_beg[tid] = beg;
            s_w[tid] = wv;
            if (tid == 0) s_pre[kGreedyThreads] = total;
            __syncthreads();
            // kGreedyUnroll items per thread at a time: their list loads are in
            // flight together
            for (long long q0 = gt; q0 < total; q0 += kGreedyUnroll * gthreads) {
                int k[kGreedyUnroll], wl[kGreedyUnroll], g2[kGreedyUnroll], w2[kGreedyUnroll];
#pragma unroll
                for (int u = 0; u < kGreedyUnroll; u++) {
                    const long long q = q0 + u * gthreads;
                    k[u] = -1;
                    wl[u] = 0;
                    if (q < total) {
                        int lo = 0, hi = kGreedyThreads - 1;   // last edge with s_pre <= q
                        while (lo < hi) {
                            const int mid = (lo + hi + 1) >> 1;
                            if (s_pre[mid] <= q) lo = mid; else hi = mid - 1;
                        }
                        k[u] = s_beg[lo] + (int)(q - s_pre[lo]);
                        wl[u] = s_w[lo];
                    }
                }
#pragma unroll
                for (int u = 0; u < kGreedyUnroll; u++) {
                    if (k[u] < 0) continue;
                    const bool out = wl[u] >= 0;
                    g2[u] = out ? a.id2i[k[u]] : a.id2o[k[u]];
                    w2[u] = out ? a.w2i[k[u]] : a.w2o[k[u]];
                }
#pragma unroll
                for (int u = 0; u < kGreedyUnroll; u++) {
                    if (k[u] < 0) continue;
                    const int c = min(wl[u] & 0x7fffffff, w2[u]);
                    if (c > 0) atomicAdd(&acc[g2[u]], c);
                }
            }
            __syncthreads();
        }
        const double4 r1 = a.ratio1[v1];
        // one grid barrier per step: this step's scatter is complete and the
        // previous step's slice bests are published
        if (!grid_barrier(a.bar, a.stall && step == 0)) return;
        if (step + 1 < a.n) {
            nv = a.order1[step + 1];
            no0 = a.off1o[nv]; ndout = a.off1o[nv + 1] - no0;
            ni0 = a.off1i[nv]; ndin = a.off1i[nv + 1] - ni0;
            if (tid < ndout + ndin) {
                nt = tid < ndout ? a.id1o[no0 + tid] : a.id1i[ni0 + tid - ndout];
                nwt = tid < ndout ? a.w1o[no0 + tid] : a.w1i[ni0 + tid - ndout];
            }
        }
        if (step > 0) {
            greedy_decide(a, (step - 1) & 1, prev, map_s, taken, base, len, wbest);
            // the edges of v1 to prev: their terms for this CTA's slice only
            const int nfix = s_nfix;
            const int f = map_s[prev];
            if (nfix > 0 && f >= 0) {
                const int nscan = nfix <= kGreedyMaxFix ? nfix : dout + din;
                for (int q = 0; q < nscan; q++) {
                    const int j = nfix <= kGreedyMaxFix ? s_fix[q] : q;
                    const bool out = j < dout;
                    const int t = out ? a.id1o[o0 + j] : a.id1i[i0 + j - dout];
                    const int w = out ? a.w1o[o0 + j] : a.w1i[i0 + j - dout];
                    if (t != prev || w <= 0) continue;
                    const int* off = out ? a.off2i : a.off2o;
                    const int* lid = out ? a.id2i : a.id2o;
                    const int* lw = out ? a.w2i : a.w2o;
                    for (int k = off[f] + tid; k < off[f + 1]; k += blockDim.x) {
                        const int g = lid[k];
                        if (g < base || g >= base + len) continue;
                        const int c = min(w, lw[k]);
                        if (c > 0) atomicAdd(&acc[g], c);
                    }
                }
            }
            __syncthreads();
        }
        // ---- this CTA's best candidate (and its acc cleared for two steps on) ----
        GreedyBest best{-1.0 / 0.0, 0x7fffffff, -1};
        for (int l = tid; l < len; l += blockDim.x) {
            const int al = __ldcg(&acc[base + l]);
            if (al) acc[base + l] = 0;
            if (taken[l]) continue;
            const GreedyBest c{greedy_score(r1, r2_s[l], al), pos_s[l], base + l};
            if (better(c, best)) best = c;
        }
        for (int o = 16; o; o >>= 1) {
            GreedyBest y;
            y.score = __shfl_xor_sync(0xffffffffu, best.score, o);
            y.pos = __shfl_xor_sync(0xffffffffu, best.pos, o);
            y.g = __shfl_xor_sync(0xffffffffu, best.g, o);
            if (better(y, best)) best = y;
        }
        if (lane == 0) wbest[wid] = best;
        __syncthreads();
        if (tid == 0) {
            for (int w = 1; w < kGreedyThreads / 32; w++)
                if (better(wbest[w], best)) best = wbest[w];
            GreedyBest* dst = a.bests + par * gridDim.x + blockIdx.x;
            __stcg(&dst->score, best.score);
            __stcg(&dst->pos, best.pos);
            __stcg(&dst->g, best.g);
            s_nfix = 0;
        }
        __syncthreads();
        prev = v1;
    }
    // the last step's decision
    if (!grid_barrier(a.bar)) return;
    greedy_decide(a, (a.n - 1) & 1, prev, map_s, taken, a.n, 0, wbest);
}

struct GreedyDev {
    std::vector<void*> bufs;
    ~GreedyDev() { for (void* p : bufs) cudaFree(p); }
    template <class T> cudaError_t alloc(T** p, size_t count) {
        cudaError_t e = cudaMalloc((void**)p, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) bufs.push_back(*p);
        return e;
    }
};

#define GK(call)                                                                      \
    do {                                                                              \
        cudaError_t _e = (call);                                                      \
        if (_e != cudaSuccess) {                                                      \
            set_err(nullptr, "%s: %s (%s:%d)", fn, cudaGetErrorString(_e), __FILE__, __LINE__); \
            return BM_E_CUDA;                                                         \
        }                                                                             \
    } while (0)

// Validates one graph's edges (ids in 1..n, weights >= 0).  The message of a
// failure goes to err (the caller records it: this may run on a helper thread).
bm_status check_edges(const char* fn, int n, long long m, const int32_t* s, const int32_t* d, const int32_t* w,
                      char* err, size_t cap) {
    if (m < 0 || (m > 0 && (!s || !d || !w))) { snprintf(err, cap, "%s: bad edge arrays", fn); return BM_E_INPUT; }
    if (m > 0x7fffffffLL) { snprintf(err, cap, "%s: %lld edges (at most 2^31-1)", fn, m); return BM_E_INPUT; }
    for (long long i = 0; i < m; i++) {
        if (s[i] < 1 || s[i] > n || d[i] < 1 || d[i] > n) {
            snprintf(err, cap, "%s: edge %lld (%d,%d) outside 1..%d", fn, i, s[i], d[i], n);
            return BM_E_INPUT;
        }
        if (w[i] < 0) { snprintf(err, cap, "%s: edge %lld has negative weight %d", fn, i, w[i]); return BM_E_INPUT; }
    }
    return BM_OK;
}

// ---- adjacency lists built on the device ----
__global__ void k_to_zero_based(int* __restrict__ s, int* __restrict__ d, long long m) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        s[i] -= 1;
        d[i] -= 1;
    }
}
__global__ void k_key_hist(const int* __restrict__ key, long long m, int* __restrict__ cnt) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        atomicAdd(&cnt[key[i] + 1], 1);
}
// Entry i goes to the next free slot of its row (order within a row: arrival).
__global__ void k_csr_scatter(const int* __restrict__ key, const int* __restrict__ other, const int* __restrict__ w,
                              long long m, int* __restrict__ cur, int* __restrict__ id, int* __restrict__ ww) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        const int p = atomicAdd(&cur[key[i]], 1);
        id[p] = other[i];
        if (ww) ww[p] = w[i];
    }
}
__global__ void k_pair_keys(const int* __restrict__ s, const int* __restrict__ d, long long m, int n,
                            unsigned long long* __restrict__ key, int* __restrict__ idx) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        key[i] = (unsigned long long)s[i] * (unsigned long long)n + (unsigned long long)d[i];
        idx[i] = (int)i;
    }
}
// 1 for the last entry of each run of equal (sorted) keys.
__global__ void k_last_of_run(const unsigned long long* __restrict__ key, long long m, char* __restrict__ flag) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x)
        flag[i] = (i + 1 == m || key[i] != key[i + 1]) ? 1 : 0;
}
__global__ void k_gather3(const int* __restrict__ sel, long long m, const int* __restrict__ s, const int* __restrict__ d,
                          const int* __restrict__ w, int* __restrict__ s2, int* __restrict__ d2, int* __restrict__ w2) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        const int j = sel[i];
        s2[i] = s[j]; d2[i] = d[j]; w2[i] = w[j];
    }
}

struct DevLists { int *off = nullptr, *id = nullptr, *w = nullptr; };

// Lists keyed by key[] (0-based): off (n+1), id and, with w, weights.
bm_status dev_csr(const char* fn, GreedyDev& D, int n, long long m, const int* key, const int* other, const int* w,
                  DevLists& L, cudaStream_t st, int blocks) {
    int *cnt, *cur;
    GK(D.alloc(&L.off, (size_t)n + 1)); GK(D.alloc(&cnt, (size_t)n + 1)); GK(D.alloc(&cur, (size_t)n));
    GK(D.alloc(&L.id, (size_t)m));
    if (w) GK(D.alloc(&L.w, (size_t)m));
    GK(cudaMemsetAsync(cnt, 0, ((size_t)n + 1) * sizeof(int), st));
    if (m) k_key_hist<<<blocks, 256, 0, st>>>(key, m, cnt);
    size_t tb = 0;
    GK(cub::DeviceScan::InclusiveSum(nullptr, tb, cnt, L.off, n + 1, st));
    char* tmp;
    GK(D.alloc(&tmp, tb));
    GK(cub::DeviceScan::InclusiveSum(tmp, tb, cnt, L.off, n + 1, st));
    GK(cudaMemcpyAsync(cur, L.off, (size_t)n * sizeof(int), cudaMemcpyDeviceToDevice, st));
    if (m) k_csr_scatter<<<blocks, 256, 0, st>>>(key, other, w, m, cur, L.id, w ? L.w : nullptr);
    GK(cudaGetLastError());
    return BM_OK;
}

// One entry per (src, dst) of a graph, the last weight given (a stable sort
// keeps the input order among equal pairs): s, d, w of the kept entries.
bm_status dev_dedup(const char* fn, GreedyDev& D, int n, long long m, const int* s, const int* d, const int* w,
                    int** ks, int** kd, int** kw, long long* mk, cudaStream_t st, int blocks) {
    unsigned long long *key, *key2;
    int *idx, *perm, *sel, *nsel;
    char* flag;
    GK(D.alloc(&key, (size_t)m)); GK(D.alloc(&key2, (size_t)m)); GK(D.alloc(&idx, (size_t)m));
    GK(D.alloc(&perm, (size_t)m)); GK(D.alloc(&sel, (size_t)m)); GK(D.alloc(&nsel, 1)); GK(D.alloc(&flag, (size_t)m));
    int bits = 1;
    while (bits < 64 && ((unsigned long long)n * (unsigned long long)n) >> bits) bits++;
    if (m) {
        k_pair_keys<<<blocks, 256, 0, st>>>(s, d, m, n, key, idx);
        size_t tb = 0;
        GK(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, idx, perm, (int)m, 0, bits, st));
        char* tmp;
        GK(D.alloc(&tmp, tb));
        GK(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, idx, perm, (int)m, 0, bits, st));
        k_last_of_run<<<blocks, 256, 0, st>>>(key2, m, flag);
        tb = 0;
        GK(cub::DeviceSelect::Flagged(nullptr, tb, perm, flag, sel, nsel, (int)m, st));
        char* tmp2;
        GK(D.alloc(&tmp2, tb));
        GK(cub::DeviceSelect::Flagged(tmp2, tb, perm, flag, sel, nsel, (int)m, st));
        GK(cudaGetLastError());
    } else {
        GK(cudaMemsetAsync(nsel, 0, sizeof(int), st));
    }
    int h = 0;
    GK(cudaMemcpyAsync(&h, nsel, sizeof(int), cudaMemcpyDeviceToHost, st));
    GK(cudaStreamSynchronize(st));
    *mk = h;
    GK(D.alloc(ks, (size_t)h)); GK(D.alloc(kd, (size_t)h)); GK(D.alloc(kw, (size_t)h));
    if (h) k_gather3<<<blocks, 256, 0, st>>>(sel, h, s, d, w, *ks, *kd, *kw);
    GK(cudaGetLastError());
    return BM_OK;
}

// The three raw edge arrays of a graph, 0-based, on the device.
bm_status dev_edges(const char* fn, GreedyDev& D, long long m, const int32_t* s, const int32_t* d, const int32_t* w,
                    int** ds, int** dd, int** dw, cudaStream_t st, int blocks) {
    GK(D.alloc(ds, (size_t)m)); GK(D.alloc(dd, (size_t)m)); GK(D.alloc(dw, (size_t)m));
    if (m) {
        GK(cudaMemcpyAsync(*ds, s, (size_t)m * sizeof(int), cudaMemcpyHostToDevice, st));
        GK(cudaMemcpyAsync(*dd, d, (size_t)m * sizeof(int), cudaMemcpyHostToDevice, st));
        GK(cudaMemcpyAsync(*dw, w, (size_t)m * sizeof(int), cudaMemcpyHostToDevice, st));
        k_to_zero_based<<<blocks, 256, 0, st>>>(*ds, *dd, m);
        GK(cudaGetLastError());
    }
    return BM_OK;
}

// Features of one graph on the device: feat (int4), ratio (double4), and the
// feature order (order[i] = vertex at place i).
bm_status device_features(const char* fn, GreedyDev& D, int n, const DevLists& lo, const DevLists& li,
                          int4* feat, double4* ratio, int* order, cudaStream_t st, int sms) {
    int *r2, *c2, *val, *val2;
    unsigned long long *key, *key2;
    GK(D.alloc(&r2, n)); GK(D.alloc(&c2, n));
    GK(D.alloc(&key, n)); GK(D.alloc(&key2, n)); GK(D.alloc(&val, n)); GK(D.alloc(&val2, n));
    const size_t bm = (size_t)((n + 31) / 32) * sizeof(unsigned);
    GK(cudaFuncSetAttribute(k_two_hop, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bm));
    k_two_hop<<<sms * 4, 512, bm, st>>>(lo.off, lo.id, n, r2);
    k_two_hop<<<sms * 4, 512, bm, st>>>(li.off, li.id, n, c2);
    k_features<<<(n + 255) / 256, 256, 0, st>>>(lo.off, li.off, r2, c2, n, feat, ratio, key, val);
    GK(cudaGetLastError());
    size_t tb = 0;
    GK(cub::DeviceRadixSort::SortPairs(nullptr, tb, key, key2, val, val2, n, 0, 64, st));
    void* tmp;
    GK(D.alloc((char**)&tmp, tb));
    GK(cub::DeviceRadixSort::SortPairs(tmp, tb, key, key2, val, order, n, 0, 64, st));
    return BM_OK;
}

}  // namespace
}  // namespace bm

using namespace bm;

extern "C" bm_status bm_greedy_features(int32_t n, int64_t e, const int32_t* src, const int32_t* dst,
                                        const int32_t* w, int32_t* out) {
    const char* fn = "bm_greedy_features";
    if (n < 1 || !out) { set_err(nullptr, "%s: bad arguments", fn); return BM_E_INPUT; }
    char err[256];
    bm_status s = check_edges(fn, n, e, src, dst, w, err, sizeof err);
    if (s) { set_err(nullptr, "%s", err); return s; }
    int dev = 0, sms = 0;
    GK(cudaGetDevice(&dev));
    GK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int blocks = sms * 8;
    GreedyDev D;
    int *ds, *dd, *dw;
    s = dev_edges(fn, D, e, src, dst, w, &ds, &dd, &dw, 0, blocks);
    DevLists lo, li;
    if (!s) s = dev_csr(fn, D, n, e, ds, dd, nullptr, lo, 0, blocks);
    if (!s) s = dev_csr(fn, D, n, e, dd, ds, nullptr, li, 0, blocks);
    int4* feat; double4* ratio; int* order;
    if (!s) {
        GK(D.alloc(&feat, n)); GK(D.alloc(&ratio, n)); GK(D.alloc(&order, n));
        s = device_features(fn, D, n, lo, li, feat, ratio, order, 0, sms);
    }
    if (s) return s;
    GK(cudaMemcpy(out, feat, (size_t)n * sizeof(int4), cudaMemcpyDeviceToHost));
    return BM_OK;
}

extern "C" bm_status bm_greedy_match(int32_t n, int64_t e1, const int32_t* src1, const int32_t* dst1,
                                     const int32_t* w1, int64_t e2, const int32_t* src2, const int32_t* dst2,
                                     const int32_t* w2, int32_t* map, bm_greedy_stats* stats) {
    const char* fn = "bm_greedy_match";
    if (n < 1 || !map) { set_err(nullptr, "%s: bad arguments", fn); return BM_E_INPUT; }
    bm_status s = BM_OK, s_2 = BM_OK;
    char err1[256], err2[256];
    {   // the two graphs are checked on two host threads
        std::thread t([&] { s_2 = check_edges(fn, n, e2, src2, dst2, w2, err2, sizeof err2); });
        s = check_edges(fn, n, e1, src1, dst1, w1, err1, sizeof err1);
        t.join();
    }
    if (s) { set_err(nullptr, "%s", err1); return s; }
    if (s_2) { set_err(nullptr, "%s", err2); return s_2; }
    int dev = 0, sms = 0, optin = 0;
    GK(cudaGetDevice(&dev));
    GK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    GK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    int per_sm = 0;
    const int slice0 = (n + sms - 1) / sms;
    size_t smem = (size_t)slice0 * sizeof(double4) + (size_t)n * 4 + (size_t)slice0 * 5 + 16;
    if (smem + 4096 > (size_t)optin) {
        set_err(nullptr, "%s: n=%d needs %zu bytes of shared memory per CTA (limit %d)", fn, n, smem, optin);
        return BM_E_INPUT;
    }
    GK(cudaFuncSetAttribute(k_greedy, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    GK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_greedy, kGreedyThreads, smem));
    if (per_sm < 1) { set_err(nullptr, "%s: the matching kernel does not fit on an SM", fn); return BM_E_INPUT; }
    const int grid = sms;
    cudaStream_t st;
    GK(cudaStreamCreate(&st));
    struct StreamGuard { cudaStream_t s; ~StreamGuard() { cudaStreamSynchronize(s); cudaStreamDestroy(s); } } sg{st};
    cudaEvent_t ev[3];
    for (auto& e : ev) GK(cudaEventCreate(&e));
    struct EvGuard { cudaEvent_t* e; ~EvGuard() { for (int i = 0; i < 3; i++) cudaEventDestroy(e[i]); } } eg{ev};
    GreedyDev D;
    int4 *feat1, *feat2;
    double4 *ratio1, *ratio2;
    int *order1, *order2, *pos2, *mapd, *acc;
    GreedyBest* bests;
    unsigned* bar;
    GK(D.alloc(&feat1, n)); GK(D.alloc(&feat2, n)); GK(D.alloc(&ratio1, n)); GK(D.alloc(&ratio2, n));
    GK(D.alloc(&order1, n)); GK(D.alloc(&order2, n)); GK(D.alloc(&pos2, n)); GK(D.alloc(&mapd, n));
    GK(D.alloc(&acc, 2 * (size_t)n)); GK(D.alloc(&bests, 2 * (size_t)grid)); GK(D.alloc(&bar, 4));
    GK(cudaMemsetAsync(acc, 0, 2 * (size_t)n * sizeof(int), st));
    GK(cudaMemsetAsync(bar, 0, 4 * sizeof(unsigned), st));
    GreedyArgs A;
    A.n = n; A.slice = slice0;
    const int blocks = sms * 8;
    int *s1d, *d1d, *w1d, *s2d, *d2d, *w2d, *ks, *kd, *kw;
    long long mk = 0;
    DevLists g1o, g1i, g2o, g2i, g2od, g2id;
    s = dev_edges(fn, D, e1, src1, dst1, w1, &s1d, &d1d, &w1d, st, blocks);
    if (!s) s = dev_edges(fn, D, e2, src2, dst2, w2, &s2d, &d2d, &w2d, st, blocks);
    if (s) return s;
    GK(cudaEventRecord(ev[0], st));   // device time from here: lists, features, matching
    if (!s) s = dev_csr(fn, D, n, e1, s1d, d1d, w1d, g1o, st, blocks);
    if (!s) s = dev_csr(fn, D, n, e1, d1d, s1d, w1d, g1i, st, blocks);
    if (!s) s = dev_csr(fn, D, n, e2, s2d, d2d, nullptr, g2o, st, blocks);
    if (!s) s = dev_csr(fn, D, n, e2, d2d, s2d, nullptr, g2i, st, blocks);
    if (!s) s = dev_dedup(fn, D, n, e2, s2d, d2d, w2d, &ks, &kd, &kw, &mk, st, blocks);
    if (!s) s = dev_csr(fn, D, n, mk, ks, kd, kw, g2od, st, blocks);
    if (!s) s = dev_csr(fn, D, n, mk, kd, ks, kw, g2id, st, blocks);
    if (s) return s;
    A.off1o = g1o.off; A.id1o = g1o.id; A.w1o = g1o.w;
    A.off1i = g1i.off; A.id1i = g1i.id; A.w1i = g1i.w;
    A.off2o = g2od.off; A.id2o = g2od.id; A.w2o = g2od.w;
    A.off2i = g2id.off; A.id2i = g2id.id; A.w2i = g2id.w;
    s = device_features(fn, D, n, g1o, g1i, feat1, ratio1, order1, st, sms);
    if (!s) s = device_features(fn, D, n, g2o, g2i, feat2, ratio2, order2, st, sms);
    if (s) return s;
    k_positions<<<(n + 255) / 256, 256, 0, st>>>(order2, n, pos2);
    GK(cudaGetLastError());
    GK(cudaEventRecord(ev[1], st));
    A.order1 = order1; A.pos2 = pos2; A.ratio1 = ratio1; A.ratio2 = ratio2;
    A.acc = acc; A.bests = bests; A.bar = bar; A.map = mapd;
    A.stall = take_stall(BM_STALL_GREEDY);
    void* kargs[] = {&A};
    GK(cudaLaunchCooperativeKernel((const void*)k_greedy, dim3(grid), dim3(kGreedyThreads), kargs, smem, st));
    GK(cudaEventRecord(ev[2], st));
    unsigned herr[4] = {0, 0, 0, 0};
    GK(cudaMemcpyAsync(herr, bar, sizeof herr, cudaMemcpyDeviceToHost, st));
    std::vector<int> h(n);
    GK(cudaMemcpyAsync(h.data(), mapd, (size_t)n * sizeof(int), cudaMemcpyDeviceToHost, st));
    GK(cudaStreamSynchronize(st));
    if (herr[2]) { set_err(nullptr, "%s: grid barrier wait timed out", fn); return BM_E_TIMEOUT; }
    map[0] = 0;
    for (int v = 0; v < n; v++) map[v + 1] = h[v] + 1;
    if (stats) {
        memset(stats, 0, sizeof *stats);
        cudaEventElapsedTime(&stats->ms_features, ev[0], ev[1]);
        cudaEventElapsedTime(&stats->ms_match, ev[1], ev[2]);
    }
    return BM_OK;
}
