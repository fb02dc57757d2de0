// bm_incr.cuh -- keeping the profit matrix S exact across commits.
//
// S[a][b] = T[a][p b] + C[a][b]: T[a][f] is the score a would earn on G2
// vertex f with its neighbours where they are (it depends on p only through
// a's G1 neighbours), C[a][b] is the corner correction of a G1 edge a->b (it
// depends on p(a) and p(b)).  When a set M of vertices changes image, from pS
// (the matching S was exact for) to p:
//   1. the corner entries of every G1 edge with an endpoint in M are removed
//      (computed on pS);
//   2. the columns of M are permuted: the new S[a][b] holds T[a][p b], which
//      sat in the old column of the vertex that held p(b) under pS;
//   3. each G1 edge u->m (m in M) changes u's out-term min(w, W2[f][p m]) for
//      every f, nonzero only on G2's in-list of the old and the new image of
//      m: its entries are subtracted and added in row u; edges m->v likewise
//      in row v through G2's out-lists;
//   4. the corner entries are added back, computed on p.
// Every step is an integer sum of exact terms, so the result equals a rebuild
// bit for bit whatever the order of the atomics.  The reference keeps its
// lookup table (src/best-swap/score-lookup.c:514-537) by recomputing only the
// rows and columns of the two swapped vertices, which leaves every pair next
// to them stale; steps 1-4 are the complete set of changes.
#pragma once
#include "bm_kernels.cuh"

namespace bm {

constexpr int kIncrMaxMoved = 12288;   // moved vertices one update handles (column buffer in shared memory)
constexpr int kIncrEdgesPerBlock = 32; // G1 edges of one moved vertex per block in the term update
constexpr int kIncrCornerEdges = 128;  // G1 edges per block in the corner passes
// Cost model of an update against a rebuild, in units of one shared-memory
// min term of the rebuild (~1.4 ps on a B200): an atomic into S (~27 ps: a
// DRAM read-modify-write of a sector of a 1.4 GB matrix), and one permuted
// column entry.
constexpr double kIncrAtomicCost = 20.0;
constexpr double kIncrPermCost = 16.0;
// A G1 edge whose two G2 lists together hold at least n/4 entries changes a
// quarter of its row: its terms are summed in shared memory first and the row
// written once with coalesced atomics (about n/8 sectors, ~3 units per column)
// instead of one scattered atomic per entry.
constexpr double kIncrRowCost = 3.0;
constexpr int kIncrRowThreads = 512;

// Whether the edges of moved vertex m in one direction take the row path:
// the two lists (old image, new image) hold >= n/4 entries together.
__device__ __forceinline__ bool incr_heavy(const int* off, int fo, int fn, int n) {
    return 4LL * ((off[fo + 1] - off[fo]) + (off[fn + 1] - off[fn])) >= (long long)n;
}

// Moved vertices (p != pS), compacted into moved[], with info[0] = count,
// info[1] = 1 when a vertex took a G2 vertex that nobody held under pS (its T
// column was never built: only a rebuild has it), info[2] = largest G1 degree
// (in + out) among them, work[0] = the list entries step 3 applies by single
// atomics, work[1] = the rows it writes whole (incr_heavy), work[2] = all list
// entries of step 3.
template <bool W16>
__global__ void k_moved(DevView<W16> g, const int* __restrict__ pS, const int* __restrict__ pinvS,
                        int* __restrict__ moved, int* __restrict__ info, unsigned long long* __restrict__ work) {
    const int n = g.n;
    const int lane = threadIdx.x & 31;
    for (int base = blockIdx.x * blockDim.x; base < n; base += gridDim.x * blockDim.x) {
        const int v = base + threadIdx.x;
        bool mv = false;
        unsigned long long w = 0, rows = 0, all = 0;
        int deg = 0;
        if (v < n) {
            const int fo = pS[v], fn = g.p[v];
            if (fo != fn) {
                mv = true;
                if (fn != n && pinvS[fn] == n) info[1] = 1;
                const int di = g.off1i[v + 1] - g.off1i[v], dout = g.off1o[v + 1] - g.off1o[v];
                const unsigned long long ei = (unsigned long long)di *
                    (unsigned long long)((g.off2i[fo + 1] - g.off2i[fo]) + (g.off2i[fn + 1] - g.off2i[fn]));
                const unsigned long long eo = (unsigned long long)dout *
                    (unsigned long long)((g.off2o[fo + 1] - g.off2o[fo]) + (g.off2o[fn + 1] - g.off2o[fn]));
                const bool hi = incr_heavy(g.off2i, fo, fn, n), ho = incr_heavy(g.off2o, fo, fn, n);
                w = (hi ? 0ull : ei) + (ho ? 0ull : eo);
                rows = (hi ? (unsigned long long)di : 0ull) + (ho ? (unsigned long long)dout : 0ull);
                all = ei + eo;
                deg = di + dout;
            }
        }
        const unsigned bal = __ballot_sync(0xffffffffu, mv);
        if (!bal) continue;
        const int leader = __ffs(bal) - 1;
        int slot = 0;
        if (lane == leader) slot = atomicAdd(&info[0], __popc(bal));
        slot = __shfl_sync(0xffffffffu, slot, leader);
        if (mv) moved[slot + __popc(bal & ((1u << lane) - 1u))] = v;
        for (int o = 16; o; o >>= 1) {
            w += __shfl_xor_sync(0xffffffffu, w, o);
            rows += __shfl_xor_sync(0xffffffffu, rows, o);
            all += __shfl_xor_sync(0xffffffffu, all, o);
            deg = max(deg, __shfl_xor_sync(0xffffffffu, deg, o));
        }
        if (lane == 0) {
            atomicAdd(&work[0], w);
            atomicAdd(&work[1], rows);
            atomicAdd(&work[2], all);
            atomicMax(&info[2], deg);
        }
    }
}

__device__ __forceinline__ int corner_term(int x, int w_ab, int w_ba, int w_aa, int w_bb) {
    return imin(x, w_ab) + imin(x, w_ba) - imin(x, w_aa) - imin(x, w_bb);
}

// Steps 1 and 4: sign * the corner correction of every G1 edge with an
// endpoint in moved[0..count), on the matching pm (pS for removal, p for the
// addition).  An edge between two moved vertices is taken from its source's
// out-list only.  grid = (count, ceil(max degree / kIncrCornerEdges)); with
// dcount, only the first *dcount moved vertices (the same in every kernel).
template <bool W16>
__global__ void k_corner(DevView<W16> g, const int* __restrict__ pm, const int* __restrict__ pS,
                         const int* __restrict__ moved, int count, const int* __restrict__ dcount, int sign) {
    typedef Ent<W16> EN;
    if (dcount) count = min(count, *dcount);
    if ((int)blockIdx.x >= count) return;
    const int n = g.n;
    const int m = moved[blockIdx.x];
    const int so = g.off1o[m], lo = g.off1o[m + 1] - so;
    const int si = g.off1i[m], li = g.off1i[m + 1] - si;
    const int j = blockIdx.y * kIncrCornerEdges + threadIdx.x;
    if (threadIdx.x >= kIncrCornerEdges || j >= lo + li) return;
    int a, b, x;
    if (j < lo) {
        const typename EN::T e = g.ent1o[so + j];
        a = m; b = EN::id(e); x = EN::w(e);
    } else {
        const typename EN::T e = g.ent1i[si + (j - lo)];
        a = EN::id(e); b = m; x = EN::w(e);
        if (pS[a] != g.p[a]) return;  // the source moved too: done from its out-list
    }
    const int pa = pm[a], pb = pm[b];
    const int c = corner_term(x, g.w2(pa, pb), g.w2t(pb, pa), g.w2d(pa), g.w2d(pb));
    if (c) atomicAdd(&g.S[(size_t)a * n + b], sign * c);
}

// Step 2: for every row, new S[a][b] = old S[a][pinvS[p b]] for b in moved
// (0 when b is unmatched: T[a][NONE] = 0).  One row per block iteration.
__global__ void k_perm_cols(int* __restrict__ S, int n, const int* __restrict__ moved, int count,
                            const int* __restrict__ p, const int* __restrict__ pinvS) {
    extern __shared__ int sh[];
    int* dst = sh;            // moved columns
    int* src = sh + count;    // where their new values sit (-1: zero)
    int* buf = sh + 2 * count;
    for (int j = threadIdx.x; j < count; j += blockDim.x) {
        const int b = moved[j];
        const int f = p[b];
        dst[j] = b;
        src[j] = f == n ? -1 : pinvS[f];
    }
    __syncthreads();
    for (int a = blockIdx.x; a < n; a += gridDim.x) {
        int* row = S + (size_t)a * n;
        for (int j = threadIdx.x; j < count; j += blockDim.x) buf[j] = src[j] < 0 ? 0 : row[src[j]];
        __syncthreads();
        for (int j = threadIdx.x; j < count; j += blockDim.x) row[dst[j]] = buf[j];
        __syncthreads();
    }
}

// Step 3: the T terms of every G1 edge at a moved vertex, old image out, new
// image in.  grid = (count, ceil(max degree / kIncrEdgesPerBlock)), 256
// threads: each warp takes an edge and its lanes walk the two G2 lists.
template <bool W16>
__global__ void __launch_bounds__(256) k_terms(DevView<W16> g, const int* __restrict__ pS,
                                               const int* __restrict__ moved, int count,
                                               const int* __restrict__ dcount) {
    typedef Ent<W16> EN;
    typedef typename EN::T E;
    if (dcount) count = min(count, *dcount);
    if ((int)blockIdx.x >= count) return;
    const int n = g.n;
    const int m = moved[blockIdx.x];
    const int fo = pS[m], fn = g.p[m];
    const int so = g.off1o[m], lo = g.off1o[m + 1] - so;
    const int si = g.off1i[m], li = g.off1i[m + 1] - si;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const bool hi = incr_heavy(g.off2i, fo, fn, n), ho = incr_heavy(g.off2o, fo, fn, n);
    for (int t = wid; t < kIncrEdgesPerBlock; t += 8) {
        const int j = blockIdx.y * kIncrEdgesPerBlock + t;
        if (j >= lo + li) break;
        if (j < li ? hi : ho) continue;  // k_terms_rows takes it
        int row, w1;
        const int* off;
        const E* list;
        if (j < li) {  // in-edge u->m: u's out-term, G2 in-lists of m's images
            const E e = g.ent1i[si + j];
            row = EN::id(e); w1 = EN::w(e);
            off = g.off2i; list = g.ent2i;
        } else {       // out-edge m->v: v's in-term, G2 out-lists of m's images
            const E e = g.ent1o[so + (j - li)];
            row = EN::id(e); w1 = EN::w(e);
            off = g.off2o; list = g.ent2o;
        }
        int* srow = g.S + (size_t)row * n;
        for (int k = off[fo] + lane; k < off[fo + 1]; k += 32) {
            const E e = list[k];
            const int col = g.pinv[EN::id(e)];
            if (col < n) atomicAdd(&srow[col], -imin(w1, EN::w(e)));
        }
        for (int k = off[fn] + lane; k < off[fn + 1]; k += 32) {
            const E e = list[k];
            const int col = g.pinv[EN::id(e)];
            if (col < n) atomicAdd(&srow[col], imin(w1, EN::w(e)));
        }
    }
}

// Step 3 for the edges whose lists cover much of their row (incr_heavy): a
// block per edge sums its terms in a shared-memory row, then adds the nonzero
// entries to S in column order.  grid = (count, up to 256 edge slots per
// moved vertex), dynamic shared memory (n+1) ints.
template <bool W16>
__global__ void __launch_bounds__(kIncrRowThreads) k_terms_rows(DevView<W16> g, const int* __restrict__ pS,
                                                               const int* __restrict__ moved, int count,
                                                               const int* __restrict__ dcount) {
    typedef Ent<W16> EN;
    typedef typename EN::T E;
    extern __shared__ int rowbuf[];
    if (dcount) count = min(count, *dcount);
    if ((int)blockIdx.x >= count) return;
    const int n = g.n;
    const int m = moved[blockIdx.x];
    const int fo = pS[m], fn = g.p[m];
    const bool hi = incr_heavy(g.off2i, fo, fn, n), ho = incr_heavy(g.off2o, fo, fn, n);
    if (!hi && !ho) return;
    const int so = g.off1o[m], lo = g.off1o[m + 1] - so;
    const int si = g.off1i[m], li = g.off1i[m + 1] - si;
    const int j0 = hi ? 0 : li, j1 = ho ? li + lo : li;
    if (j0 + (int)blockIdx.y >= j1) return;
    for (int c = threadIdx.x; c <= n; c += blockDim.x) rowbuf[c] = 0;
    for (int j = j0 + blockIdx.y; j < j1; j += gridDim.y) {
        int row, w1;
        const int* off;
        const E* list;
        if (j < li) {
            const E e = g.ent1i[si + j];
            row = EN::id(e); w1 = EN::w(e);
            off = g.off2i; list = g.ent2i;
        } else {
            const E e = g.ent1o[so + (j - li)];
            row = EN::id(e); w1 = EN::w(e);
            off = g.off2o; list = g.ent2o;
        }
        __syncthreads();
        for (int k = off[fo] + threadIdx.x; k < off[fo + 1]; k += blockDim.x) {
            const E e = list[k];
            atomicAdd(&rowbuf[g.pinv[EN::id(e)]], -imin(w1, EN::w(e)));   // column n: unmatched, dropped
        }
        for (int k = off[fn] + threadIdx.x; k < off[fn + 1]; k += blockDim.x) {
            const E e = list[k];
            atomicAdd(&rowbuf[g.pinv[EN::id(e)]], imin(w1, EN::w(e)));
        }
        __syncthreads();
        int* srow = g.S + (size_t)row * n;
        for (int c = threadIdx.x; c < n; c += blockDim.x) {
            const int v = rowbuf[c];
            if (v) { atomicAdd(&srow[c], v); rowbuf[c] = 0; }
        }
        if (threadIdx.x == 0) rowbuf[n] = 0;
    }
}

}  // namespace bm

namespace bm {

constexpr int kSmallMoved = 4;    // moved vertices of the thread-per-row column permutation
constexpr int kLookupBatch = 32;  // best-swap steps enqueued between host checks

// Step 2 for at most kSmallMoved moved vertices (*dcount of them): one thread per row.
__global__ void k_perm_cols_small(int* __restrict__ S, int n, const int* __restrict__ moved,
                                  const int* __restrict__ dcount, const int* __restrict__ p,
                                  const int* __restrict__ pinvS) {
    const int count = min(*dcount, kSmallMoved);
    if (count == 0) return;
    int dst[kSmallMoved], src[kSmallMoved], val[kSmallMoved];
#pragma unroll
    for (int j = 0; j < kSmallMoved; j++) {
        dst[j] = 0; src[j] = -1; val[j] = 0;
        if (j < count) {
            dst[j] = moved[j];
            const int f = p[dst[j]];
            src[j] = f == n ? -1 : pinvS[f];
        }
    }
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < n; a += gridDim.x * blockDim.x) {
        int* row = S + (size_t)a * n;
#pragma unroll
        for (int j = 0; j < kSmallMoved; j++)
            if (j < count) val[j] = src[j] < 0 ? 0 : row[src[j]];
#pragma unroll
        for (int j = 0; j < kSmallMoved; j++)
            if (j < count) row[dst[j]] = val[j];
    }
}

// Best swap over all pairs from the per-row bests: largest delta, then the
// smallest a, then the smallest b (the first in lexicographic pair order).
// When it improves (> 0) and the descent has not converged, it is committed:
// p and pinv swapped, moved[0..1] = (a, b), info[0] = 2, acc[0] += delta,
// acc[1] += 1; otherwise info[0] = 0 and info[3] = 1.  One block.
__global__ void __launch_bounds__(1024) k_pick_commit(const unsigned long long* __restrict__ rowbest, int n,
                                                      int* __restrict__ p, int* __restrict__ pinv,
                                                      int* __restrict__ moved, int* __restrict__ info,
                                                      long long* __restrict__ acc) {
    __shared__ unsigned long long red[32];
    unsigned long long best = 0;
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        const unsigned long long k = rowbest[a];
        if (!k) continue;
        const unsigned long long key = (k & 0xffffffff00000000ull) | (unsigned)(~a);
        best = key > best ? key : best;
    }
    for (int o = 16; o; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
        best = x > best ? x : best;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x >= 32) return;
    best = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
    for (int o = 16; o; o >>= 1) {
        const unsigned long long x = __shfl_xor_sync(0xffffffffu, best, o);
        best = x > best ? x : best;
    }
    if (threadIdx.x) return;
    info[0] = 0;
    if (info[3] || !best) { info[3] = 1; return; }
    const int d = (int)((unsigned)(best >> 32) - 0x80000000u);
    const int a = (int)(~(unsigned)(best & 0xffffffffu));
    const int b = (int)(~(unsigned)(rowbest[a] & 0xffffffffu));
    if (d <= 0) { info[3] = 1; return; }
    const int fa = p[a], fb = p[b];
    p[a] = fb; p[b] = fa;
    if (fb != n) pinv[fb] = a;
    if (fa != n) pinv[fa] = b;
    moved[0] = a; moved[1] = b;
    info[0] = 2;
    acc[0] += d;
    acc[1] += 1;
}

// pS / pinvS follow p for the first *dcount moved vertices.
__global__ void k_sync_exact(const int* __restrict__ moved, const int* __restrict__ dcount, const int* __restrict__ p,
                             int* __restrict__ pS, int* __restrict__ pinvS, int n) {
    const int j = threadIdx.x;
    if (j >= *dcount) return;
    const int m = moved[j];
    pS[m] = p[m];
    if (p[m] != n) pinvS[p[m]] = m;
}

// Delta rows of the exact table: out[r*n + b] = delta(a0 + r, b), 0 on the
// diagonal.
__global__ void k_delta_rows(const int* __restrict__ S, int n, int a0, int rows, int* __restrict__ out) {
    const long long total = (long long)rows * n;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int a = a0 + (int)(i / n), b = (int)(i % n);
        out[i] = a == b ? 0
                        : S[(size_t)a * n + b] + S[(size_t)b * n + a] - S[(size_t)a * n + a] - S[(size_t)b * n + b];
    }
}

}  // namespace bm
