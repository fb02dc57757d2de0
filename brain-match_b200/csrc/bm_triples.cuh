// bm_triples.cuh -- 3-cycle moves and the reference-order (first-improvement)
// row scan.
//
// A 3-cycle on G1 vertices (a,b,c) moves their images around: rotation 0 is
// permutation 3 of calculateThreeNodeSwapKernel, (f1,f2,f3) <- (f2,f3,f1);
// rotation 1 is permutation 4, (f1,f2,f3) <- (f3,f1,f2) (src/triple.cu:85-92,
// applied by apply_permutation src/triple.cu:903-934).  sigma(x) names the
// vertex whose image x takes: rotation 0: a<-b, b<-c, c<-a; rotation 1:
// a<-c, b<-a, c<-b.
//
// Exact delta from the profit matrix S of the current matching:
//   delta = sum_x S'[x][sigma x] - sum_x S[x][x]
//         + sum over G1 edges (x,y,w) with x,y in {a,b,c}, x != y of
//             min(w,W2[p'x][p'y]) - min(w,W2[p'x][p y]) - min(w,W2[p x][p'y]) + min(w,W2[p x][p y])
// where p'x = p(sigma x) and S'[x][y] is S[x][y] without the swap corner
// corrections folded in for edges x->y.  The edge-walk form used for
// verification sums, over every G1 edge incident to {a,b,c} counted once,
// min(w,W2[p'x][p'y]) - min(w,W2[p x][p y]); it equals the difference of the
// reference's local scores calculate_permutation_delta
// (src/permutation.c:623-696) before and after the move.
#pragma once
#include "bm_kernels.cuh"

namespace bm {

__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
    unsigned long long z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Undirected G1 neighbour k of x: out-list entries first, then in-list.
template <bool W16>
__device__ __forceinline__ int nbr_at(const DevView<W16>& g, int x, int k) {
    typedef Ent<W16> EN;
    const int lo = g.off1o[x + 1] - g.off1o[x];
    return k < lo ? EN::id(g.ent1o[g.off1o[x] + k]) : EN::id(g.ent1i[g.off1i[x] + (k - lo)]);
}
template <bool W16>
__device__ __forceinline__ int ndeg(const DevView<W16>& g, int x) {
    return (g.off1o[x + 1] - g.off1o[x]) + (g.off1i[x + 1] - g.off1i[x]);
}

// The 2-hop sample of slot j of vertex a: a -> b -> c along undirected G1
// edges, b = nbr(a)[h1 mod deg a], c = nbr(b)[h2 mod deg b] with
// h1 = mix64(seed ^ (a << 32 | j)), h2 = mix64(h1).  Returns false when the
// sample is degenerate (isolated vertex, or c in {a,b}).
template <bool W16>
__device__ __forceinline__ bool sample_triple(const DevView<W16>& g, unsigned long long seed, int a,
                                              int j, int& b, int& c) {
    const int da = ndeg(g, a);
    if (da == 0) return false;
    const unsigned long long h1 = mix64(seed ^ (((unsigned long long)a << 32) | (unsigned)j));
    b = nbr_at(g, a, (int)(h1 % (unsigned long long)da));
    const int db = ndeg(g, b);
    if (db == 0) return false;
    const unsigned long long h2 = mix64(h1);
    c = nbr_at(g, b, (int)(h2 % (unsigned long long)db));
    return c != a && c != b;
}

// First index in out1(x) whose id is >= y (rows are sorted by id).
template <bool W16>
__device__ __forceinline__ int lower_bound_out(const DevView<W16>& g, int x, int y) {
    typedef Ent<W16> EN;
    int lo = g.off1o[x], hi = g.off1o[x + 1];
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (EN::id(g.ent1o[mid]) < y) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool adj_bit(const unsigned* __restrict__ bits, int words, int x, int y) {
    return (bits[(size_t)x * words + (y >> 5)] >> (y & 31)) & 1u;
}

// Delta of one rotation from the profit matrix (see header comment).
template <bool W16>
__device__ int triple_delta_S(const DevView<W16>& g, const unsigned* __restrict__ adj, int words,
                              int a, int b, int c, int rot) {
    typedef Ent<W16> EN;
    const int n = g.n;
    const int M[3] = {a, b, c};
    int sig[3];
    if (rot == 0) { sig[0] = b; sig[1] = c; sig[2] = a; }
    else          { sig[0] = c; sig[1] = a; sig[2] = b; }
    const int pm[3] = {g.p[a], g.p[b], g.p[c]};
    const int pn[3] = {g.p[sig[0]], g.p[sig[1]], g.p[sig[2]]};
    int d = 0;
    for (int i = 0; i < 3; i++)
        d += g.S[(size_t)M[i] * n + sig[i]] - g.S[(size_t)M[i] * n + M[i]];
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) {
            if (i == j) continue;
            const int x = M[i], y = M[j];
            if (!adj_bit(adj, words, x, y)) continue;
            const bool folded = (y == sig[i]);
            for (int q = lower_bound_out(g, x, y); q < g.off1o[x + 1]; q++) {
                const typename EN::T e = g.ent1o[q];
                if (EN::id(e) != y) break;
                const int w = EN::w(e);
                if (folded)  // undo the swap correction folded into S[x][y]
                    d -= imin(w, g.w2(pm[i], pm[j])) + imin(w, g.w2(pm[j], pm[i]))
                       - imin(w, g.w2(pm[i], pm[i])) - imin(w, g.w2(pm[j], pm[j]));
                d += imin(w, g.w2(pn[i], pn[j])) - imin(w, g.w2(pn[i], pm[j]))
                   - imin(w, g.w2(pm[i], pn[j])) + imin(w, g.w2(pm[i], pm[j]));
            }
        }
    }
    return d;
}

// Edge-walk delta of one rotation, elements t, t+nt, ... of the group.
template <bool W16>
__device__ int triple_delta_walk_part(const DevView<W16>& g, int a, int b, int c, int rot, int t, int nt) {
    typedef Ent<W16> EN;
    const int M[3] = {a, b, c};
    int sig[3];
    if (rot == 0) { sig[0] = b; sig[1] = c; sig[2] = a; }
    else          { sig[0] = c; sig[1] = a; sig[2] = b; }
    const int pm[3] = {g.p[a], g.p[b], g.p[c]};
    const int pn[3] = {g.p[sig[0]], g.p[sig[1]], g.p[sig[2]]};
    int lo[3], li[3];
    for (int i = 0; i < 3; i++) {
        lo[i] = g.off1o[M[i] + 1] - g.off1o[M[i]];
        li[i] = g.off1i[M[i] + 1] - g.off1i[M[i]];
    }
    const int tot = lo[0] + lo[1] + lo[2] + li[0] + li[1] + li[2];
    int d = 0;
    for (int k = t; k < tot; k += nt) {
        int q = k, i = 0;
        bool out = true;
        for (i = 0; i < 3; i++) { if (q < lo[i]) break; q -= lo[i]; }
        if (i == 3) {
            out = false;
            for (i = 0; i < 3; i++) { if (q < li[i]) break; q -= li[i]; }
        }
        const typename EN::T e = out ? g.ent1o[g.off1o[M[i]] + q] : g.ent1i[g.off1i[M[i]] + q];
        const int y = EN::id(e), w = EN::w(e);
        int jy = -1;
        for (int j = 0; j < 3; j++) if (M[j] == y) jy = j;
        if (!out && jy >= 0) continue;  // internal edge, counted from its source's out-list
        const int py = g.p[y];
        const int py_new = jy >= 0 ? pn[jy] : py;
        if (out) d += imin(w, g.w2(pn[i], py_new)) - imin(w, g.w2(pm[i], py));
        else     d += imin(w, g.w2(py_new, pn[i])) - imin(w, g.w2(py, pm[i]));
    }
    if (t == 0) {
        for (int i = 0; i < 3; i++)
            for (int q = g.offs[M[i]]; q < g.offs[M[i] + 1]; q++)
                d += imin(g.selfw[q], g.w2(pn[i], pn[i])) - imin(g.selfw[q], g.w2(pm[i], pm[i]));
    }
    return d;
}

// One warp per requested triple, both rotations.
template <bool W16>
__global__ void k_triple_deltas(DevView<W16> g, const int* __restrict__ ta, const int* __restrict__ tb,
                                const int* __restrict__ tc, long long k, int* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (; w < k; w += nw) {
        for (int rot = 0; rot < 2; rot++) {
            int d = triple_delta_walk_part<W16>(g, ta[w], tb[w], tc[w], rot, lane, 32);
            for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
            if (lane == 0) out[2 * w + rot] = d;
        }
    }
}

// Adjacency bitmap of G1 (x -> y), n rows of `words` 32-bit words.
template <bool W16>
__global__ void k_adj_bits(DevView<W16> g, unsigned* __restrict__ bits, int words) {
    typedef Ent<W16> EN;
    const int lane = threadIdx.x & 31;
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int x = warp; x < g.n; x += nwarps)
        for (int i = g.off1o[x] + lane; i < g.off1o[x + 1]; i += 32) {
            const int y = EN::id(g.ent1o[i]);
            atomicOr(&bits[(size_t)x * words + (y >> 5)], 1u << (y & 31));
        }
}

// Sample `partners` triples per vertex, evaluate both rotations from S and
// keep, per vertex a, the best improving (delta, slot, rotation) as a sort key
//   (0x7fffffff - delta) << 32 | a << 16 | slot << 1 | rot     (~0 if none)
// so ascending order is delta desc, a asc, slot asc, rotation asc.
template <bool W16>
__global__ void __launch_bounds__(256)
k_triple_eval(DevView<W16> g, const unsigned* __restrict__ adj, int words, int partners,
              unsigned long long seed, unsigned long long* __restrict__ keys,
              unsigned long long* __restrict__ counters /* [0]=valid triples */) {
    __shared__ unsigned long long best[8];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int a = blockIdx.x; a < g.n; a += gridDim.x) {
        unsigned long long k = ~0ull;
        unsigned valid = 0;
        for (int j = tid; j < partners; j += blockDim.x) {
            int b, c;
            if (!sample_triple<W16>(g, seed, a, j, b, c)) continue;
            valid++;
            for (int rot = 0; rot < 2; rot++) {
                const int d = triple_delta_S<W16>(g, adj, words, a, b, c, rot);
                if (d > 0) {
                    const unsigned long long kk = ((unsigned long long)(0x7fffffffu - (unsigned)d) << 32) |
                                                  ((unsigned long long)a << 16) | ((unsigned)j << 1) | (unsigned)rot;
                    if (kk < k) k = kk;
                }
            }
        }
        for (int o = 16; o; o >>= 1) {
            const unsigned long long x = __shfl_xor_sync(0xffffffffu, k, o);
            k = x < k ? x : k;
            valid += __shfl_xor_sync(0xffffffffu, valid, o);
        }
        if (lane == 0) { best[wid] = k; if (valid) atomicAdd(&counters[0], (unsigned long long)valid); }
        __syncthreads();
        if (tid == 0) {
            unsigned long long m = best[0];
            for (int i = 1; i < (int)(blockDim.x >> 5); i++) m = best[i] < m ? best[i] : m;
            keys[a] = m;
        }
        __syncthreads();
    }
}

// Sequential commit of sorted 3-cycle candidates (one CTA); same rule as
// k_commit: skip if a vertex was moved, re-verify if a vertex is tainted.
template <bool W16>
__global__ void __launch_bounds__(1024)
k_triple_commit(DevView<W16> g, const unsigned long long* __restrict__ keys, int nkeys, int max_scan,
                int max_verify, unsigned long long seed, CommitStats* __restrict__ st) {
    typedef Ent<W16> EN;
    extern __shared__ unsigned char flags[];
    unsigned char* used = flags;
    unsigned char* taint = flags + g.n;
    __shared__ int red[32];
    __shared__ int s_delta;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int i = tid; i < 2 * g.n; i += blockDim.x) flags[i] = 0;
    long long total = 0;
    int scanned = 0, verified = 0, committed = 0;
    __syncthreads();
    const int lim = (max_scan > 0 && max_scan < nkeys) ? max_scan : nkeys;
    for (int k = 0; k < lim; k++) {
        const unsigned long long key = keys[k];
        if (key == ~0ull) break;
        const int a = (int)((key >> 16) & 0xffffu), j = (int)((key >> 1) & 0x7fffu), rot = (int)(key & 1u);
        const int d0 = (int)(0x7fffffffu - (unsigned)(key >> 32));
        int b = 0, c = 0;
        sample_triple<W16>(g, seed, a, j, b, c);
        scanned++;
        if (used[a] | used[b] | used[c]) continue;
        int d = d0;
        if (taint[a] | taint[b] | taint[c]) {
            if (max_verify >= 0 && verified >= max_verify) continue;
            verified++;
            int part = triple_delta_walk_part<W16>(g, a, b, c, rot, tid, blockDim.x);
            for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            if (lane == 0) red[wid] = part;
            __syncthreads();
            if (wid == 0) {
                int v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0;
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) s_delta = v;
            }
            __syncthreads();
            d = s_delta;
            __syncthreads();
        }
        if (d <= 0) continue;
        if (tid == 0) {
            const int fa = g.p[a], fb = g.p[b], fc = g.p[c];
            int na, nb, nc;
            if (rot == 0) { na = fb; nb = fc; nc = fa; } else { na = fc; nb = fa; nc = fb; }
            g.p[a] = na; g.p[b] = nb; g.p[c] = nc;
            if (na < g.n) g.pinv[na] = a;
            if (nb < g.n) g.pinv[nb] = b;
            if (nc < g.n) g.pinv[nc] = c;
            used[a] = used[b] = used[c] = 1;
        }
        total += d;
        committed++;
        const int M[3] = {a, b, c};
        for (int i = 0; i < 3; i++) {
            const int x = M[i];
            const int o0 = g.off1o[x], o1 = g.off1o[x + 1] - o0;
            const int i0 = g.off1i[x], i1 = g.off1i[x + 1] - i0;
            for (int q = tid; q < o1 + i1; q += blockDim.x)
                taint[q < o1 ? EN::id(g.ent1o[o0 + q]) : EN::id(g.ent1i[i0 + q - o1])] = 1;
        }
        __syncthreads();
    }
    if (tid == 0) {
        st->total_delta = total;
        st->scanned = scanned;
        st->verified = verified;
        st->committed = committed;
    }
}

// ---------------------------------------------------------------------------
// Reference-order row scan: deltas of (m1, m2) for every m2 >= start, m2 != m1,
// on the current matching, and the smallest m2 whose delta is > 0.
template <bool W16>
__global__ void k_row_first(DevView<W16> g, int m1, int start, int* __restrict__ row_d,
                            int* __restrict__ first) {
    const int lane = threadIdx.x & 31;
    int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int m2 = start + w; m2 < g.n; m2 += nw) {
        if (m2 == m1) continue;
        int d = swap_delta_part<W16>(g, m1, m2, lane, 32);
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) {
            row_d[m2] = d;
            if (d > 0) atomicMin(first, m2);
        }
    }
}

// Applies the swap (m1, *first) when *first < n and records its delta.
static __global__ void k_apply_first(int* p, int* pinv, int n, int m1, const int* __restrict__ first,
                              const int* __restrict__ row_d, long long* __restrict__ acc) {
    const int m2 = *first;
    if (m2 >= n) return;
    const int f1 = p[m1], f2 = p[m2];
    p[m1] = f2; p[m2] = f1;
    if (f2 < n) pinv[f2] = m1;
    if (f1 < n) pinv[f1] = m2;
    acc[0] += row_d[m2];
    acc[1] += 1;
}

}  // namespace bm
