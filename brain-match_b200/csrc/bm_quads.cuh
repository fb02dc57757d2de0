// bm_quads.cuh -- 4-set permutation moves.
//
// The k = 4 case of the reference's k-permutation search
// (src/permutation.c:700-744: all permutations of the images of a vertex set,
// scored with calculate_permutation_delta :623-696), on sampled connected
// 4-sets.  Permutation q (1..23) is the q-th permutation of (0,1,2,3) in
// lexicographic order (0 = identity): vertex i of the set takes the image of
// vertex kQuadPerm[q][i].
//
// Delta of a permutation sigma of the set M from the profit matrix S:
//     sum_i S[M_i][M_sigma(i)] - S[M_i][M_i]
// plus, for every G1 edge x -> y inside the set, the exact term
//     min(w, W2[p'x][p'y]) - min(w, W2[p'x][p y]) - min(w, W2[p x][p'y]) + min(w, W2[p x][p y])
// (S counts the edge once at each end with the other end's current image),
// and, where y is the vertex whose image x takes, minus the pair-swap
// correction that S folds into S[x][y] -- the same algebra as the 3-cycles.
#pragma once
#include <cstdint>
#include "bm_triples.cuh"

namespace bm {

__constant__ unsigned char kQuadPerm[24][4] = {
    {0,1,2,3},{0,1,3,2},{0,2,1,3},{0,2,3,1},{0,3,1,2},{0,3,2,1},
    {1,0,2,3},{1,0,3,2},{1,2,0,3},{1,2,3,0},{1,3,0,2},{1,3,2,0},
    {2,0,1,3},{2,0,3,1},{2,1,0,3},{2,1,3,0},{2,3,0,1},{2,3,1,0},
    {3,0,1,2},{3,0,2,1},{3,1,0,2},{3,1,2,0},{3,2,0,1},{3,2,1,0}};

// The 3-step walk of slot j of vertex a: a -> b -> c -> d along undirected G1
// edges, h1 = mix64(seed ^ (a << 32 | j)), h2 = mix64(h1), h3 = mix64(h2);
// false unless the four vertices are distinct.
template <bool W16>
__device__ __forceinline__ bool sample_quad(const DevView<W16>& g, unsigned long long seed, int a, int j, int& b,
                                            int& c, int& d) {
    const int da = ndeg(g, a);
    if (da == 0) return false;
    const unsigned long long h1 = mix64(seed ^ (((unsigned long long)a << 32) | (unsigned)j));
    b = nbr_at(g, a, (int)(h1 % (unsigned long long)da));
    const int db = ndeg(g, b);
    if (db == 0) return false;
    const unsigned long long h2 = mix64(h1);
    c = nbr_at(g, b, (int)(h2 % (unsigned long long)db));
    const int dc = ndeg(g, c);
    if (dc == 0) return false;
    const unsigned long long h3 = mix64(h2);
    d = nbr_at(g, c, (int)(h3 % (unsigned long long)dc));
    return b != a && c != a && c != b && d != a && d != b && d != c;
}

// Delta of permutation q of the set M from S (see the header comment).
template <bool W16>
__device__ int quad_delta_S(const DevView<W16>& g, const unsigned* __restrict__ adj, int words, const int* M,
                            const int* pm, int q) {
    typedef Ent<W16> EN;
    const int n = g.n;
    int sg[4], pn[4];
#pragma unroll
    for (int i = 0; i < 4; i++) { sg[i] = kQuadPerm[q][i]; pn[i] = pm[sg[i]]; }
    int d = 0;
#pragma unroll
    for (int i = 0; i < 4; i++) {
        if (sg[i] == i) continue;  // a vertex that keeps its image adds nothing from S
        d += g.S[(size_t)M[i] * n + M[sg[i]]] - g.S[(size_t)M[i] * n + M[i]];
    }
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) {
            if (i == j) continue;
            const int x = M[i], y = M[j];
            if (!adj_bit(adj, words, x, y)) continue;
            const bool folded = (sg[i] == j);  // S[x][y] was read, with the swap correction of edge x -> y
            for (int e = lower_bound_out(g, x, y); e < g.off1o[x + 1]; e++) {
                const typename EN::T en = g.ent1o[e];
                if (EN::id(en) != y) break;
                const int w = EN::w(en);
                if (folded)
                    d -= imin(w, g.w2(pm[i], pm[j])) + imin(w, g.w2(pm[j], pm[i]))
                       - imin(w, g.w2(pm[i], pm[i])) - imin(w, g.w2(pm[j], pm[j]));
                // terms S counted for this edge: x's out-edge with y's current image
                // (only when x moves) and y's in-edge with x's current image (only when y moves)
                int counted = 0;
                if (sg[i] != i) counted += imin(w, g.w2(pn[i], pm[j])) - imin(w, g.w2(pm[i], pm[j]));
                if (sg[j] != j) counted += imin(w, g.w2(pm[i], pn[j])) - imin(w, g.w2(pm[i], pm[j]));
                d += imin(w, g.w2(pn[i], pn[j])) - imin(w, g.w2(pm[i], pm[j])) - counted;
            }
        }
    }
    return d;
}

// Exact edge-walk delta of permutation q of the set M on the current
// matching: elements t, t + nt, ... of the set's incident list entries.
template <bool W16>
__device__ int quad_delta_walk_part(const DevView<W16>& g, const int* M, int q, int t, int nt) {
    typedef Ent<W16> EN;
    int pm[4], pn[4], lo[4], li[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        pm[i] = g.p[M[i]];
        lo[i] = g.off1o[M[i] + 1] - g.off1o[M[i]];
        li[i] = g.off1i[M[i] + 1] - g.off1i[M[i]];
    }
#pragma unroll
    for (int i = 0; i < 4; i++) pn[i] = pm[kQuadPerm[q][i]];
    const int tot = lo[0] + lo[1] + lo[2] + lo[3] + li[0] + li[1] + li[2] + li[3];
    int d = 0;
    for (int k = t; k < tot; k += nt) {
        int r = k, i = 0;
        bool out = true;
        for (i = 0; i < 4; i++) { if (r < lo[i]) break; r -= lo[i]; }
        if (i == 4) {
            out = false;
            for (i = 0; i < 4; i++) { if (r < li[i]) break; r -= li[i]; }
        }
        const typename EN::T e = out ? g.ent1o[g.off1o[M[i]] + r] : g.ent1i[g.off1i[M[i]] + r];
        const int y = EN::id(e), w = EN::w(e);
        int jy = -1;
        for (int j = 0; j < 4; j++) if (M[j] == y) jy = j;
        if (!out && jy >= 0) continue;  // internal edge, counted from its source's out-list
        const int py = g.p[y];
        const int py_new = jy >= 0 ? pn[jy] : py;
        if (out) d += imin(w, g.w2(pn[i], py_new)) - imin(w, g.w2(pm[i], py));
        else     d += imin(w, g.w2(py_new, pn[i])) - imin(w, g.w2(py, pm[i]));
    }
    if (t == 0) {
        for (int i = 0; i < 4; i++)
            for (int s = g.offs[M[i]]; s < g.offs[M[i] + 1]; s++)
                d += imin(g.selfw[s], g.w2(pn[i], pn[i])) - imin(g.selfw[s], g.w2(pm[i], pm[i]));
    }
    return d;
}

// One warp per requested (set, permutation).
template <bool W16>
__global__ void k_quad_deltas(DevView<W16> g, const int* __restrict__ sets, const int* __restrict__ perms,
                              long long k, int* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (; w < k; w += nw) {
        const int M[4] = {sets[4 * w], sets[4 * w + 1], sets[4 * w + 2], sets[4 * w + 3]};
        int d = quad_delta_walk_part<W16>(g, M, perms[w], lane, 32);
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) out[w] = d;
    }
}

// Best improving permutation of the set M (largest delta, then smallest q;
// q = 0 and delta 0 if none improves).  Every value the 23 permutations need
// is loaded once: the 4x4 block of S among the set's vertices, the 4x4 block
// of W2 among their current images, and the set's internal G1 edges (up to
// kQuadMaxInternal entries; a set with more falls back to quad_delta_S per
// permutation, with the same result).
constexpr int kQuadMaxInternal = 12;
template <bool W16>
__device__ void quad_best(const DevView<W16>& g, const unsigned* __restrict__ adj, int words, const int* M,
                          const int* pm, int& best_d, int& best_q) {
    typedef Ent<W16> EN;
    const int n = g.n;
    best_d = 0;
    best_q = 0;
    int ie_ij[kQuadMaxInternal], ie_w[kQuadMaxInternal];  // (i << 2 | j), weight
    int ne = 0;
    bool overflow = false;
    for (int i = 0; i < 4 && !overflow; i++)
        for (int j = 0; j < 4 && !overflow; j++) {
            if (i == j || !adj_bit(adj, words, M[i], M[j])) continue;
            for (int e = lower_bound_out(g, M[i], M[j]); e < g.off1o[M[i] + 1]; e++) {
                const typename EN::T en = g.ent1o[e];
                if (EN::id(en) != M[j]) break;
                if (ne == kQuadMaxInternal) { overflow = true; break; }
                ie_ij[ne] = (i << 2) | j;
                ie_w[ne] = EN::w(en);
                ne++;
            }
        }
    if (overflow) {
        for (int q = 1; q < 24; q++) {
            const int dd = quad_delta_S<W16>(g, adj, words, M, pm, q);
            if (dd > best_d) { best_d = dd; best_q = q; }
        }
        return;
    }
    int sm[4][4], wm[4][4];  // S[M_i][M_j]; W2[p M_i][p M_j]
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            sm[i][j] = g.S[(size_t)M[i] * n + M[j]];
            wm[i][j] = g.w2(pm[i], pm[j]);
        }
    for (int q = 1; q < 24; q++) {
        int sg[4];
#pragma unroll
        for (int i = 0; i < 4; i++) sg[i] = kQuadPerm[q][i];
        int d = 0;
#pragma unroll
        for (int i = 0; i < 4; i++)
            if (sg[i] != i) d += sm[i][sg[i]] - sm[i][i];
        for (int t = 0; t < ne; t++) {
            const int i = ie_ij[t] >> 2, j = ie_ij[t] & 3, w = ie_w[t];
            if (sg[i] == j)
                d -= imin(w, wm[i][j]) + imin(w, wm[j][i]) - imin(w, wm[i][i]) - imin(w, wm[j][j]);
            int counted = 0;
            if (sg[i] != i) counted += imin(w, wm[sg[i]][j]) - imin(w, wm[i][j]);
            if (sg[j] != j) counted += imin(w, wm[i][sg[j]]) - imin(w, wm[i][j]);
            d += imin(w, wm[sg[i]][sg[j]]) - imin(w, wm[i][j]) - counted;
        }
        if (d > best_d) { best_d = d; best_q = q; }
    }
}

// Sample `partners` 4-sets per vertex a, evaluate the 23 permutations of each
// from S, keep per vertex the best improving one as a sort key
//   (0x7fffffff - delta) << 32 | a << 16 | slot << 5 | q     (~0 if none)
// (ascending order: delta desc, a asc, slot asc, q asc).
template <bool W16>
__global__ void __launch_bounds__(256)
k_quad_eval(DevView<W16> g, const unsigned* __restrict__ adj, int words, int partners, unsigned long long seed,
            unsigned long long* __restrict__ keys, unsigned long long* __restrict__ counters /* [0] valid sets */) {
    __shared__ unsigned long long best[8];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int a = blockIdx.x; a < g.n; a += gridDim.x) {
        unsigned long long k = ~0ull;
        unsigned valid = 0;
        for (int j = tid; j < partners; j += blockDim.x) {
            int b, c, d;
            if (!sample_quad<W16>(g, seed, a, j, b, c, d)) continue;
            valid++;
            const int M[4] = {a, b, c, d};
            const int pm[4] = {g.p[a], g.p[b], g.p[c], g.p[d]};
            int dd, q;
            quad_best<W16>(g, adj, words, M, pm, dd, q);
            if (dd > 0) {
                const unsigned long long kk = ((unsigned long long)(0x7fffffffu - (unsigned)dd) << 32) |
                                              ((unsigned long long)a << 16) | ((unsigned)j << 5) | (unsigned)q;
                if (kk < k) k = kk;
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

// Sequential commit of the sorted 4-set candidates (one CTA), the rule of the
// 3-cycle round: skip a set with a vertex already moved, re-evaluate exactly
// a set with a moved G1 neighbour, commit iff the delta is > 0.
template <bool W16>
__global__ void __launch_bounds__(1024)
k_quad_commit(DevView<W16> g, const unsigned long long* __restrict__ keys, int nkeys, int max_scan,
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
        const int a = (int)((key >> 16) & 0xffffu), j = (int)((key >> 5) & 0x7ffu), q = (int)(key & 31u);
        const int d0 = (int)(0x7fffffffu - (unsigned)(key >> 32));
        int b = 0, c = 0, d = 0;
        sample_quad<W16>(g, seed, a, j, b, c, d);
        scanned++;
        if (used[a] | used[b] | used[c] | used[d]) continue;
        const int M[4] = {a, b, c, d};
        int dd = d0;
        if (taint[a] | taint[b] | taint[c] | taint[d]) {
            if (max_verify >= 0 && verified >= max_verify) continue;
            verified++;
            int part = quad_delta_walk_part<W16>(g, M, q, tid, blockDim.x);
            for (int o = 16; o; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
            if (lane == 0) red[wid] = part;
            __syncthreads();
            if (wid == 0) {
                int v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0;
                for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) s_delta = v;
            }
            __syncthreads();
            dd = s_delta;
            __syncthreads();
        }
        if (dd <= 0) continue;
        if (tid == 0) {
            int f[4];
            for (int i = 0; i < 4; i++) f[i] = g.p[M[i]];
            for (int i = 0; i < 4; i++) {
                const int nf = f[kQuadPerm[q][i]];
                g.p[M[i]] = nf;
                if (nf < g.n) g.pinv[nf] = M[i];
                used[M[i]] = 1;
            }
        }
        total += dd;
        committed++;
        for (int i = 0; i < 4; i++) {
            const int x = M[i];
            const int o0 = g.off1o[x], o1 = g.off1o[x + 1] - o0;
            const int i0 = g.off1i[x], i1 = g.off1i[x + 1] - i0;
            for (int r = tid; r < o1 + i1; r += blockDim.x)
                taint[r < o1 ? EN::id(g.ent1o[o0 + r]) : EN::id(g.ent1i[i0 + r - o1])] = 1;
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

}  // namespace bm
