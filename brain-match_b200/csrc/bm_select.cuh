// bm_select.cuh -- pair combine and move selection of the sweep.
//
// k_combine64: 64x64 tiles of the upper triangle of S.  Each tile (I,J), I<=J,
//   reads S[I][J] and S[J][I] once (coalesced rows), forms
//   delta(a,b) = S[a][b] + S[b][a] - S[a][a] - S[b][b] and writes, for every
//   vertex of the tile, its best partner inside the tile to a partial array
//   P[tile column][vertex]; k_best_reduce folds the partials into rowbest.
//   No atomics; every (tile, vertex) slot is written exactly once.
// k_commit_seq: the sequential set commit (candidates sorted by delta desc,
//   skip a pair whose vertex already moved, re-evaluate it on the current
//   matching, commit iff > 0).
#pragma once
#include "bm_kernels.cuh"

namespace bm {

constexpr int kTile = 64;

__global__ void __launch_bounds__(256)
k_combine64(const int* __restrict__ S, int n, unsigned long long* __restrict__ part,
            int* __restrict__ all_out) {
    __shared__ int sA[kTile][kTile + 1];  // sA[r][c] = S[a0+r][b0+c]
    __shared__ int sB[kTile][kTile + 1];  // sB[r][c] = S[b0+r][a0+c]
    __shared__ int dA[kTile], dB[kTile];
    __shared__ unsigned long long cpart[8][kTile];
    const int ti = blockIdx.y, tj = blockIdx.x;
    if (ti > tj) return;
    const int a0 = ti * kTile, b0 = tj * kTile;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;  // 8 warps
    for (int i = tid; i < kTile * kTile; i += 256) {
        const int r = i >> 6, c = i & 63;
        const int a = a0 + r, b = b0 + c;
        sA[r][c] = (a < n && b < n) ? S[(size_t)a * n + b] : 0;
        const int bb = b0 + r, aa = a0 + c;
        sB[r][c] = (bb < n && aa < n) ? S[(size_t)bb * n + aa] : 0;
    }
    if (tid < kTile) {
        const int a = a0 + tid, b = b0 + tid;
        dA[tid] = a < n ? S[(size_t)a * n + a] : 0;
        dB[tid] = b < n ? S[(size_t)b * n + b] : 0;
    }
    __syncthreads();
    const bool diag = (ti == tj);
    // columns handled by this lane: c0 = lane, c1 = lane + 32; rows r = wid, wid+8, ...
    unsigned long long cb0 = 0, cb1 = 0;
    const int c0 = lane, c1 = lane + 32;
    const int b_0 = b0 + c0, b_1 = b0 + c1;
    for (int r = wid; r < kTile; r += 8) {
        const int a = a0 + r;
        unsigned long long rb = 0;
        if (a < n) {
            if (b_0 < n && b_0 != a) {
                const int d = sA[r][c0] + sB[c0][r] - dA[r] - dB[c0];
                rb = kmax(rb, pack_best(d, b_0));
                cb0 = kmax(cb0, pack_best(d, a));
                if (all_out && a < b_0) all_out[(long long)a * (2LL * n - a - 1) / 2 + (b_0 - a - 1)] = d;
            }
            if (b_1 < n && b_1 != a) {
                const int d = sA[r][c1] + sB[c1][r] - dA[r] - dB[c1];
                rb = kmax(rb, pack_best(d, b_1));
                cb1 = kmax(cb1, pack_best(d, a));
                if (all_out && a < b_1) all_out[(long long)a * (2LL * n - a - 1) / 2 + (b_1 - a - 1)] = d;
            }
        }
        for (int o = 16; o; o >>= 1) rb = kmax(rb, __shfl_xor_sync(0xffffffffu, rb, o));
        if (lane == 0 && a < n) part[(size_t)tj * n + a] = rb;  // row partial of a over this tile
    }
    // column partials (vertices b of the tile, over this tile's rows); a
    // diagonal tile's row partials already cover both orders of every pair
    if (!diag) {
        cpart[wid][c0] = cb0;
        cpart[wid][c1] = cb1;
        __syncthreads();
        if (tid < kTile) {
            unsigned long long k = cpart[0][tid];
            for (int w = 1; w < 8; w++) k = kmax(k, cpart[w][tid]);
            const int b = b0 + tid;
            if (b < n) part[(size_t)ti * n + b] = k;
        }
    }
}

// rowbest[x] = max over tile columns t of part[t][x]
__global__ void k_best_reduce(const unsigned long long* __restrict__ part, int n, int tiles,
                              unsigned long long* __restrict__ rowbest) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    unsigned long long k = 0;
    for (int t = 0; t < tiles; t++) k = kmax(k, part[(size_t)t * n + x]);
    rowbest[x] = k;
}

// ---------------------------------------------------------------------------
// Sequential set commit (one CTA), candidates in sorted order:
//   * skip the pair if either vertex already moved in this sweep;
//   * otherwise its current delta is the sweep delta plus, for every G1 edge
//     from one of its vertices x to an already-moved vertex z, the change of
//     that edge's term between z's pre-move image (pold) and its image now.
//     The CTA finds those edges in one coalesced pass over the pair's four
//     edge lists (a flag check per entry; W2 is read only for moved
//     neighbours).  A pair with at least one moved neighbour is the
//     "re-verified" case of the rule (counted, and limited by max_verify);
//   * commit iff the current delta is > 0.
// Warp 0 skips runs of candidates with a moved vertex 32 at a time, so only
// live candidates cost a pass of the CTA.
template <bool W16>
__global__ void __launch_bounds__(1024)
k_commit_seq(DevView<W16> g, const unsigned long long* __restrict__ keys, int lim, int max_verify,
             int* __restrict__ pold, CommitStats* __restrict__ st) {
    typedef Ent<W16> EN;
    extern __shared__ unsigned char used[];  // n bytes
    __shared__ int s_k, s_lo, s_hi, s_d0, s_done, s_scanned;
    __shared__ int s_red[32], s_cnt[32];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarp = blockDim.x >> 5;
    const int n = g.n;
    for (int i = tid; i < n; i += blockDim.x) used[i] = 0;
    if (tid == 0) { s_k = 0; s_scanned = 0; }
    long long total = 0;
    int verified = 0, committed = 0;
    __syncthreads();
    for (;;) {
        // ---- warp 0: next candidate whose vertices have not moved ----
        if (wid == 0) {
            int k = s_k, scanned = s_scanned, done = 1;
            while (k < lim) {
                const int idx = k + lane;
                const unsigned long long key = idx < lim ? keys[idx] : ~0ull;
                const bool valid = key != ~0ull;
                const int lo = valid ? (int)((key >> 16) & 0xffffu) : 0;
                const int hi = valid ? (int)(key & 0xffffu) : 0;
                const bool live = valid && !used[lo] && !used[hi];
                const unsigned vmask = __ballot_sync(0xffffffffu, valid);
                const unsigned lmask = __ballot_sync(0xffffffffu, live);
                if (lmask) {
                    const int l = __ffs(lmask) - 1;
                    scanned += l + 1;
                    if (lane == l) {
                        s_lo = lo; s_hi = hi;
                        s_d0 = (int)(0x7fffffffu - (unsigned)(key >> 32));
                    }
                    k += l + 1;
                    done = 0;
                    break;
                }
                const int nvalid = __popc(vmask);  // valid keys form a prefix
                scanned += nvalid;
                k += 32;
                if (nvalid < 32) { k = lim; break; }
            }
            if (lane == 0) { s_k = k; s_scanned = scanned; s_done = done; }
        }
        __syncthreads();
        if (s_done) break;
        const int a = s_lo, b = s_hi;
        // ---- corrections from edges to already-moved vertices ----
        int corr = 0, cnt = 0;
        {
            const int pa = g.p[a], pb = g.p[b];
            const int la0 = g.off1o[a], la = g.off1o[a + 1] - la0;
            const int ia0 = g.off1i[a], ia = g.off1i[a + 1] - ia0;
            const int lb0 = g.off1o[b], lb = g.off1o[b + 1] - lb0;
            const int ib0 = g.off1i[b], ib = g.off1i[b + 1] - ib0;
            const int tot = la + ia + lb + ib;
            for (int e = tid; e < tot; e += blockDim.x) {
                int q = e, kind;
                typename EN::T en;
                if (q < la) { en = g.ent1o[la0 + q]; kind = 0; }
                else if ((q -= la) < ia) { en = g.ent1i[ia0 + q]; kind = 1; }
                else if ((q -= ia) < lb) { en = g.ent1o[lb0 + q]; kind = 2; }
                else { q -= lb; en = g.ent1i[ib0 + q]; kind = 3; }
                const int x = EN::id(en);
                if (x == a || x == b || !used[x]) continue;
                const int w = EN::w(en), px = g.p[x], qx = pold[x];
                if (kind == 0)      corr += (imin(w, g.w2(pb, px)) - imin(w, g.w2(pa, px))) - (imin(w, g.w2(pb, qx)) - imin(w, g.w2(pa, qx)));
                else if (kind == 1) corr += (imin(w, g.w2(px, pb)) - imin(w, g.w2(px, pa))) - (imin(w, g.w2(qx, pb)) - imin(w, g.w2(qx, pa)));
                else if (kind == 2) corr += (imin(w, g.w2(pa, px)) - imin(w, g.w2(pb, px))) - (imin(w, g.w2(pa, qx)) - imin(w, g.w2(pb, qx)));
                else                corr += (imin(w, g.w2(px, pa)) - imin(w, g.w2(px, pb))) - (imin(w, g.w2(qx, pa)) - imin(w, g.w2(qx, pb)));
                cnt++;
            }
        }
        for (int o = 16; o; o >>= 1) {
            corr += __shfl_xor_sync(0xffffffffu, corr, o);
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        }
        if (lane == 0) { s_red[wid] = corr; s_cnt[wid] = cnt; }
        __syncthreads();
        // ---- decide (thread 0) ----
        if (tid == 0) {
            int c = 0, m = 0;
            for (int w = 0; w < nwarp; w++) { c += s_red[w]; m += s_cnt[w]; }
            bool ok = true;
            int d = s_d0;
            if (m > 0) {
                if (max_verify >= 0 && verified >= max_verify) ok = false;
                else { verified++; d += c; }
            }
            if (ok && d > 0) {
                const int fa = g.p[a], fb = g.p[b];
                pold[a] = fa; pold[b] = fb;
                g.p[a] = fb; g.p[b] = fa;
                if (fb < n) g.pinv[fb] = a;
                if (fa < n) g.pinv[fa] = b;
                used[a] = 1; used[b] = 1;
                total += d;
                committed++;
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        st->total_delta = total;
        st->scanned = s_scanned;
        st->verified = verified;
        st->committed = committed;
    }
}

}  // namespace bm
