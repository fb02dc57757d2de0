// bm_combine_tma.cuh -- the sweep's pair combine with TMA-staged tiles.
//
// Same result as k_combine64 (bm_select.cuh): for every 64x64 tile (I,J),
// I <= J, of the profit matrix S, delta(a,b) = S[a][b] + S[b][a] - S[a][a]
// - S[b][b] and the best partner of every vertex inside the tile, written to
// the per-tile partial array that k_best_reduce folds.  The difference is how
// S reaches shared memory: a persistent CTA walks its share of the tile pairs
// and keeps kCmbStages pairs in flight, each pair's two 16 KB tiles
// (S[I][J] and S[J][I]) fetched by cp.async.bulk.tensor (TMA, the CTA's own
// shared memory, no multicast) onto one mbarrier with an expected byte count.
// Rows land densely (64 ints, 256 bytes), so lanes read the tiles along
// diagonals: lane l of a warp takes row r = l and column (l + k) mod 32 at
// step k, which hits 32 distinct banks both in S[I][J] (bank = column) and
// in the transposed S[J][I] (bank = row).  A row's best accumulates in one
// thread; a column's best arrives by one shuffle per step.
//
// Needs n % 4 == 0 (the tensor map's row stride must be a multiple of 16
// bytes); other n take k_combine64.  Every wait on a tile is bounded: when
// one runs out the CTA sets bit 4 of err, waits (bounded) for the copies it
// issued and returns, and the host reports BM_E_TIMEOUT.
#pragma once
#include <cstdint>
#include <climits>
#include <cuda.h>
#include "bm_kernels.cuh"

namespace bm {

constexpr int kCmbT = 64;                                // tile edge
constexpr int kCmbStages = 3;                            // tile pairs in flight per CTA
constexpr int kCmbTileBytes = kCmbT * kCmbT * 4;         // 16 KB
constexpr int kCmbStageBytes = 2 * kCmbTileBytes;        // S[I][J] and S[J][I]
constexpr int kCmbThreads = 512;                         // 16 warps: 4 sub-blocks x 4 step ranges
constexpr int kCmbSteps = 8;                             // diagonal steps per warp
constexpr int kCmbSmem = kCmbStages * kCmbStageBytes + 128 + 64;   // + alignment + barriers
constexpr int kCmbErrBit = 4;

__device__ __forceinline__ uint32_t cmb_smem(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ bool cmb_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool cmb_wait(uint32_t bar, uint32_t parity, int limit = 1 << 22) {
    for (int i = 0; i < limit; i++)
        if (cmb_try_wait(bar, parity)) return true;
    return false;
}

// Both tiles of a pair onto one mbarrier: tile A = rows a0.., columns b0..;
// tile B = rows b0.., columns a0.. (x = column, y = row; x is a multiple of
// 64 elements, so every copy starts on a 256-byte boundary).
__device__ __forceinline__ void cmb_issue(const CUtensorMap* tm, uint32_t dst, uint32_t bar, int a0, int b0) {
    // the stage's earlier reads (generic proxy) are ordered before the copy's writes
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(bar), "r"(kCmbStageBytes) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :: "r"(dst), "l"(tm), "r"(b0), "r"(a0), "r"(bar) : "memory");
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :: "r"(dst + kCmbTileBytes), "l"(tm), "r"(a0), "r"(b0), "r"(bar) : "memory");
}

// Tile pair p (0 .. tiles*(tiles+1)/2 - 1) -> (ti, tj), ti <= tj, row-major
// over the upper triangle.
__device__ __forceinline__ void cmb_pair(long long p, int tiles, int* ti, int* tj) {
    // first pair of row t: t*tiles - t*(t-1)/2
    const double T = (double)tiles + 0.5;
    int t = (int)(T - sqrt(T * T - 2.0 * (double)p));
    if (t < 0) t = 0;
    if (t > tiles - 1) t = tiles - 1;
    auto first = [&](int r) { return (long long)r * tiles - (long long)r * (r - 1) / 2; };
    while (t > 0 && first(t) > p) t--;
    while (t + 1 < tiles && first(t + 1) <= p) t++;
    *ti = t;
    *tj = t + (int)(p - first(t));
}

static __global__ void __launch_bounds__(kCmbThreads)
k_combine_tma(const __grid_constant__ CUtensorMap tm, const int* __restrict__ diag, int n, int tiles,
              unsigned long long* __restrict__ part, int* __restrict__ err, int stall) {
    extern __shared__ __align__(128) unsigned char cmb_raw[];
    const uint32_t raw = cmb_smem(cmb_raw);
    const uint32_t base = (raw + 127u) & ~127u;
    unsigned char* basep = cmb_raw + (base - raw);
    const uint32_t bars = base + kCmbStages * kCmbStageBytes;
    __shared__ int s_db[kCmbT];                             // S[b][b] of the tile's columns
    __shared__ unsigned long long s_rk[8][kCmbT], s_ck[8][kCmbT];
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    // warp: 32x32 sub-block (row half hr, column half hc), steps kq*8 .. kq*8+7
    const int hr = wid & 1, hc = (wid >> 1) & 1, kq = wid >> 2;
    const long long npairs = (long long)tiles * (tiles + 1) / 2;
    const long long step = gridDim.x;
    const long long first = blockIdx.x;
    if (tid == 0) {
        for (int s = 0; s < kCmbStages; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bars + 8 * s) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        for (int s = 0; s < kCmbStages; s++) {
            const long long p = first + s * step;
            if (p < npairs) {
                int ti, tj;
                cmb_pair(p, tiles, &ti, &tj);
                cmb_issue(&tm, base + s * kCmbStageBytes, bars + 8 * s, ti * kCmbT, tj * kCmbT);
            }
        }
    }
    __syncthreads();
    __shared__ int s_ok;
    if (tid == 0) s_ok = 1;
    int it = 0;
    for (long long p = first; p < npairs; p += step, it++) {
        const int s = it % kCmbStages;
        const uint32_t phase = (uint32_t)((it / kCmbStages) & 1);
        int ti, tj;
        cmb_pair(p, tiles, &ti, &tj);
        const int a0 = ti * kCmbT, b0 = tj * kCmbT;
        if (tid < kCmbT) s_db[tid] = (b0 + tid < n) ? __ldg(&diag[b0 + tid]) : 0;
        if (tid == 0) {
            bool ok = cmb_wait(bars + 8 * s, phase);
            // test hook (bm_test_stall): CTA 0's first tile also waits for the
            // stage's next phase, which no copy completes before it is issued
            if (ok && stall && blockIdx.x == 0 && it == 0) ok = cmb_wait(bars + 8 * s, phase ^ 1u, 1 << 12);
            if (!ok) { s_ok = 0; atomicOr(err, 1 << kCmbErrBit); }
        }
        __syncthreads();
        if (!s_ok) break;
        const int* sA = reinterpret_cast<const int*>(basep + s * kCmbStageBytes);   // [row a][col b]
        const int* sB = sA + kCmbT * kCmbT;                                          // [row b][col a]
        const int r = 32 * hr + lane, a = a0 + r;
        const int da = a < n ? __ldg(&diag[a]) : 0;
        const bool diagt = ti == tj;
        // bests as packed keys (delta + 2^31) << 32 | ~partner: larger delta,
        // then smaller partner; 0 = none
        unsigned long long rk = 0, ck = 0;
        if (!diagt && a0 + kCmbT <= n && b0 + kCmbT <= n) {   // full off-diagonal tile: no checks
#pragma unroll
            for (int q = 0; q < kCmbSteps; q++) {
                const int k = kCmbSteps * kq + q;
                const int c = 32 * hc + ((lane + k) & 31);
                const int d = sA[r * kCmbT + c] + sB[c * kCmbT + r] - da - s_db[c];
                rk = kmax(rk, pack_best(d, b0 + c));
                // column 32 hc + lane was taken at this step by lane (lane - k) mod 32
                const int src = (lane - k) & 31;
                const int dc = __shfl_sync(0xffffffffu, d, src);
                ck = kmax(ck, pack_best(dc, a0 + 32 * hr + src));
            }
        } else {
            for (int q = 0; q < kCmbSteps; q++) {
                const int k = kCmbSteps * kq + q;
                const int c = 32 * hc + ((lane + k) & 31), b = b0 + c;
                const bool v = a < n && b < n && a != b;
                const int d = v ? sA[r * kCmbT + c] + sB[c * kCmbT + r] - da - s_db[c] : 0;
                if (v) rk = kmax(rk, pack_best(d, b));
                const int src = (lane - k) & 31;
                const int dc = __shfl_sync(0xffffffffu, d, src);
                const bool vc = __shfl_sync(0xffffffffu, v ? 1 : 0, src) != 0;
                if (vc) ck = kmax(ck, pack_best(dc, a0 + 32 * hr + src));
            }
        }
        s_rk[2 * kq + hc][r] = rk;
        s_ck[2 * kq + hr][32 * hc + lane] = ck;
        __syncthreads();   // stage s is free again, the partials are complete
        if (tid == 0) {
            const long long q = p + kCmbStages * step;
            if (q < npairs) {
                int qi, qj;
                cmb_pair(q, tiles, &qi, &qj);
                cmb_issue(&tm, base + s * kCmbStageBytes, bars + 8 * s, qi * kCmbT, qj * kCmbT);
            }
        }
        if (tid < kCmbT) {
            const int x = a0 + tid;
            unsigned long long k = s_rk[0][tid];
#pragma unroll
            for (int w = 1; w < 8; w++) k = kmax(k, s_rk[w][tid]);
            if (x < n) part[(size_t)tj * n + x] = k;
        } else if (tid < 2 * kCmbT && !diagt) {   // a diagonal tile's rows already cover both orders
            const int c = tid - kCmbT, x = b0 + c;
            unsigned long long k = s_ck[0][c];
#pragma unroll
            for (int w = 1; w < 8; w++) k = kmax(k, s_ck[w][c]);
            if (x < n) part[(size_t)ti * n + x] = k;
        }
        // s_rk / s_ck and s_db are rewritten only after the next tile's wait,
        // which every thread reaches through a barrier
    }
    // on a timeout: wait (bounded) for the copies still in flight into this
    // CTA's shared memory before it exits
    if (tid == 0 && !s_ok) {
        for (int j = 0; j < kCmbStages; j++) {
            const int jt = it + j;
            const long long q = first + (long long)jt * step;
            if (q < npairs) cmb_wait(bars + 8 * (jt % kCmbStages), (uint32_t)((jt / kCmbStages) & 1));
        }
    }
}

// S[a][a] for every a (the combine reads it per tile row and column).
static __global__ void k_diag(const int* __restrict__ S, int n, int* __restrict__ diag) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a < n) diag[a] = S[(size_t)a * n + a];
}

}  // namespace bm
