// bm_hub.cuh -- the hub part of the profit matrix on the tensor cores.
//
// The in-edge terms of the profit matrix,
//     S[a][b] += sum_{(u,a,w1) in in1(a)} min(w1, W2[p u][p b]),
// are dominated, once hubs are matched to hubs, by the few G1 vertices u of
// largest out-degree: each such u is an in-neighbour of almost every a and
// its image's G2 out-list covers almost every b.  For small integers
//     min(x, y) = sum_{t=1..T} [x >= t][y >= t]  +  [x > T][y > T] (min(x,y) - T)
// so the hub terms split into an exact binary GEMM
//     S_H[a][b] = sum_{h, t} A[a][h*T + t-1] * B[b][h*T + t-1]
//     A[a][h*T+t-1] = #{G1 entries u_h -> a with weight >= t}   (fixed)
//     B[b][h*T+t-1] = [W2[p u_h][p b] >= t]                     (per sweep)
// and a sparse residual over the few entries above T (scattered by the
// profit-row kernel).  The GEMM runs as tcgen05.mma kind::i8 (u8 x u8 -> s32,
// exact) with the accumulator in TMEM; operand tiles are staged in shared
// memory in the 128-byte-swizzled K-major layout by cp.async.
#pragma once
#include <cstdint>
#include "bm_kernels.cuh"

namespace bm {

constexpr int kHubT = 8;          // thresholds per hub
constexpr int kHubMaxHubs = 256;  // K up to 2048
constexpr int kGemmM = 128, kGemmN = 256, kGemmKC = 128;  // tile rows, cols, K bytes per stage
constexpr int kGemmStages = 2;
constexpr int kGemmThreads = 128;
constexpr int kGemmStageBytes = (kGemmM + kGemmN) * kGemmKC;          // 48 KB
constexpr int kGemmSmem = kGemmStages * kGemmStageBytes + 1024 + 256;  // + alignment + barriers

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (SBO), Blackwell descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);           // start address
    d |= (uint64_t)1u << 16;                          // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;                // stride byte offset
    d |= (uint64_t)1u << 46;                          // version
    d |= (uint64_t)2u << 61;                          // SWIZZLE_128B
    return d;
}

// Instruction descriptor: s32 accumulator, u8 x u8, both K-major, M=128, N=256.
constexpr uint32_t kIdescI8 = (2u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(kGemmN >> 3) << 17) |
                              ((uint32_t)(kGemmM >> 4) << 24);

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok) : "r"(bar), "r"(parity) : "memory");
    return ok != 0;
}

// Bounded wait; returns false (and records it) if the barrier never flips.
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t bar, uint32_t parity, int* err, int limit = 1 << 22) {
    for (int i = 0; i < limit; i++)
        if (mbar_try_wait(bar, parity)) return true;
    atomicOr(err, 1);
    return false;
}

// Polls of a wait that the stall test hook (bm_test_stall) makes run out.
constexpr int kStallPolls = 1 << 12;

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(dst), "l"(src) : "memory");
}

// Stage one K-chunk of the A (128 rows) and B (256 rows) tiles: row r's
// 16-byte chunk c goes to r*128 + ((c ^ (r & 7)) * 16) -- the 128-byte swizzle.
__device__ __forceinline__ void load_stage(uint32_t sA, uint32_t sB, const uint8_t* __restrict__ A,
                                           const uint8_t* __restrict__ B, int K, int a0, int b0, int kc,
                                           int tid) {
    const size_t koff = (size_t)kc * kGemmKC;
    for (int i = tid; i < kGemmM * 8; i += kGemmThreads) {
        const int r = i >> 3, c = i & 7;
        cp_async16(sA + r * 128 + ((c ^ (r & 7)) << 4), A + (size_t)(a0 + r) * K + koff + c * 16);
    }
    for (int i = tid; i < kGemmN * 8; i += kGemmThreads) {
        const int r = i >> 3, c = i & 7;
        cp_async16(sB + r * 128 + ((c ^ (r & 7)) << 4), B + (size_t)(b0 + r) * K + koff + c * 16);
    }
}

// One 128x256 tile of S_H per CTA, written into S (rows a < n, cols b < n).
// A: Mpad x K, B: Npad x K, both row-major u8 (K-major); K a multiple of 128.
static __global__ void __launch_bounds__(kGemmThreads, 1)
k_hub_gemm(const uint8_t* __restrict__ A, const uint8_t* __restrict__ B, int K, int n,
           int* __restrict__ S, int* __restrict__ err, int stall) {
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;                    // 1024-aligned stages
    const uint32_t bars = base + kGemmStages * kGemmStageBytes;       // kGemmStages mbarriers
    const uint32_t tslot = bars + 8 * kGemmStages;                    // TMEM base address
    uint32_t* tslot_ptr = reinterpret_cast<uint32_t*>(smem_raw + (tslot - raw));
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    const int b0 = blockIdx.x * kGemmN, a0 = blockIdx.y * kGemmM;
    const int KC = K / kGemmKC;

    if (wid == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(tslot), "r"(kGemmN) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < kGemmStages; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bars + 8 * s) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot_ptr;
    bool ok = true;

    // prologue: chunks 0 .. S-2
    for (int s = 0; s < kGemmStages - 1; s++) {
        if (s < KC) load_stage(base + s * kGemmStageBytes, base + s * kGemmStageBytes + kGemmM * kGemmKC,
                               A, B, K, a0, b0, s, tid);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kc = 0; kc < KC; kc++) {
        const int nxt = kc + kGemmStages - 1;
        if (nxt < KC) {
            const int st = nxt % kGemmStages;
            if (kc >= 1) {  // stage st was last read by chunk kc-1's MMAs
                const int prev = kc - 1;
                ok = ok && mbar_wait_bounded(bars + 8 * (prev % kGemmStages), (prev / kGemmStages) & 1, err);
            }
            load_stage(base + st * kGemmStageBytes, base + st * kGemmStageBytes + kGemmM * kGemmKC,
                       A, B, K, a0, b0, nxt, tid);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group %0;" :: "n"(kGemmStages - 1) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && ok) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int st = kc % kGemmStages;
            const uint32_t sa = base + st * kGemmStageBytes, sb = sa + kGemmM * kGemmKC;
#pragma unroll
            for (int j = 0; j < kGemmKC / 32; j++) {
                const uint64_t da = umma_desc_sw128(sa + j * 32), db = umma_desc_sw128(sb + j * 32);
                const uint32_t acc = (kc > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                    :: "r"(tmem), "l"(da), "l"(db), "r"(kIdescI8), "r"(acc) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(bars + 8 * st) : "memory");
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    // the last commit tracks every earlier MMA of the tile
    if (KC > 0) {
        const int last = KC - 1;
        ok = ok && mbar_wait_bounded(bars + 8 * (last % kGemmStages), (last / kGemmStages) & 1, err);
        // test hook: with every MMA of the tile complete, tile (0,0) also waits
        // for the barrier's next phase, which no commit ever completes
        if (stall && blockIdx.x == 0 && blockIdx.y == 0)
            ok = ok && mbar_wait_bounded(bars + 8 * (last % kGemmStages), ((last / kGemmStages) + 1) & 1, err,
                                         kStallPolls);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w owns TMEM lanes (tile rows) 32w .. 32w+31
    const int a = a0 + wid * 32 + lane;
    for (int cb = 0; cb < kGemmN / 32; cb++) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(wid * 32) << 16) + (uint32_t)(cb * 32);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
            "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
              "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
              "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (ok && a < n) {
            int* row = S + (size_t)a * n;
            const int c0 = b0 + cb * 32;
            if ((n & 3) == 0 && c0 + 32 <= n) {
                int4* d4 = reinterpret_cast<int4*>(row + c0);
#pragma unroll
                for (int q = 0; q < 8; q++)
                    d4[q] = make_int4((int)r[4 * q], (int)r[4 * q + 1], (int)r[4 * q + 2], (int)r[4 * q + 3]);
            } else {
                for (int q = 0; q < 32; q++)
                    if (c0 + q < n) row[c0 + q] = (int)r[q];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (wid == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kGemmN) : "memory");
}

// ---------------------------------------------------------------------------
// Operand builders.
// A[a][h*T+t-1] = number of G1 entries u_h -> a with weight >= t (rows sorted,
// so repeated entries are adjacent; the first of a run writes the counts).
template <bool W16>
__global__ void k_hub_build_A(DevView<W16> g, const int* __restrict__ hubs, int nh, int K,
                              uint8_t* __restrict__ A) {
    typedef Ent<W16> EN;
    for (int h = blockIdx.x; h < nh; h += gridDim.x) {
        const int u = hubs[h];
        const int s0 = g.off1o[u], s1 = g.off1o[u + 1];
        for (int i = s0 + threadIdx.x; i < s1; i += blockDim.x) {
            const int a = EN::id(g.ent1o[i]);
            if (i > s0 && EN::id(g.ent1o[i - 1]) == a) continue;
            int cnt[kHubT];
            for (int t = 0; t < kHubT; t++) cnt[t] = 0;
            for (int j = i; j < s1 && EN::id(g.ent1o[j]) == a; j++) {
                const int w = EN::w(g.ent1o[j]);
                for (int t = 0; t < kHubT; t++) cnt[t] += (w >= t + 1);
            }
            for (int t = 0; t < kHubT; t++) A[(size_t)a * K + h * kHubT + t] = (uint8_t)min(cnt[t], 255);
        }
    }
}

// B[b][h*T+t-1] = [W2[p u_h][p b] >= t], from the relabelled G2 out-list of p(u_h).
template <bool W16>
__global__ void k_hub_build_B(DevView<W16> g, const int* __restrict__ hubs, int nh, int K,
                              uint8_t* __restrict__ B) {
    typedef Ent<W16> EN;
    // hub h's list is split over gridDim.y blocks; a row's kHubT = 8 threshold
    // bytes go out as one 8-byte store
    static_assert(kHubT == 8, "one 64-bit store per entry");
    for (int h = blockIdx.x; h < nh; h += gridDim.x) {
        const int f = g.p[hubs[h]];
        const int s0 = g.off2o[f], s1 = g.off2o[f + 1];  // f == n (unmatched): empty
        for (int i = s0 + blockIdx.y * blockDim.x + threadIdx.x; i < s1; i += gridDim.y * blockDim.x) {
            const typename EN::T e = g.ent2oP[i];
            const int b = EN::id(e), w = EN::w(e);
            if (b >= g.n) continue;  // image without a preimage
            unsigned long long v = 0;
#pragma unroll
            for (int t = 0; t < kHubT; t++) v |= (unsigned long long)(w >= t + 1) << (8 * t);
            *reinterpret_cast<unsigned long long*>(B + (size_t)b * K + h * kHubT) = v;
        }
    }
}

}  // namespace bm
