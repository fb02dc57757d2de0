// bm_hub_ws.cuh -- the hub GEMM as a persistent, warp-specialised kernel.
//
// Same product as k_hub_gemm (bm_hub.cuh): S[a][b] = sum_k A[a][k] B[b][k]
// over u8 operands, exact s32 accumulation.  The operands (K = 1,024 bytes a
// row) come from L2 once per tile, and with 128 x 256 tiles those re-reads
// (4 GB at N = 18,524) bound the kernel; a 256 x 256 tile reads each B chunk
// once for two 128-row MMAs, a third less operand traffic per output.
// One CTA per SM walks tiles blockIdx.x, blockIdx.x + gridDim.x, ... with
// three roles:
//   warp 0 (one lane)   TMA producer: cp.async.bulk.tensor of the A (256 x 128 B)
//                       and B (256 x 128 B) K-chunks into a kWsStages-deep ring,
//                       128-byte swizzle (the layout the MMA descriptors expect),
//                       running ahead into the next tile;
//   warp 1 (one lane)   MMA issuer: per K-chunk 4 tcgen05.mma kind::i8 for each
//                       128-row half into its TMEM accumulator (2 x 256 columns),
//                       a commit per chunk frees its stage, a commit per tile
//                       hands the accumulators to the epilogue;
//   warps 2-5           epilogue: tcgen05.ld of their TMEM lane quarter of both
//                       halves, stores into S, then release the accumulators.
// The tensor maps cover this GPU's own operand buffers; no load is multicast.
//
// Every wait is bounded.  A role whose wait runs out sets bit 0 of err and the
// CTA's abort word; the other roles see the word in their own waits and stop.
// Before the CTA exits, thread 0 waits (bounded) for the copies it issued and
// the MMA thread for its last commit, and warp 1 frees the TMEM.
#pragma once
#include <cstdint>
#include <cuda.h>
#include "bm_hub.cuh"

namespace bm {

constexpr int kWsM = 2 * kGemmM;                             // 256 tile rows: two MMA halves
constexpr int kWsStages = 3;
constexpr int kWsABytes = kWsM * kGemmKC;                    // 32 KB
constexpr int kWsStageBytes = (kWsM + kGemmN) * kGemmKC;     // 64 KB
constexpr int kWsThreads = 192;                              // 6 warps
constexpr int kWsEpiThreads = 128;                           // warps 2-5
constexpr int kWsEpiStride = 33;                             // padded 32 x 32 transpose block per warp
constexpr int kWsEpiBytes = 4 * 32 * kWsEpiStride * 4;
constexpr int kWsSmem = kWsStages * kWsStageBytes + kWsEpiBytes + 1024 + 256;
constexpr int kWsTmemCols = 2 * kGemmN;                      // one accumulator per half

struct WsShared {                 // at the end of the stage ring
    unsigned long long full[kWsStages], empty[kWsStages], tfull, tempty;
    uint32_t tmem;
    int abort;
    int issued[kWsStages];        // parity of the last fill issued into each stage, -1 none
    int last_bar, last_par;       // the MMA thread's last commit (barrier index, parity), -1 none
};

__device__ __forceinline__ bool ws_wait(uint32_t bar, uint32_t parity, volatile int* abort, int limit) {
    for (int i = 0; i < limit; i++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((i & 63) == 63 && *abort) return false;
    }
    return false;
}

__device__ __forceinline__ void ws_fail(volatile int* abort, int* err) {
    *abort = 1;
    atomicOr(err, 1);
}

static __global__ void __launch_bounds__(kWsThreads, 1)
k_hub_gemm_ws(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, int K, int n,
              int mtiles, int ntiles, int* __restrict__ S, int* __restrict__ err, int stall) {
    extern __shared__ uint8_t ws_raw[];
    const uint32_t raw = smem_u32(ws_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    int* epi = reinterpret_cast<int*>(ws_raw + (base - raw) + kWsStages * kWsStageBytes);
    WsShared* sh = reinterpret_cast<WsShared*>(ws_raw + (base - raw) + kWsStages * kWsStageBytes + kWsEpiBytes);
    volatile int* abort = &sh->abort;
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    const int KC = K / kGemmKC;
    const int tiles = mtiles * ntiles;
    const uint32_t fullb = smem_u32(&sh->full[0]), emptyb = smem_u32(&sh->empty[0]);
    const uint32_t tfullb = smem_u32(&sh->tfull), temptyb = smem_u32(&sh->tempty);
    constexpr int kLimit = 1 << 22;

    if (tid == 0) {
        for (int s = 0; s < kWsStages; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(fullb + 8 * s) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(emptyb + 8 * s) : "memory");
            sh->issued[s] = -1;
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(tfullb) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(temptyb), "r"(kWsEpiThreads) : "memory");
        sh->abort = 0;
        sh->last_bar = -1;
        sh->last_par = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    if (wid == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_u32(&sh->tmem)), "r"(kWsTmemCols) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = sh->tmem;

    if (wid == 0) {
        if (lane == 0) {   // ---- TMA producer ----
            int s = 0;
            uint32_t ph = 0;
            for (int t = blockIdx.x; t < tiles && !*abort; t += gridDim.x) {
                const int a0 = (t / ntiles) * kWsM, b0 = (t % ntiles) * kGemmN;
                for (int kc = 0; kc < KC; kc++) {
                    if (!ws_wait(emptyb + 8 * s, ph ^ 1u, abort, kLimit)) { ws_fail(abort, err); break; }
                    const uint32_t sa = base + s * kWsStageBytes, fb = fullb + 8 * s;
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;"
                                 :: "r"(fb), "r"(kWsStageBytes) : "memory");
                    asm volatile(
                        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
                        " [%0], [%1, {%2, %3}], [%4];"
                        :: "r"(sa), "l"(&tmA), "r"(kc * kGemmKC), "r"(a0), "r"(fb) : "memory");
                    asm volatile(
                        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes"
                        " [%0], [%1, {%2, %3}], [%4];"
                        :: "r"(sa + kWsABytes), "l"(&tmB), "r"(kc * kGemmKC), "r"(b0), "r"(fb) : "memory");
                    sh->issued[s] = (int)ph;
                    if (++s == kWsStages) { s = 0; ph ^= 1u; }
                }
            }
        }
    } else if (wid == 1) {
        if (lane == 0) {   // ---- MMA issuer ----
            int s = 0;
            uint32_t ph = 0, aph = 0;
            for (int t = blockIdx.x; t < tiles && !*abort; t += gridDim.x) {
                if (!ws_wait(temptyb, aph ^ 1u, abort, kLimit)) { ws_fail(abort, err); break; }
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                bool ok = true;
                for (int kc = 0; kc < KC; kc++) {
                    if (!ws_wait(fullb + 8 * s, ph, abort, kLimit)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = base + s * kWsStageBytes, sb = sa + kWsABytes;
#pragma unroll
                    for (int h = 0; h < 2; h++) {   // rows 128 h .. 128 h + 127 into columns 256 h ..
#pragma unroll
                        for (int j = 0; j < kGemmKC / 32; j++) {
                            const uint64_t da = umma_desc_sw128(sa + h * kGemmM * kGemmKC + j * 32);
                            const uint64_t db = umma_desc_sw128(sb + j * 32);
                            const uint32_t accum = (kc > 0 || j > 0) ? 1u : 0u;
                            asm volatile(
                                "{\n\t.reg .pred p;\n\t"
                                "setp.ne.b32 p, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}"
                                :: "r"(tmem + (uint32_t)(h * kGemmN)), "l"(da), "l"(db), "r"(kIdescI8), "r"(accum)
                                : "memory");
                        }
                    }
                    // the stage is free once these MMAs have read it
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                                 :: "r"(emptyb + 8 * s) : "memory");
                    sh->last_bar = s;
                    sh->last_par = (int)ph;
                    if (++s == kWsStages) { s = 0; ph ^= 1u; }
                }
                if (!ok) { ws_fail(abort, err); break; }
                // the accumulators are complete once every MMA above has finished
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                             :: "r"(tfullb) : "memory");
                sh->last_bar = kWsStages;
                sh->last_par = (int)aph;
                aph ^= 1u;
            }
        }
    } else {               // ---- epilogue: warps 2-5, TMEM lane quarter wid % 4 ----
        const int q = wid & 3;
        int* blk = epi + q * 32 * kWsEpiStride;   // this warp's transpose block
        uint32_t aph = 0;
        bool first = true;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x) {
            bool ok = ws_wait(tfullb, aph, abort, kLimit);
            // test hook (bm_test_stall): CTA 0's first tile also waits for the
            // accumulators' next hand-over, which cannot come before they are released
            if (ok && stall && first && blockIdx.x == 0) ok = ws_wait(tfullb, aph ^ 1u, abort, kStallPolls);
            first = false;
            if (!ok) { ws_fail(abort, err); break; }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int a0 = (t / ntiles) * kWsM, b0 = (t % ntiles) * kGemmN;
            for (int hc = 0; hc < 2 * (kGemmN / 32); hc++) {   // half hc / 8, column block hc % 8
                const int h = hc >> 3, cb = hc & 7;
                const int a = a0 + h * kGemmM + q * 32 + lane;
                uint32_t r[32];
                const uint32_t taddr = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(h * kGemmN + cb * 32);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                    "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
                      "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
                      "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]),
                      "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]),
                      "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                    : "r"(taddr));
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                // lane l holds row l of the warp's 32 x 32 block; through shared
                // memory each store then writes four rows' 128-byte segments
                // (lane l: row 4j + l / 8, columns 4 (l % 8) ..) instead of 32 rows'
                // 16-byte pieces
#pragma unroll
                for (int u = 0; u < 32; u++) blk[lane * kWsEpiStride + u] = (int)r[u];
                __syncwarp();
                const int c0 = b0 + cb * 32, cl = 4 * (lane & 7);
                const bool full = (n & 3) == 0 && c0 + 32 <= n;
#pragma unroll
                for (int jr = 0; jr < 8; jr++) {
                    const int rl = 4 * jr + (lane >> 3), ar = a - lane + rl;   // ar: that row's vertex
                    const int* src = blk + rl * kWsEpiStride + cl;
                    if (ar < n) {
                        int* dst = S + (size_t)ar * n + c0 + cl;
                        if (full) *reinterpret_cast<int4*>(dst) = make_int4(src[0], src[1], src[2], src[3]);
                        else
                            for (int u = 0; u < 4; u++)
                                if (c0 + cl + u < n) dst[u] = src[u];
                    }
                }
                __syncwarp();
            }
            // this thread's reads of the accumulators are done
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(temptyb) : "memory");
            aph ^= 1u;
        }
    }
    __syncwarp();
    __syncthreads();
    if (*abort) {
        // nothing of this CTA may still be writing its shared memory or TMEM
        if (tid == 0)
            for (int s = 0; s < kWsStages; s++)
                if (sh->issued[s] >= 0)
                    for (int i = 0; i < kLimit; i++)
                        if (mbar_try_wait(fullb + 8 * s, (uint32_t)sh->issued[s])) break;
        if (tid == 32 && sh->last_bar >= 0) {
            const uint32_t lb = sh->last_bar < kWsStages ? emptyb + 8 * sh->last_bar : tfullb;
            for (int i = 0; i < kLimit; i++)
                if (mbar_try_wait(lb, (uint32_t)sh->last_par)) break;
        }
        __syncthreads();
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (wid == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kWsTmemCols) : "memory");
}

}  // namespace bm
