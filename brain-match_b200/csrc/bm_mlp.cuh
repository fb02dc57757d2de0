// bm_mlp.cuh -- device code of the learned swap-proposal network.
//
// MLP 128 -> 256 -> 256 -> 1 (ReLU), bf16 weights and activations, fp32
// accumulation.  The two wide layers and every backward GEMM run through one
// tcgen05 kernel, C = A * B^T with A (M x K) and B (N x K) bf16 row-major
// (K-major) and C fp32, accumulated in TMEM (kind::f16, bf16 inputs); the same
// shared-memory staging and 128-byte swizzle as the hub GEMM.  The 256 -> 1
// head, bias/ReLU backward, loss and SGD are small CUDA-core kernels.
// Ranking many pairs uses a second, fused kernel (k_mlp_rank, below).
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include "bm_hub.cuh"

namespace bm {

constexpr int kMlpIn = 128, kMlpHid = 256;

// C[M x N] (+ bias[col]) (ReLU) = A[M x K] * B[N x K]^T; M % 128 == 0,
// N % BN == 0, K % 64 == 0.  Optional bf16 copy of the result.
template <int BN>
static __global__ void __launch_bounds__(kGemmThreads, 1)
k_gemm_bf16(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B, int M, int N, int K,
            float* __restrict__ C, const float* __restrict__ bias, int relu, __nv_bfloat16* __restrict__ Cb,
            int* __restrict__ err, int stall) {
    constexpr int kStage = (kGemmM + BN) * kGemmKC;                   // bytes per stage
    constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) |  // f32 accum, bf16 x bf16
                                ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(kGemmM >> 4) << 24);
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t bars = base + kGemmStages * kStage;
    const uint32_t tslot = bars + 8 * kGemmStages;
    uint32_t* tslot_ptr = reinterpret_cast<uint32_t*>(smem_raw + (tslot - raw));
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    const int b0 = blockIdx.x * BN, a0 = blockIdx.y * kGemmM;
    const int KB = K * 2;                        // bytes per row
    const int KC = KB / kGemmKC;                 // 128-byte chunks
    const uint8_t* Ab = reinterpret_cast<const uint8_t*>(A);
    const uint8_t* Bb = reinterpret_cast<const uint8_t*>(B);

    if (wid == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(tslot), "r"(BN) : "memory");
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

    auto load = [&](int st, int kc) {
        const uint32_t sA = base + st * kStage, sB = sA + kGemmM * kGemmKC;
        const size_t koff = (size_t)kc * kGemmKC;
        for (int i = tid; i < kGemmM * 8; i += kGemmThreads) {
            const int r = i >> 3, c = i & 7;
            cp_async16(sA + r * 128 + ((c ^ (r & 7)) << 4), Ab + (size_t)(a0 + r) * KB + koff + c * 16);
        }
        for (int i = tid; i < BN * 8; i += kGemmThreads) {
            const int r = i >> 3, c = i & 7;
            cp_async16(sB + r * 128 + ((c ^ (r & 7)) << 4), Bb + (size_t)(b0 + r) * KB + koff + c * 16);
        }
    };
    for (int s = 0; s < kGemmStages - 1; s++) {
        if (s < KC) load(s, s);
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    for (int kc = 0; kc < KC; kc++) {
        const int nxt = kc + kGemmStages - 1;
        if (nxt < KC) {
            if (kc >= 1) {
                const int prev = kc - 1;
                ok = ok && mbar_wait_bounded(bars + 8 * (prev % kGemmStages), (prev / kGemmStages) & 1, err);
            }
            load(nxt % kGemmStages, nxt);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group %0;" :: "n"(kGemmStages - 1) : "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0 && ok) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const int st = kc % kGemmStages;
            const uint32_t sa = base + st * kStage, sb = sa + kGemmM * kGemmKC;
#pragma unroll
            for (int j = 0; j < kGemmKC / 32; j++) {  // 16 bf16 = 32 bytes of K per MMA
                const uint64_t da = umma_desc_sw128(sa + j * 32), db = umma_desc_sw128(sb + j * 32);
                const uint32_t acc = (kc > 0 || j > 0) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                    :: "r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(acc) : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(bars + 8 * st) : "memory");
        }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (KC > 0) {
        const int last = KC - 1;
        ok = ok && mbar_wait_bounded(bars + 8 * (last % kGemmStages), (last / kGemmStages) & 1, err);
        // test hook (bm_test_stall): the barrier's next phase never completes
        if (stall && blockIdx.x == 0 && blockIdx.y == 0)
            ok = ok && mbar_wait_bounded(bars + 8 * (last % kGemmStages), ((last / kGemmStages) + 1) & 1, err,
                                         kStallPolls);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const int row = a0 + wid * 32 + lane;
    for (int cb = 0; cb < BN / 32; cb++) {
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
        if (ok && row < M) {
            const int c0 = b0 + cb * 32;
            float v[32];
#pragma unroll
            for (int q = 0; q < 32; q++) {
                float x = __uint_as_float(r[q]);
                if (bias) x += bias[c0 + q];
                if (relu) x = fmaxf(x, 0.f);
                v[q] = x;
            }
            if (C) {
                float4* d4 = reinterpret_cast<float4*>(C + (size_t)row * N + c0);
#pragma unroll
                for (int q = 0; q < 8; q++) d4[q] = make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
            if (Cb) {
                __nv_bfloat162* d2 = reinterpret_cast<__nv_bfloat162*>(Cb + (size_t)row * N + c0);
#pragma unroll
                for (int q = 0; q < 16; q++) d2[q] = __floats2bfloat162_rn(v[2 * q], v[2 * q + 1]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (wid == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(BN) : "memory");
}

template <int BN>
constexpr int gemm_bf16_smem() { return kGemmStages * (kGemmM + BN) * kGemmKC + 1024 + 256; }

// out[c][r] = in[r][c] for an R x C bf16 matrix.
static __global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, int R, int C,
                                        __nv_bfloat16* __restrict__ out) {
    __shared__ __nv_bfloat16 t[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        t[y][threadIdx.x] = (r < R && c < C) ? in[(size_t)r * C + c] : __float2bfloat16(0.f);
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (c < C && r < R) out[(size_t)c * R + r] = t[threadIdx.x][y];
    }
}

// Head and loss: y = H2 . w3 + b3 (rows < Bv valid), dy = 2 (y - t) / Bv,
// dH2 = dy w3 masked by ReLU'(H2) (bf16), dw3 += H2^T dy, db3 += sum dy.
// One warp per row.
static __global__ void k_head(const float* __restrict__ H2, int Bv, int Bpad, const float* __restrict__ w3,
                              const float* __restrict__ b3, float* __restrict__ y, const float* __restrict__ target,
                              float* __restrict__ loss, __nv_bfloat16* __restrict__ dH2, float* __restrict__ dw3,
                              float* __restrict__ db3) {
    const int lane = threadIdx.x & 31;
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (row >= Bpad) return;
    const float* h = H2 + (size_t)row * kMlpHid;
    float s = 0.f;
    for (int c = lane; c < kMlpHid; c += 32) s += h[c] * w3[c];
    for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const float out = s + b3[0];
    if (lane == 0 && y && row < Bv) y[row] = out;
    if (!target) return;
    const float dy = row < Bv ? 2.f * (out - target[row]) / (float)Bv : 0.f;
    if (lane == 0 && row < Bv) {
        atomicAdd(loss, (out - target[row]) * (out - target[row]) / (float)Bv);
        atomicAdd(db3, dy);
    }
    for (int c = lane; c < kMlpHid; c += 32) {
        const float hv = h[c];
        dH2[(size_t)row * kMlpHid + c] = __float2bfloat16(hv > 0.f ? dy * w3[c] : 0.f);
        if (dy != 0.f) atomicAdd(&dw3[c], hv * dy);
    }
}

// dH1 (fp32 from the GEMM) masked by ReLU'(H1), to bf16; db (column sums of
// the masked gradient) accumulated.
static __global__ void k_relu_bwd(const float* __restrict__ dH, const float* __restrict__ H, int rows, int cols,
                                  __nv_bfloat16* __restrict__ out, float* __restrict__ db) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float acc = 0.f;
    for (int r = blockIdx.y; r < rows; r += gridDim.y) {
        const float g = H[(size_t)r * cols + c] > 0.f ? dH[(size_t)r * cols + c] : 0.f;
        out[(size_t)r * cols + c] = __float2bfloat16(g);
        acc += g;
    }
    if (db) atomicAdd(&db[c], acc);
}

// Column sums of a bf16 gradient (bias gradient of the second hidden layer).
static __global__ void k_colsum_bf16(const __nv_bfloat16* __restrict__ G, int rows, int cols, float* __restrict__ out) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cols) return;
    float acc = 0.f;
    for (int r = blockIdx.y; r < rows; r += gridDim.y) acc += __bfloat162float(G[(size_t)r * cols + c]);
    atomicAdd(&out[c], acc);
}

// SGD on fp32 master weights, refreshing the bf16 copy: w -= lr * g, the
// product and the difference each rounded to nearest (no fused multiply-add),
// so the update is reproducible on any IEEE host.
static __global__ void k_sgd(float* __restrict__ w, const float* __restrict__ g, int count, float lr,
                             __nv_bfloat16* __restrict__ wb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float v = __fsub_rn(w[i], __fmul_rn(lr, g[i]));
    w[i] = v;
    if (wb) wb[i] = __float2bfloat16(v);
}

static __global__ void k_to_bf16(const float* __restrict__ x, int count, __nv_bfloat16* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) y[i] = __float2bfloat16(x[i]);
}

// ---------------------------------------------------------------------------
// Ranking many pairs (inference), factorised.  The first layer is linear in
// the concatenated input x = [f1(a), f1(b), f2(p a), f2(p b)], so
// W1 x + b1 = U[a] + V[b] with per-vertex vectors
//   U[a] = b1 + W1[:, 0:32] f1(a) + W1[:, 64:96]  f2(p a)
//   V[b] =      W1[:, 32:64] f1(b) + W1[:, 96:128] f2(p b)
// (bf16-rounded weights and features, fp32 sums -- the values the GEMM path
// multiplies).  One persistent kernel then scores every pair: the CTA keeps
// W2 (bf16, 128 KB) resident in shared memory, builds each 128-pair A tile
// bf16(relu(U[a] + V[b])) directly in the swizzled operand layout, runs one
// 128 x 256 x 256 tcgen05 MMA into TMEM, and its epilogue applies b2, ReLU
// and the 256 -> 1 head, writing one float per pair.

constexpr int kFeatDim = 32;

// U and V for n vertices: block of 256 threads (one per hidden unit), 8
// vertices per block.  F1, F2: n x 32 fp32; W1b: 256 x 128 bf16; p: matching.
static __global__ void __launch_bounds__(256) k_uv(const float* __restrict__ F1, const float* __restrict__ F2,
                                                   const int* __restrict__ p, int n,
                                                   const __nv_bfloat16* __restrict__ W1b,
                                                   const float* __restrict__ b1, float* __restrict__ U,
                                                   float* __restrict__ V) {
    __shared__ float f[8][2][kFeatDim];  // per vertex: f1, f2(p), as bf16-rounded floats
    const int c = threadIdx.x;
    const int v0 = blockIdx.x * 8;
    for (int i = c; i < 8 * 2 * kFeatDim; i += 256) {
        const int v = i / (2 * kFeatDim), k = i % (2 * kFeatDim), a = v0 + v;
        float x = 0.f;
        if (a < n) {
            if (k < kFeatDim) x = F1[(size_t)a * kFeatDim + k];
            else {
                const int img = p[a];
                x = img < n ? F2[(size_t)img * kFeatDim + (k - kFeatDim)] : 0.f;
            }
        }
        f[v][k < kFeatDim ? 0 : 1][k & (kFeatDim - 1)] = __bfloat162float(__float2bfloat16(x));
    }
    __syncthreads();
    float w[4][kFeatDim];  // W1[c] in four 32-column quarters: f1(a), f1(b), f2(pa), f2(pb)
#pragma unroll
    for (int q = 0; q < 4; q++)
#pragma unroll
        for (int k = 0; k < kFeatDim; k++) w[q][k] = __bfloat162float(W1b[(size_t)c * kMlpIn + q * kFeatDim + k]);
    const float bias = b1[c];
    for (int v = 0; v < 8; v++) {
        const int a = v0 + v;
        if (a >= n) break;
        float u = 0.f, x = 0.f;
#pragma unroll
        for (int k = 0; k < kFeatDim; k++) {
            u = fmaf(w[0][k], f[v][0][k], u);
            x = fmaf(w[1][k], f[v][0][k], x);
        }
#pragma unroll
        for (int k = 0; k < kFeatDim; k++) {
            u = fmaf(w[2][k], f[v][1][k], u);
            x = fmaf(w[3][k], f[v][1][k], x);
        }
        U[(size_t)a * kMlpHid + c] = u + bias;
        V[(size_t)a * kMlpHid + c] = x;
    }
}

constexpr int kRankThreads = 256;
constexpr int kRankA = kGemmM * 512;          // A tile: 128 rows x 256 bf16 (4 k-blocks of 16 KB)
constexpr int kRankB = kMlpHid * 512;         // W2: 256 rows x 256 bf16 (4 k-blocks of 32 KB)
constexpr int kRankSmem = kRankA + kRankB + 2 * kMlpHid * 4 + 1024 + 256;

// y[i] = w3 . relu(W2 relu(U[pa i] + V[pb i]) + b2) + b3 for i < k.
static __global__ void __launch_bounds__(kRankThreads, 1)
k_mlp_rank(const float* __restrict__ U, const float* __restrict__ V, const int* __restrict__ pa,
           const int* __restrict__ pb, long long k, const __nv_bfloat16* __restrict__ W2b,
           const float* __restrict__ b2, const float* __restrict__ w3, const float* __restrict__ b3,
           float* __restrict__ y, int* __restrict__ err) {
    constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kMlpHid >> 3) << 17) |
                                ((uint32_t)(kGemmM >> 4) << 24);
    extern __shared__ uint8_t smem_raw[];
    const uint32_t raw = smem_u32(smem_raw);
    const uint32_t base = (raw + 1023u) & ~1023u;
    const uint32_t sA = base, sB = base + kRankA;
    float* sb2 = reinterpret_cast<float*>(smem_raw + (sB + kRankB - raw));
    float* sw3 = sb2 + kMlpHid;
    const uint32_t bar = sB + kRankB + 2 * kMlpHid * 4;
    const uint32_t tslot = bar + 8;
    uint32_t* tslot_ptr = reinterpret_cast<uint32_t*>(smem_raw + (tslot - raw));
    __shared__ int s_abort;
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;

    if (wid == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(tslot), "r"(kMlpHid) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(bar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
    }
    // W2 resident: row r (output unit), 16-byte chunk c of its 512 bytes
    const uint8_t* W2 = reinterpret_cast<const uint8_t*>(W2b);
    for (int i = tid; i < kMlpHid * 32; i += kRankThreads) {
        const int r = i >> 5, c = i & 31, kb = c >> 3, cc = c & 7;
        const uint4 v = *reinterpret_cast<const uint4*>(W2 + (size_t)r * 512 + c * 16);
        const uint32_t dst = sB + kb * (kMlpHid * 128) + r * 128 + ((cc ^ (r & 7)) << 4);
        asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" :: "r"(dst), "r"(v.x), "r"(v.y), "r"(v.z), "r"(v.w) : "memory");
    }
    for (int i = tid; i < kMlpHid; i += kRankThreads) { sb2[i] = b2[i]; sw3[i] = w3[i]; }
    const float bias3 = b3[0];
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = *tslot_ptr;

    const long long tiles = (k + kGemmM - 1) / kGemmM;
    uint32_t phase = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x) {
        const long long row0 = t * kGemmM;
        // A tile: warp w builds rows w, w + 8, ... (four rows per pass, their
        // loads all issued before any store); lane = 16-byte chunk (8 units)
        for (int r0 = wid; r0 < kGemmM; r0 += 4 * (kRankThreads / 32)) {
            float4 u[4][2], x[4][2];
            bool live[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int r = r0 + q * (kRankThreads / 32);
                const long long i = row0 + r;
                live[q] = i < k;
                if (live[q]) {
                    const int a = pa[i], b = pb[i];
                    const float4* u4 = reinterpret_cast<const float4*>(U + (size_t)a * kMlpHid + lane * 8);
                    const float4* v4 = reinterpret_cast<const float4*>(V + (size_t)b * kMlpHid + lane * 8);
                    u[q][0] = u4[0]; u[q][1] = u4[1]; x[q][0] = v4[0]; x[q][1] = v4[1];
                }
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int r = r0 + q * (kRankThreads / 32);
                uint4 out = make_uint4(0, 0, 0, 0);
                if (live[q]) {
                    const float4 u0 = u[q][0], u1 = u[q][1], x0 = x[q][0], x1 = x[q][1];
                    __nv_bfloat162 h0 = __floats2bfloat162_rn(fmaxf(u0.x + x0.x, 0.f), fmaxf(u0.y + x0.y, 0.f));
                    __nv_bfloat162 h1 = __floats2bfloat162_rn(fmaxf(u0.z + x0.z, 0.f), fmaxf(u0.w + x0.w, 0.f));
                    __nv_bfloat162 h2 = __floats2bfloat162_rn(fmaxf(u1.x + x1.x, 0.f), fmaxf(u1.y + x1.y, 0.f));
                    __nv_bfloat162 h3 = __floats2bfloat162_rn(fmaxf(u1.z + x1.z, 0.f), fmaxf(u1.w + x1.w, 0.f));
                    out.x = *reinterpret_cast<uint32_t*>(&h0);
                    out.y = *reinterpret_cast<uint32_t*>(&h1);
                    out.z = *reinterpret_cast<uint32_t*>(&h2);
                    out.w = *reinterpret_cast<uint32_t*>(&h3);
                }
                const int kb = lane >> 3, cc = lane & 7;
                const uint32_t dst = sA + kb * (kGemmM * 128) + r * 128 + ((cc ^ (r & 7)) << 4);
                asm volatile("st.shared.v4.b32 [%0], {%1,%2,%3,%4};" :: "r"(dst), "r"(out.x), "r"(out.y), "r"(out.z), "r"(out.w) : "memory");
            }
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
            for (int kb = 0; kb < 4; kb++)
#pragma unroll
                for (int j = 0; j < 4; j++) {  // 16 bf16 = 32 bytes of K per MMA
                    const uint64_t da = umma_desc_sw128(sA + kb * (kGemmM * 128) + j * 32);
                    const uint64_t db = umma_desc_sw128(sB + kb * (kMlpHid * 128) + j * 32);
                    const uint32_t acc = (kb | j) ? 1u : 0u;
                    asm volatile(
                        "{\n\t.reg .pred p;\n\t"
                        "setp.ne.b32 p, %4, 0;\n\t"
                        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                        :: "r"(tmem), "l"(da), "l"(db), "r"(kIdesc), "r"(acc) : "memory");
                }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                         :: "r"(bar) : "memory");
        }
        if (!mbar_wait_bounded(bar, phase, err)) s_abort = 1;
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (wid < 4) {  // epilogue: warp w reads TMEM lanes 32w..32w+31 = tile rows
            const long long i = row0 + wid * 32 + lane;
            float acc = 0.f;
            for (int cb = 0; cb < kMlpHid / 32; cb++) {
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
#pragma unroll
                for (int q = 0; q < 32; q++) {
                    const int c = cb * 32 + q;
                    acc = fmaf(fmaxf(__uint_as_float(r[q]) + sb2[c], 0.f), sw3[c], acc);
                }
            }
            if (i < k) y[i] = acc + bias3;
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        if (s_abort) break;
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (wid == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(kMlpHid) : "memory");
}

}  // namespace bm
