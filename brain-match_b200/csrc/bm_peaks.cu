// bm_peaks.cu -- microbenchmarks for the roofline denominators of the sweep.
//
// The profit-row kernel is bound neither by HBM nor by tensor cores: each
// nonzero min term is one shared-memory atomic add at a data-dependent
// address of an (n+1)-int row.  bm_measure_peaks times, on the current
// device, (1) that access pattern at full occupancy with no global traffic
// (random addresses over an n-int shared array, 3 CTAs x 512 threads per SM,
// like the profit kernel, two integer operations of address arithmetic per
// atomic) and (2) independent int32 min+add pairs, the operation count the
// dense formulation of the sweep is quoted in.
#include <cuda_runtime.h>
#include <cstdint>
#include "bm.h"

namespace {

__global__ void __launch_bounds__(512) k_peak_red(int n, int iters, unsigned seed, int* sink) {
    extern __shared__ int acc[];
    for (int i = threadIdx.x; i <= n; i += blockDim.x) acc[i] = 0;
    __syncthreads();
    // addresses uniform over the largest power of two <= n, from four
    // independent LCG streams: two integer operations per atomic, so the
    // shared-memory atomic unit (not the address arithmetic) is what is timed
    int lg = 0;
    while ((2 << lg) <= n) lg++;
    const unsigned sh = 32u - (unsigned)lg;
    unsigned x0 = seed ^ (blockIdx.x * 9781u + threadIdx.x * 6271u), x1 = x0 * 3u + 1u, x2 = x0 * 5u + 7u,
             x3 = x0 * 9u + 3u;
    for (int it = 0; it < iters; it++) {
        x0 = x0 * 1664525u + 1013904223u;
        x1 = x1 * 1664525u + 1013904223u;
        x2 = x2 * 1664525u + 1013904223u;
        x3 = x3 * 1664525u + 1013904223u;
        atomicAdd(&acc[x0 >> sh], 1);
        atomicAdd(&acc[x1 >> sh], 2);
        atomicAdd(&acc[x2 >> sh], 3);
        atomicAdd(&acc[x3 >> sh], 4);
    }
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(sink, acc[blockIdx.x % n]);
}

__global__ void __launch_bounds__(512) k_peak_minadd(int iters, int* sink) {
    int w = threadIdx.x + 1, v[8], s[8];
    for (int k = 0; k < 8; k++) { v[k] = (blockIdx.x * 131 + k * 17 + threadIdx.x) & 1023; s[k] = 0; }
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) { s[k] += min(w, v[k]); v[k] ^= s[k] & 7; }
    }
    int t = 0;
    for (int k = 0; k < 8; k++) t += s[k];
    if (t == 0x7fffffff) *sink = t;
}

}  // namespace

extern "C" bm_status bm_measure_peaks(int32_t n, double* red_per_s, double* minadd_per_s) {
    if (n < 64 || n > 56000 || !red_per_s || !minadd_per_s) return BM_E_INPUT;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return BM_E_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return BM_E_CUDA;
    int* sink = nullptr;
    cudaEvent_t e0, e1;
    if (cudaMalloc(&sink, sizeof(int)) != cudaSuccess) return BM_E_CUDA;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const size_t smem = (size_t)(n + 1) * sizeof(int);
    cudaFuncSetAttribute(k_peak_red, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_peak_red, 512, smem);
    if (per_sm < 1) per_sm = 1;
    const int blocks = sms * per_sm, iters = 4096;
    float best = 1e30f, ms = 0;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        k_peak_red<<<blocks, 512, smem>>>(n, iters, 12345u + rep, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep && ms < best) best = ms;
    }
    *red_per_s = (double)blocks * 512 * iters * 4 / (best / 1e3);
    best = 1e30f;
    const int mblocks = sms * 4, miters = 8192;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        k_peak_minadd<<<mblocks, 512>>>(miters, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep && ms < best) best = ms;
    }
    // one min + one add per term (the xor keeps the chains honest and is not counted)
    *minadd_per_s = (double)mblocks * 512 * miters * 8 / (best / 1e3);
    cudaError_t err = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return err == cudaSuccess ? BM_OK : BM_E_CUDA;
}
