// bm_mlp.cu -- the learned swap-proposal network and the learned sweep.
//
// Per-vertex features (32 floats; G1 vertices in F1, G2 vertices in F2):
//   0 log1p out-degree   1 log1p in-degree    2 log1p out-weight sum
//   3 log1p in-weight sum 4 log1p 2-hop out count  5 log1p 2-hop in count
//   6 log1p max out weight 7 log1p max in weight  8 log1p self-loop weight
//   9 log1p current contribution (G2: of the G1 vertex matched to it)
//  10 contribution / (incident weight + 1); 11..31 zero;
// then z-scored per column over the vertices.  A pair (a,b) is
// [F1 a, F1 b, F2 p(a), F2 p(b)] (128 inputs); the target is
// sign(delta) log1p|delta| of its exact swap delta.
// Training samples come from the exact profit matrix of the current matching
// (each row's best partner plus candidate-pool partners); the learned sweep
// scores a pool of partners per vertex, evaluates the top-ranked ones exactly
// and commits them with the engine's exact set commit; when nothing improves
// it falls back to a full sweep.
#include <cstdio>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>
#include <numeric>
#include <random>
#include <cuda_runtime.h>
#include <cuda_bf16.h>
#include <cub/device/device_radix_sort.cuh>
#include "bm.h"
#include "bm_internal.cuh"
#include "bm_select.cuh"
#include "bm_triples.cuh"
#include "bm_mlp.cuh"

namespace {

constexpr int kFeat = 32;
// exhaustive sweeps of the learned paths keep the profit matrix exact across
// commits (updated from the moved vertices where that is cheaper): same moves
const bm_sweep_opts kIncremental = {0, -1, 0, 1, {0, 0, 0, 0}};
// parameter layout (fp32): W1[256x128] b1[256] W2[256x256] b2[256] w3[256] b3[1]
constexpr int oW1 = 0, oB1 = oW1 + kMlpHid * kMlpIn, oW2 = oB1 + kMlpHid, oB2 = oW2 + kMlpHid * kMlpHid,
              oW3 = oB2 + kMlpHid, oB3 = oW3 + kMlpHid, kParams = oB3 + 1;

// ---- features ----
template <bool W16>
__global__ void k_contrib(DevView<W16> g, float* __restrict__ contrib) {
    typedef Ent<W16> EN;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < g.n; a += nw) {
        const int pa = g.p[a];
        long long s = 0;
        for (int i = g.off1o[a] + lane; i < g.off1o[a + 1]; i += 32) {
            const typename EN::T e = g.ent1o[i];
            s += imin(EN::w(e), g.w2(pa, g.p[EN::id(e)]));
        }
        for (int i = g.off1i[a] + lane; i < g.off1i[a + 1]; i += 32) {
            const typename EN::T e = g.ent1i[i];
            s += imin(EN::w(e), g.w2(g.p[EN::id(e)], pa));
        }
        for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            for (int q = g.offs[a]; q < g.offs[a + 1]; q++) s += imin(g.selfw[q], g.w2(pa, pa));
            contrib[a] = (float)s;
        }
    }
}

// Structural features of one graph (G1 lists if g2 == 0, else G2's): a warp
// per vertex.
template <bool W16>
__global__ void k_static_features(DevView<W16> g, int g2, float* __restrict__ F) {
    typedef Ent<W16> EN;
    const int lane = threadIdx.x & 31;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    const int* offo = g2 ? g.off2o : g.off1o;
    const int* offi = g2 ? g.off2i : g.off1i;
    const typename EN::T* eo = g2 ? g.ent2o : g.ent1o;
    const typename EN::T* ei = g2 ? g.ent2i : g.ent1i;
    for (int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; a < g.n; a += nw) {
        float wo = 0, wi = 0, h2o = 0, h2i = 0, mo = 0, mi = 0;
        for (int i = offo[a] + lane; i < offo[a + 1]; i += 32) {
            const int v = EN::id(eo[i]), w = EN::w(eo[i]);
            wo += w; mo = fmaxf(mo, (float)w); h2o += offo[v + 1] - offo[v];
        }
        for (int i = offi[a] + lane; i < offi[a + 1]; i += 32) {
            const int u = EN::id(ei[i]), w = EN::w(ei[i]);
            wi += w; mi = fmaxf(mi, (float)w); h2i += offi[u + 1] - offi[u];
        }
        for (int o = 16; o; o >>= 1) {
            wo += __shfl_xor_sync(0xffffffffu, wo, o); wi += __shfl_xor_sync(0xffffffffu, wi, o);
            h2o += __shfl_xor_sync(0xffffffffu, h2o, o); h2i += __shfl_xor_sync(0xffffffffu, h2i, o);
            mo = fmaxf(mo, __shfl_xor_sync(0xffffffffu, mo, o)); mi = fmaxf(mi, __shfl_xor_sync(0xffffffffu, mi, o));
        }
        float v = 0.f;
        switch (lane) {
            case 0: v = log1pf((float)(offo[a + 1] - offo[a])); break;
            case 1: v = log1pf((float)(offi[a + 1] - offi[a])); break;
            case 2: v = log1pf(wo); break;
            case 3: v = log1pf(wi); break;
            case 4: v = log1pf(h2o); break;
            case 5: v = log1pf(h2i); break;
            case 6: v = log1pf(mo); break;
            case 7: v = log1pf(mi); break;
            case 8: {
                float s = 0.f;
                if (!g2) for (int q = g.offs[a]; q < g.offs[a + 1]; q++) s += g.selfw[q];
                v = log1pf(s);
            } break;
            default: v = 0.f;
        }
        F[(size_t)a * kFeat + lane] = v;
    }
}

// Dynamic features 9, 10: current contribution (G2 side: of pinv(f)).
__global__ void k_dyn_features(const float* __restrict__ contrib, const int* __restrict__ pinv, int n,
                               float* __restrict__ F1, float* __restrict__ F2) {
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const float c = contrib[a];
    const float tot1 = expm1f(F1[(size_t)a * kFeat + 2]) + expm1f(F1[(size_t)a * kFeat + 3]);
    F1[(size_t)a * kFeat + 9] = log1pf(c);
    F1[(size_t)a * kFeat + 10] = c / (tot1 + 1.f);
    const int b = pinv[a];  // a read as a G2 vertex
    const float c2 = b < n ? contrib[b] : 0.f;
    const float tot2 = expm1f(F2[(size_t)a * kFeat + 2]) + expm1f(F2[(size_t)a * kFeat + 3]);
    F2[(size_t)a * kFeat + 9] = log1pf(c2);
    F2[(size_t)a * kFeat + 10] = c2 / (tot2 + 1.f);
}

// Column statistics of the features (block c: F1 column c for c < 32, F2
// column c - 32): mean and 1/std (population), 0 for a constant column.
__global__ void k_col_stats(const float* __restrict__ F1, const float* __restrict__ F2, int n,
                            float* __restrict__ mean, float* __restrict__ scale) {
    const int c = blockIdx.x;
    const float* F = c < kFeat ? F1 : F2;
    const int col = c & (kFeat - 1);
    double s = 0, q = 0;
    for (int a = threadIdx.x; a < n; a += blockDim.x) {
        const double v = F[(size_t)a * kFeat + col];
        s += v;
        q += v * v;
    }
    __shared__ double rs[32], rq[32];
    for (int o = 16; o; o >>= 1) { s += __shfl_xor_sync(0xffffffffu, s, o); q += __shfl_xor_sync(0xffffffffu, q, o); }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { rs[wid] = s; rq[wid] = q; }
    __syncthreads();
    if (threadIdx.x == 0) {
        s = 0; q = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { s += rs[w]; q += rq[w]; }
        const double mu = s / n, var = q / n - mu * mu;
        const double sd = var > 0 ? sqrt(var) : 0.0;
        mean[c] = (float)mu;
        scale[c] = sd > 1e-6 ? (float)(1.0 / sd) : 0.f;
    }
}

// F = (F - mean) * scale, column-wise (z-scores).
__global__ void k_normalise(float* __restrict__ F1, float* __restrict__ F2, int n, const float* __restrict__ mean,
                            const float* __restrict__ scale) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long half = (long long)n * kFeat;
    if (i >= 2 * half) return;
    const int c = (int)(i % kFeat) + (i < half ? 0 : kFeat);
    float* F = i < half ? F1 + i : F2 + (i - half);
    *F = (*F - mean[c]) * scale[c];
}

// Training batch: rows i < k take sample j = ((off + i) * mul + add) mod count,
// a permutation of the samples when gcd(mul, count) = 1.  Samples are laid out
// sweep-major, `per` to a sweep, and sweep s has its own features
// (F1s + s*n*32, F2s + s*n*32) and matching (ps + s*n).  X row i gets
// [F1 a, F1 b, F2 p(a), F2 p(b)] in bf16 (zero rows from k to kpad), t[i]
// the target.
__global__ void k_batch_inputs(const int* __restrict__ pa, const int* __restrict__ pb, const float* __restrict__ tall,
                               long long count, long long per, long long off, long long mul, long long add, int k,
                               int kpad, const float* __restrict__ F1s, const float* __restrict__ F2s,
                               const int* __restrict__ ps, int n, __nv_bfloat16* __restrict__ X,
                               float* __restrict__ t) {
    const int i = blockIdx.x, c = threadIdx.x;  // 128 threads
    if (i >= kpad) return;
    float v = 0.f;
    if (i < k) {
        const long long j = (long long)(((unsigned long long)(off + i) * (unsigned long long)mul +
                                         (unsigned long long)add) % (unsigned long long)count);
        const long long sw = j / per;
        const float* F1 = F1s + sw * n * kFeat;
        const float* F2 = F2s + sw * n * kFeat;
        const int* p = ps + sw * n;
        const int a = pa[j], b = pb[j], q = c >> 5, f = c & 31;
        if (q == 0) v = F1[(size_t)a * kFeat + f];
        else if (q == 1) v = F1[(size_t)b * kFeat + f];
        else {
            const int img = p[q == 2 ? a : b];
            v = img < n ? F2[(size_t)img * kFeat + f] : 0.f;
        }
        if (c == 0) t[i] = tall[j];
    }
    X[(size_t)i * kMlpIn + c] = __float2bfloat16(v);
}

// acc += loss * k (the batch's share of an epoch's mean loss).
__global__ void k_loss_acc(const float* __restrict__ loss, int k, double* __restrict__ acc) {
    if (threadIdx.x == 0 && blockIdx.x == 0) *acc += (double)*loss * k;
}

// Partner j of vertex a in the candidate pool: a vertex b whose image the
// matching would like a to hold.  Draw h1 = mix64(seed ^ (a << 32 | j)), a
// G1 edge of a (out-list then in-list) with h1, then with h2 = mix64(h1) a G2
// vertex f on the matching side of that edge -- for a -> v an in-neighbour of
// p(v), for u -> a an out-neighbour of p(u) -- and take b = pinv(f): after
// swapping, a's image would carry that G2 edge.  Only such partners can raise
// a's own overlap.  Vertices without usable edges take (a + 1 + j) mod n;
// never a itself.
template <bool W16>
__device__ __forceinline__ int pool_partner(const DevView<W16>& g, int a, int j, unsigned long long seed) {
    typedef Ent<W16> EN;
    int b = -1;
    const int lo = g.off1o[a + 1] - g.off1o[a], li = g.off1i[a + 1] - g.off1i[a];
    if (lo + li > 0) {
        const unsigned long long h1 = mix64(seed ^ (((unsigned long long)a << 32) | (unsigned)j));
        const unsigned long long h2 = mix64(h1);
        const int k = (int)(h1 % (unsigned long long)(lo + li));
        if (k < lo) {
            const int pv = g.p[EN::id(g.ent1o[g.off1o[a] + k])];
            if (pv < g.n) {
                const int d = g.off2i[pv + 1] - g.off2i[pv];
                if (d > 0) b = g.pinv[EN::id(g.ent2i[g.off2i[pv] + (int)(h2 % (unsigned long long)d)])];
            }
        } else {
            const int pu = g.p[EN::id(g.ent1i[g.off1i[a] + (k - lo)])];
            if (pu < g.n) {
                const int d = g.off2o[pu + 1] - g.off2o[pu];
                if (d > 0) b = g.pinv[EN::id(g.ent2o[g.off2o[pu] + (int)(h2 % (unsigned long long)d)])];
            }
        }
    }
    if (b < 0 || b >= g.n || b == a) b = (int)(((long long)a + 1 + j) % g.n);
    if (b == a) b = (a + 1) % g.n;
    return b;
}

// Candidate pool: P partners per vertex, vertex-major.
template <bool W16>
__global__ void k_pool(DevView<W16> g, int P, unsigned long long seed, int* __restrict__ pa, int* __restrict__ pb) {
    const long long total = (long long)g.n * P;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(i / P), j = (int)(i % P);
        pa[i] = a;
        pb[i] = pool_partner(g, a, j, seed);
    }
}

// Training samples from the exact profit matrix S of the current matching:
// per row its best partner and `extra` pool partners, each with the target
// sign(d) log1p|d| of its exact delta d = S[a][b] + S[b][a] - S[a][a] - S[b][b].
template <bool W16>
__global__ void k_samples(DevView<W16> g, const unsigned long long* __restrict__ rowbest, int extra,
                          unsigned long long seed, int* __restrict__ pa, int* __restrict__ pb,
                          float* __restrict__ t) {
    const int n = g.n;
    const int a = blockIdx.x * blockDim.x + threadIdx.x;
    if (a >= n) return;
    const int* S = g.S;
    for (int j = 0; j <= extra; j++) {
        int b = j == 0 ? (int)(~(unsigned)(rowbest[a] & 0xffffffffu)) : pool_partner(g, a, j - 1, seed);
        if (b < 0 || b >= n || b == a) b = (a + 1) % n;
        const int d = S[(size_t)a * n + b] + S[(size_t)b * n + a] - S[(size_t)a * n + a] - S[(size_t)b * n + b];
        const size_t o = (size_t)a * (extra + 1) + j;
        pa[o] = a; pb[o] = b;
        t[o] = (d > 0 ? 1.f : (d < 0 ? -1.f : 0.f)) * log1pf(fabsf((float)d));
    }
}

// Exact deltas of many selected pairs, one 256-thread block per pair (a hub
// pair's lists spread over eight warps instead of one).
template <bool W16>
__global__ void __launch_bounds__(256) k_pair_deltas_block(DevView<W16> g, const int* __restrict__ pa,
                                                           const int* __restrict__ pb, long long k,
                                                           int* __restrict__ out) {
    __shared__ int part[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (long long i = blockIdx.x; i < k; i += gridDim.x) {
        int d = swap_delta_part<W16>(g, pa[i], pb[i], threadIdx.x, 256);
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) part[wid] = d;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < 8; w++) t += part[w];
            out[i] = t;
        }
        __syncthreads();
    }
}

// Per-row selection: one warp per vertex a picks the r best-scored of its P
// pool partners (P <= 1024, r <= 32; ties to the lower slot).
__global__ void k_row_topr(const float* __restrict__ ys, const int* __restrict__ pb, int n, int P, int r,
                           int* __restrict__ qa, int* __restrict__ qb) {
    const int lane = threadIdx.x & 31;
    const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (a >= n) return;
    const float* y = ys + (size_t)a * P;
    unsigned taken = 0;  // bit k: slot lane + 32k already chosen
    for (int t = 0; t < r; t++) {
        float best = -INFINITY;
        int bslot = 0x7fffffff;
        for (int k = 0; lane + 32 * k < P; k++) {
            if (taken & (1u << k)) continue;
            const float v = y[lane + 32 * k];
            if (v > best || (v == best && lane + 32 * k < bslot)) { best = v; bslot = lane + 32 * k; }
        }
        for (int o = 16; o; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, best, o);
            const int os = __shfl_xor_sync(0xffffffffu, bslot, o);
            if (ov > best || (ov == best && os < bslot)) { best = ov; bslot = os; }
        }
        if (bslot == 0x7fffffff) bslot = 0;  // fewer than r usable slots (NaN scores): repeat slot 0
        if ((bslot & 31) == lane) taken |= 1u << (bslot >> 5);
        if (lane == 0) {
            qa[(size_t)a * r + t] = a;
            qb[(size_t)a * r + t] = pb[(size_t)a * P + bslot];
        }
    }
}

__global__ void k_score_keys(const float* __restrict__ y, int k, unsigned* __restrict__ key, int* __restrict__ idx) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    unsigned u = __float_as_uint(y[i]);
    key[i] = (u & 0x80000000u) ? ~u : (u | 0x80000000u);  // order-preserving float -> uint
    idx[i] = i;
}

__global__ void k_gather_pairs(const int* __restrict__ idx, int k, const int* __restrict__ pa,
                               const int* __restrict__ pb, int* __restrict__ qa, int* __restrict__ qb) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    qa[i] = pa[idx[i]]; qb[i] = pb[idx[i]];
}

// Candidate keys of exactly evaluated pairs (delta > 0), ~0 otherwise.
__global__ void k_learned_keys(const int* __restrict__ qa, const int* __restrict__ qb, const int* __restrict__ d,
                               int k, unsigned long long* __restrict__ keys) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    unsigned long long out = ~0ull;
    if (d[i] > 0) {
        const int lo = min(qa[i], qb[i]), hi = max(qa[i], qb[i]);
        out = ((unsigned long long)(0x7fffffffu - (unsigned)d[i]) << 32) | ((unsigned long long)lo << 16) | hi;
    }
    keys[i] = out;
}

// Grow-only device buffer.
struct DBuf {
    void* p = nullptr;
    size_t cap = 0;
    cudaError_t need(size_t bytes) {
        if (bytes <= cap) return cudaSuccess;
        if (p) cudaFree(p);
        p = nullptr;
        cap = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e == cudaSuccess) cap = bytes;
        return e;
    }
    template <class T> T* as() const { return static_cast<T*>(p); }
    void release() { if (p) cudaFree(p); p = nullptr; cap = 0; }
};

}  // namespace

struct bm_mlp {
    int dev = 0;
    cudaStream_t st = nullptr;  // own stream
    cudaStream_t cs = nullptr;  // stream of the current call (own, or the engine's)
    char err[512] = {0};
    float *P = nullptr, *G = nullptr;
    __nv_bfloat16 *W1b = nullptr, *W2b = nullptr, *W2Tb = nullptr;
    int cap = 0;  // batch capacity (multiple of 128)
    __nv_bfloat16 *X = nullptr, *H1b = nullptr, *H2b = nullptr, *dH2b = nullptr, *dH1b = nullptr;
    __nv_bfloat16 *T1 = nullptr, *T2 = nullptr;  // transposes, 256 x cap
    float *H1f = nullptr, *H2f = nullptr, *dH1f = nullptr, *y = nullptr, *t = nullptr, *loss = nullptr;
    int* err_d = nullptr;
    // engine-side workspace: features, pool, ranking, exact evaluation
    DBuf contrib, F1, F2, fstat, pa, pb, ys, key, key2, idx, idx2, qa, qb, dd, ckeys, tmp, tall, xin;
    DBuf F1s, F2s, ps, eacc;  // training: per-sweep features and matchings, epoch losses
    DBuf U, V;                // factorised first layer, n x 256 each
    DBuf cinfo;               // list extents of the sorted candidates
    DBuf S1, S2;              // structural features of the context last seen
    unsigned long long static_serial = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr, ea = nullptr, eb = nullptr, ec = nullptr;
};

#define MK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            snprintf(M->err, sizeof M->err, "%s:%d: %s: %s", __FILE__, __LINE__, #call,  \
                     cudaGetErrorString(e_));                                            \
            return BM_E_CUDA;                                                            \
        }                                                                                \
    } while (0)

static thread_local char g_mlp_err[512];

extern "C" int64_t bm_mlp_param_count(void) { return kParams; }
extern "C" const char* bm_mlp_last_error(const bm_mlp* M) { return M ? M->err : g_mlp_err; }

static void mlp_free(bm_mlp* M) {
    if (!M) return;
    void* b[] = {M->P, M->G, M->W1b, M->W2b, M->W2Tb, M->X, M->H1b, M->H2b, M->dH2b, M->dH1b, M->T1, M->T2,
                 M->H1f, M->H2f, M->dH1f, M->y, M->t, M->loss, M->err_d};
    for (void* p : b) if (p) cudaFree(p);
    DBuf* w[] = {&M->contrib, &M->F1, &M->F2, &M->fstat, &M->pa, &M->pb, &M->ys, &M->key, &M->key2, &M->idx,
                 &M->idx2, &M->qa, &M->qb, &M->dd, &M->ckeys, &M->tmp, &M->tall, &M->xin,
                 &M->F1s, &M->F2s, &M->ps, &M->eacc, &M->U, &M->V, &M->S1, &M->S2, &M->cinfo};
    for (DBuf* d : w) d->release();
    for (cudaEvent_t e : {M->e0, M->e1, M->ea, M->eb, M->ec}) if (e) cudaEventDestroy(e);
    if (M->st) cudaStreamDestroy(M->st);
    delete M;
}
extern "C" void bm_mlp_destroy(bm_mlp* M) { mlp_free(M); }

static bm_status mlp_refresh_bf16(bm_mlp* M) {
    k_to_bf16<<<(kMlpHid * kMlpIn + 255) / 256, 256, 0, M->cs>>>(M->P + oW1, kMlpHid * kMlpIn, M->W1b);
    k_to_bf16<<<(kMlpHid * kMlpHid + 255) / 256, 256, 0, M->cs>>>(M->P + oW2, kMlpHid * kMlpHid, M->W2b);
    k_transpose_bf16<<<dim3(kMlpHid / 32, kMlpHid / 32), dim3(32, 8), 0, M->cs>>>(M->W2b, kMlpHid, kMlpHid, M->W2Tb);
    MK(cudaGetLastError());
    return BM_OK;
}

static bm_status mlp_reserve(bm_mlp* M, int rows) {
    const int need = (rows + 127) / 128 * 128;
    if (need <= M->cap) return BM_OK;
    void** bufs[] = {(void**)&M->X, (void**)&M->H1b, (void**)&M->H2b, (void**)&M->dH2b, (void**)&M->dH1b,
                     (void**)&M->T1, (void**)&M->T2, (void**)&M->H1f, (void**)&M->H2f, (void**)&M->dH1f,
                     (void**)&M->y, (void**)&M->t};
    for (void** b : bufs) if (*b) { cudaFree(*b); *b = nullptr; }
    M->cap = 0;
    const size_t c = (size_t)need;
    MK(cudaMalloc(&M->X, c * kMlpIn * sizeof(__nv_bfloat16)));
    MK(cudaMalloc(&M->H1b, c * kMlpHid * sizeof(__nv_bfloat16)));
    MK(cudaMalloc(&M->H2b, c * kMlpHid * sizeof(__nv_bfloat16)));
    MK(cudaMalloc(&M->dH2b, c * kMlpHid * sizeof(__nv_bfloat16)));
    MK(cudaMalloc(&M->dH1b, c * kMlpHid * sizeof(__nv_bfloat16)));
    MK(cudaMalloc(&M->T1, c * kMlpHid * sizeof(__nv_bfloat16)));
    MK(cudaMalloc(&M->T2, c * kMlpHid * sizeof(__nv_bfloat16)));
    MK(cudaMalloc(&M->H1f, c * kMlpHid * sizeof(float)));
    MK(cudaMalloc(&M->H2f, c * kMlpHid * sizeof(float)));
    MK(cudaMalloc(&M->dH1f, c * kMlpHid * sizeof(float)));
    MK(cudaMalloc(&M->y, c * sizeof(float)));
    MK(cudaMalloc(&M->t, c * sizeof(float)));
    M->cap = need;
    return BM_OK;
}

extern "C" bm_status bm_mlp_create(bm_mlp** out, uint64_t seed) {
    if (!out) return BM_E_INPUT;
    *out = nullptr;
    bm_mlp* M = new (std::nothrow) bm_mlp();
    if (!M) return BM_E_NOMEM;
    auto body = [&]() -> bm_status {
        MK(cudaGetDevice(&M->dev));
        MK(cudaStreamCreateWithFlags(&M->st, cudaStreamNonBlocking));
        M->cs = M->st;
        for (cudaEvent_t* e : {&M->e0, &M->e1, &M->ea, &M->eb, &M->ec}) MK(cudaEventCreate(e));
        MK(cudaMalloc(&M->P, kParams * sizeof(float)));
        MK(cudaMalloc(&M->G, kParams * sizeof(float)));
        MK(cudaMalloc(&M->W1b, kMlpHid * kMlpIn * sizeof(__nv_bfloat16)));
        MK(cudaMalloc(&M->W2b, kMlpHid * kMlpHid * sizeof(__nv_bfloat16)));
        MK(cudaMalloc(&M->W2Tb, kMlpHid * kMlpHid * sizeof(__nv_bfloat16)));
        MK(cudaMalloc(&M->loss, sizeof(float)));
        MK(cudaMalloc(&M->err_d, sizeof(int)));
        MK(cudaMemset(M->err_d, 0, sizeof(int)));
        // He-uniform initialisation from a seeded generator; zero biases
        std::mt19937_64 rng(seed);
        std::vector<float> h(kParams, 0.f);
        auto fill = [&](int off, int cnt, int fan_in) {
            const double lim = std::sqrt(6.0 / fan_in);
            std::uniform_real_distribution<double> u(-lim, lim);
            for (int i = 0; i < cnt; i++) h[off + i] = (float)u(rng);
        };
        fill(oW1, kMlpHid * kMlpIn, kMlpIn);
        fill(oW2, kMlpHid * kMlpHid, kMlpHid);
        fill(oW3, kMlpHid, kMlpHid);
        MK(cudaMemcpy(M->P, h.data(), kParams * sizeof(float), cudaMemcpyHostToDevice));
        bm_status s = mlp_refresh_bf16(M);
        if (s) return s;
        MK(cudaStreamSynchronize(M->cs));
        return BM_OK;
    };
    bm_status s = body();
    if (s) { snprintf(g_mlp_err, sizeof g_mlp_err, "%s", M->err); mlp_free(M); return s; }
    *out = M;
    return BM_OK;
}

extern "C" bm_status bm_mlp_get_params(bm_mlp* M, float* params) {
    if (!M || !params) return BM_E_INPUT;
    MK(cudaMemcpyAsync(params, M->P, kParams * sizeof(float), cudaMemcpyDeviceToHost, M->cs));
    MK(cudaStreamSynchronize(M->cs));
    return BM_OK;
}

extern "C" bm_status bm_mlp_set_params(bm_mlp* M, const float* params) {
    if (!M || !params) return BM_E_INPUT;
    MK(cudaMemcpyAsync(M->P, params, kParams * sizeof(float), cudaMemcpyHostToDevice, M->cs));
    bm_status s = mlp_refresh_bf16(M);
    if (s) return s;
    MK(cudaStreamSynchronize(M->cs));
    return BM_OK;
}

template <int BN>
static bm_status gemm(bm_mlp* M, const __nv_bfloat16* A, const __nv_bfloat16* B, int m, int n, int k, float* C,
                      const float* bias, int relu, __nv_bfloat16* Cb) {
    MK(cudaFuncSetAttribute(k_gemm_bf16<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, gemm_bf16_smem<BN>()));
    k_gemm_bf16<BN><<<dim3(n / BN, m / kGemmM), kGemmThreads, gemm_bf16_smem<BN>(), M->cs>>>(
        A, B, m, n, k, C, bias, relu, Cb, M->err_d, take_stall(BM_STALL_MLP_GEMM));
    MK(cudaGetLastError());
    return BM_OK;
}

// Forward of rows [0, kpad) of M->X through both wide layers.
static bm_status mlp_forward_dev(bm_mlp* M, int kpad) {
    bm_status s;
    if ((s = gemm<256>(M, M->X, M->W1b, kpad, kMlpHid, kMlpIn, M->H1f, M->P + oB1, 1, M->H1b))) return s;
    if ((s = gemm<256>(M, M->H1b, M->W2b, kpad, kMlpHid, kMlpHid, M->H2f, M->P + oB2, 1, M->H2b))) return s;
    return BM_OK;
}

// One forward + backward on rows [0,k) of X with targets t; gradients into M->G.
static bm_status mlp_fwd_bwd_dev(bm_mlp* M, int k) {
    const int kpad = (k + 127) / 128 * 128;
    bm_status s = mlp_forward_dev(M, kpad);
    if (s) return s;
    MK(cudaMemsetAsync(M->G, 0, kParams * sizeof(float), M->cs));
    MK(cudaMemsetAsync(M->loss, 0, sizeof(float), M->cs));
    k_head<<<(kpad * 32 + 255) / 256, 256, 0, M->cs>>>(M->H2f, k, kpad, M->P + oW3, M->P + oB3, M->y, M->t, M->loss,
                                                       M->dH2b, M->G + oW3, M->G + oB3);
    MK(cudaGetLastError());
    // dW2 = dH2^T H1 ; db2 = colsum dH2
    k_transpose_bf16<<<dim3(kMlpHid / 32, kpad / 32), dim3(32, 8), 0, M->cs>>>(M->dH2b, kpad, kMlpHid, M->T1);
    k_transpose_bf16<<<dim3(kMlpHid / 32, kpad / 32), dim3(32, 8), 0, M->cs>>>(M->H1b, kpad, kMlpHid, M->T2);
    MK(cudaGetLastError());
    if ((s = gemm<256>(M, M->T1, M->T2, kMlpHid, kMlpHid, kpad, M->G + oW2, nullptr, 0, nullptr))) return s;
    k_colsum_bf16<<<dim3(1, 64), kMlpHid, 0, M->cs>>>(M->dH2b, kpad, kMlpHid, M->G + oB2);
    // dH1 = dH2 W2, masked by ReLU'(H1); db1
    if ((s = gemm<256>(M, M->dH2b, M->W2Tb, kpad, kMlpHid, kMlpHid, M->dH1f, nullptr, 0, nullptr))) return s;
    k_relu_bwd<<<dim3(1, 64), kMlpHid, 0, M->cs>>>(M->dH1f, M->H1f, kpad, kMlpHid, M->dH1b, M->G + oB1);
    // dW1 = dH1^T X
    k_transpose_bf16<<<dim3(kMlpHid / 32, kpad / 32), dim3(32, 8), 0, M->cs>>>(M->dH1b, kpad, kMlpHid, M->T1);
    k_transpose_bf16<<<dim3(kMlpIn / 32, kpad / 32), dim3(32, 8), 0, M->cs>>>(M->X, kpad, kMlpIn, M->T2);
    MK(cudaGetLastError());
    if ((s = gemm<128>(M, M->T1, M->T2, kMlpHid, kMlpIn, kpad, M->G + oW1, nullptr, 0, nullptr))) return s;
    return BM_OK;
}

static bm_status check_err(bm_mlp* M) {
    int e = 0;
    MK(cudaMemcpyAsync(&e, M->err_d, sizeof e, cudaMemcpyDeviceToHost, M->cs));
    MK(cudaStreamSynchronize(M->cs));
    if (e) {
        // the call's results are not trusted; the network object stays usable
        snprintf(M->err, sizeof M->err, "tensor-core GEMM wait timed out");
        MK(cudaMemset(M->err_d, 0, sizeof(int)));
        return BM_E_TIMEOUT;
    }
    return BM_OK;
}

// Host rows x (k x 128 fp32) into M->X as bf16, padded with zero rows.
static bm_status upload_rows(bm_mlp* M, int64_t k, const float* x, int kpad) {
    MK(M->xin.need((size_t)kpad * kMlpIn * sizeof(float)));
    float* xf = M->xin.as<float>();
    MK(cudaMemsetAsync(xf, 0, (size_t)kpad * kMlpIn * sizeof(float), M->cs));
    MK(cudaMemcpyAsync(xf, x, (size_t)k * kMlpIn * sizeof(float), cudaMemcpyHostToDevice, M->cs));
    k_to_bf16<<<(kpad * kMlpIn + 255) / 256, 256, 0, M->cs>>>(xf, kpad * kMlpIn, M->X);
    MK(cudaGetLastError());
    return BM_OK;
}

extern "C" bm_status bm_mlp_forward(bm_mlp* M, int64_t k, const float* x, float* out) {
    if (!M || k < 0 || (k && (!x || !out))) return BM_E_INPUT;
    if (!k) return BM_OK;
    if (k > (1 << 24)) { snprintf(M->err, sizeof M->err, "bm_mlp_forward: at most 2^24 rows"); return BM_E_INPUT; }
    bm_status s = mlp_reserve(M, (int)k);
    if (s) return s;
    const int kpad = ((int)k + 127) / 128 * 128;
    if ((s = upload_rows(M, k, x, kpad))) return s;
    if ((s = mlp_forward_dev(M, kpad))) return s;
    k_head<<<(kpad * 32 + 255) / 256, 256, 0, M->cs>>>(M->H2f, (int)k, kpad, M->P + oW3, M->P + oB3, M->y, nullptr,
                                                       nullptr, nullptr, nullptr, nullptr);
    MK(cudaGetLastError());
    MK(cudaMemcpyAsync(out, M->y, (size_t)k * sizeof(float), cudaMemcpyDeviceToHost, M->cs));
    return check_err(M);
}

extern "C" bm_status bm_mlp_train_step(bm_mlp* M, int64_t k, const float* x, const float* target, float lr,
                                       float* loss, float* grads) {
    if (!M || k <= 0 || !x || !target) return BM_E_INPUT;
    if (k > (1 << 24)) { snprintf(M->err, sizeof M->err, "bm_mlp_train_step: at most 2^24 rows"); return BM_E_INPUT; }
    bm_status s = mlp_reserve(M, (int)k);
    if (s) return s;
    const int kpad = ((int)k + 127) / 128 * 128;
    if ((s = upload_rows(M, k, x, kpad))) return s;
    MK(cudaMemcpyAsync(M->t, target, (size_t)k * sizeof(float), cudaMemcpyHostToDevice, M->cs));
    if ((s = mlp_fwd_bwd_dev(M, (int)k))) return s;
    if (grads) MK(cudaMemcpyAsync(grads, M->G, kParams * sizeof(float), cudaMemcpyDeviceToHost, M->cs));
    if (loss) MK(cudaMemcpyAsync(loss, M->loss, sizeof(float), cudaMemcpyDeviceToHost, M->cs));
    if (lr != 0.f) {
        k_sgd<<<(kParams + 255) / 256, 256, 0, M->cs>>>(M->P, M->G, kParams, lr, nullptr);
        if ((s = mlp_refresh_bf16(M))) return s;
    }
    return check_err(M);
}

// ---------------------------------------------------------------------------
// Engine-side pieces: features, ranking, sampling, training, learned sweep.

// Per-vertex features of ctx's graphs and current matching into M->F1, M->F2
// (normalised).  The structural columns depend on the graphs only and are
// kept for the context last seen.
template <bool W16>
static bm_status features(bm_ctx* ctx, bm_mlp* M) {
    const int n = ctx->n;
    const size_t fbytes = (size_t)n * kFeat * sizeof(float);
    MK(M->contrib.need((size_t)n * sizeof(float)));
    MK(M->F1.need(fbytes));
    MK(M->F2.need(fbytes));
    DevView<W16> g = view<W16>(ctx);
    const int blocks = (n + 7) / 8;
    if (M->static_serial != ctx->serial) {
        MK(M->S1.need(fbytes));
        MK(M->S2.need(fbytes));
        k_static_features<W16><<<blocks, 256, 0, M->cs>>>(g, 0, M->S1.as<float>());
        k_static_features<W16><<<blocks, 256, 0, M->cs>>>(g, 1, M->S2.as<float>());
        MK(cudaGetLastError());
        M->static_serial = ctx->serial;
    }
    MK(cudaMemcpyAsync(M->F1.p, M->S1.p, fbytes, cudaMemcpyDeviceToDevice, M->cs));
    MK(cudaMemcpyAsync(M->F2.p, M->S2.p, fbytes, cudaMemcpyDeviceToDevice, M->cs));
    k_contrib<W16><<<blocks, 256, 0, M->cs>>>(g, M->contrib.as<float>());
    k_dyn_features<<<(n + 255) / 256, 256, 0, M->cs>>>(M->contrib.as<float>(), ctx->pinv, n, M->F1.as<float>(),
                                                       M->F2.as<float>());
    MK(M->fstat.need(4 * kFeat * sizeof(float)));
    float* mean = M->fstat.as<float>();
    k_col_stats<<<2 * kFeat, 256, 0, M->cs>>>(M->F1.as<float>(), M->F2.as<float>(), n, mean, mean + 2 * kFeat);
    const long long tot = 2LL * n * kFeat;
    k_normalise<<<(unsigned)((tot + 255) / 256), 256, 0, M->cs>>>(M->F1.as<float>(), M->F2.as<float>(), n, mean,
                                                                   mean + 2 * kFeat);
    MK(cudaGetLastError());
    return BM_OK;
}

// Network scores y[i] of the pairs (pa[i], pb[i]), i < k, on ctx's current
// features (M->F1, M->F2): factorised first layer (U, V; skipped when they are
// current), then the fused kernel.
static bm_status rank_pairs_dev(bm_ctx* ctx, bm_mlp* M, const int* pa, const int* pb, long long k, float* y,
                                bool uv_current = false) {
    const int n = ctx->n;
    if (!uv_current) {
        MK(M->U.need((size_t)n * kMlpHid * sizeof(float)));
        MK(M->V.need((size_t)n * kMlpHid * sizeof(float)));
        k_uv<<<(n + 7) / 8, 256, 0, M->cs>>>(M->F1.as<float>(), M->F2.as<float>(), ctx->p, n, M->W1b, M->P + oB1,
                                             M->U.as<float>(), M->V.as<float>());
        MK(cudaGetLastError());
    }
    if (k == 0) return BM_OK;
    MK(cudaFuncSetAttribute(k_mlp_rank, cudaFuncAttributeMaxDynamicSharedMemorySize, kRankSmem));
    const long long tiles = (k + kGemmM - 1) / kGemmM;
    const int grid = (int)std::min<long long>(tiles, ctx->num_sms);
    k_mlp_rank<<<grid, kRankThreads, kRankSmem, M->cs>>>(M->U.as<float>(), M->V.as<float>(), pa, pb, k, M->W2b,
                                                         M->P + oB2, M->P + oW3, M->P + oB3, y, M->err_d);
    MK(cudaGetLastError());
    return BM_OK;
}

extern "C" bm_status bm_mlp_features(bm_mlp* M, bm_ctx* ctx, float* f1, float* f2) {
    if (!M || !ctx || !f1 || !f2) return BM_E_INPUT;
    if (!ctx->mapped) { snprintf(M->err, sizeof M->err, "bm_mlp_features: no mapping set"); return BM_E_STATE; }
    M->cs = ctx->st;
    auto body = [&]() -> bm_status {
        bm_status r = ctx->w16 ? features<true>(ctx, M) : features<false>(ctx, M);
        if (r) return r;
        const size_t bytes = (size_t)ctx->n * kFeat * sizeof(float);
        MK(cudaMemcpyAsync(f1, M->F1.p, bytes, cudaMemcpyDeviceToHost, M->cs));
        MK(cudaMemcpyAsync(f2, M->F2.p, bytes, cudaMemcpyDeviceToHost, M->cs));
        MK(cudaStreamSynchronize(M->cs));
        return BM_OK;
    };
    bm_status s = body();
    M->cs = M->st;
    return s;
}

extern "C" bm_status bm_mlp_rank_pairs(bm_mlp* M, bm_ctx* ctx, int64_t k, const int32_t* m1, const int32_t* m2,
                                       float* out) {
    if (!M || !ctx || k < 0 || (k && (!m1 || !m2 || !out))) return BM_E_INPUT;
    if (!ctx->mapped) { snprintf(M->err, sizeof M->err, "bm_mlp_rank_pairs: no mapping set"); return BM_E_STATE; }
    if (k > (1LL << 31)) { snprintf(M->err, sizeof M->err, "bm_mlp_rank_pairs: too many pairs"); return BM_E_INPUT; }
    std::vector<int> a((size_t)k), b((size_t)k);
    for (int64_t i = 0; i < k; i++) {
        if (m1[i] < 1 || m1[i] > ctx->n || m2[i] < 1 || m2[i] > ctx->n) {
            snprintf(M->err, sizeof M->err, "bm_mlp_rank_pairs: pair %lld has an id outside 1..%d", (long long)i,
                     ctx->n);
            return BM_E_INPUT;
        }
        a[i] = m1[i] - 1;
        b[i] = m2[i] - 1;
    }
    M->cs = ctx->st;
    auto body = [&]() -> bm_status {
        bm_status r = ctx->w16 ? features<true>(ctx, M) : features<false>(ctx, M);
        if (r) return r;
        const size_t kk = (size_t)std::max<int64_t>(k, 1);
        MK(M->pa.need(kk * sizeof(int)));
        MK(M->pb.need(kk * sizeof(int)));
        MK(M->ys.need(kk * sizeof(float)));
        if (k) {
            MK(cudaMemcpyAsync(M->pa.p, a.data(), (size_t)k * sizeof(int), cudaMemcpyHostToDevice, M->cs));
            MK(cudaMemcpyAsync(M->pb.p, b.data(), (size_t)k * sizeof(int), cudaMemcpyHostToDevice, M->cs));
        }
        if ((r = rank_pairs_dev(ctx, M, M->pa.as<int>(), M->pb.as<int>(), k, M->ys.as<float>()))) return r;
        if (k) MK(cudaMemcpyAsync(out, M->ys.p, (size_t)k * sizeof(float), cudaMemcpyDeviceToHost, M->cs));
        return check_err(M);
    };
    bm_status s = body();
    M->cs = M->st;
    return s;
}

template <bool W16>
static bm_status train_from_impl(bm_mlp* M, bm_ctx* ctx, int sweeps, int extra, int epochs, float lr,
                                 uint64_t seed, bm_mlp_train_stats* out) {
    const int n = ctx->n;
    const long long per = (long long)n * (extra + 1);
    const long long count = per * sweeps;
    if (out) memset(out, 0, sizeof *out);
    if (count == 0) return BM_OK;
    if (count > (1LL << 40)) { snprintf(M->err, sizeof M->err, "too many training samples"); return BM_E_INPUT; }
    const int batch = 1024;
    bm_status s = mlp_reserve(M, batch);
    if (s) return s;
    const size_t fbytes = (size_t)n * kFeat * sizeof(float);
    MK(M->pa.need((size_t)count * sizeof(int)));
    MK(M->pb.need((size_t)count * sizeof(int)));
    MK(M->tall.need((size_t)count * sizeof(float)));
    MK(M->F1s.need(fbytes * sweeps));
    MK(M->F2s.need(fbytes * sweeps));
    MK(M->ps.need((size_t)n * sweeps * sizeof(int)));
    MK(M->eacc.need(2 * sizeof(double)));
    int *pa = M->pa.as<int>(), *pb = M->pb.as<int>();
    float* tall = M->tall.as<float>();
    // 1. log: per sweep the exact deltas of the current matching (profit matrix,
    //    row bests), the samples, the features; then one ordinary sweep
    for (int sw = 0; sw < sweeps; sw++) {
        if ((s = ensure_S(ctx))) return s;
        int mode = 0;
        if ((s = stage_refresh<W16>(ctx, &mode))) return s;
        if ((s = stage_combine(ctx, nullptr))) return s;
        if ((s = features<W16>(ctx, M))) return s;
        k_samples<W16><<<(n + 255) / 256, 256, 0, M->cs>>>(view<W16>(ctx), ctx->rowbest, extra,
                                                           seed + 7919ull * sw, pa + sw * per, pb + sw * per,
                                                           tall + sw * per);
        MK(cudaGetLastError());
        MK(cudaMemcpyAsync(M->F1s.as<char>() + fbytes * sw, M->F1.p, fbytes, cudaMemcpyDeviceToDevice, M->cs));
        MK(cudaMemcpyAsync(M->F2s.as<char>() + fbytes * sw, M->F2.p, fbytes, cudaMemcpyDeviceToDevice, M->cs));
        MK(cudaMemcpyAsync(M->ps.as<int>() + (size_t)n * sw, ctx->p, (size_t)n * sizeof(int),
                           cudaMemcpyDeviceToDevice, M->cs));
        bm_sweep_stats st;
        if ((s = bm_sweep(ctx, &kIncremental, &st))) { snprintf(M->err, sizeof M->err, "%s", ctx->err); return s; }
    }
    // 2. train: epochs of SGD over all logged samples, freshly shuffled each epoch
    double* eacc = M->eacc.as<double>();
    MK(cudaMemsetAsync(eacc, 0, 2 * sizeof(double), M->cs));
    long long samples = 0, steps = 0;
    for (int ep = 0; ep < epochs; ep++) {
        const unsigned long long h = mix64(seed ^ (0x5bd1e995ull * (unsigned long long)(ep + 1)));
        long long mul = (long long)(h % (unsigned long long)count) | 1;
        while (std::gcd(mul, count) != 1) mul += 2;
        const long long add = (long long)(mix64(h) % (unsigned long long)count);
        for (long long off = 0; off < count; off += batch) {
            const int k = (int)std::min<long long>(batch, count - off);
            const int kpad = (k + 127) / 128 * 128;
            k_batch_inputs<<<kpad, kMlpIn, 0, M->cs>>>(pa, pb, tall, count, per, off, mul, add, k, kpad,
                                                       M->F1s.as<float>(), M->F2s.as<float>(), M->ps.as<int>(),
                                                       n, M->X, M->t);
            if ((s = mlp_fwd_bwd_dev(M, k))) return s;
            if (ep == 0) k_loss_acc<<<1, 32, 0, M->cs>>>(M->loss, k, eacc);
            if (ep == epochs - 1) k_loss_acc<<<1, 32, 0, M->cs>>>(M->loss, k, eacc + 1);
            k_sgd<<<(kParams + 255) / 256, 256, 0, M->cs>>>(M->P, M->G, kParams, lr, nullptr);
            if ((s = mlp_refresh_bf16(M))) return s;
            samples += k;
            steps++;
        }
    }
    double el[2] = {0, 0};
    MK(cudaMemcpyAsync(el, eacc, sizeof el, cudaMemcpyDeviceToHost, M->cs));
    if ((s = check_err(M))) return s;
    if (out) {
        out->samples = samples;
        out->steps = steps;
        out->first_loss = (float)(el[0] / count);
        out->last_loss = (float)(el[1] / count);
    }
    return BM_OK;
}

extern "C" bm_status bm_mlp_train_from(bm_mlp* M, bm_ctx* ctx, int32_t sweeps, int32_t extra_partners,
                                       int32_t epochs, float lr, uint64_t seed, bm_mlp_train_stats* stats) {
    if (!M || !ctx || sweeps < 0 || extra_partners < 0 || epochs < 1) return BM_E_INPUT;
    if (!ctx->mapped) { snprintf(M->err, sizeof M->err, "bm_mlp_train_from: no mapping set"); return BM_E_STATE; }
    M->cs = ctx->st;  // one stream with the engine: samples read its profit matrix
    bm_status s = ctx->w16 ? train_from_impl<true>(M, ctx, sweeps, extra_partners, epochs, lr, seed, stats)
                           : train_from_impl<false>(M, ctx, sweeps, extra_partners, epochs, lr, seed, stats);
    cudaStreamSynchronize(M->cs);
    M->cs = M->st;
    return s;
}

template <bool W16>
static bm_status learned_impl(bm_ctx* ctx, bm_mlp* M, const bm_learned_opts* o, bm_sweep_stats* stats,
                              int* fell_back, bool allow_fallback = true) {
    const int n = ctx->n;
    const int P = o && o->pool > 0 ? o->pool : 64;
    const double frac = o && o->top_fraction > 0 ? std::min(o->top_fraction, 1.0) : 0.02;
    const long long pool_ll = (long long)n * P;
    if (pool_ll > INT32_MAX / 2) { snprintf(M->err, sizeof M->err, "candidate pool too large"); return BM_E_INPUT; }
    const int pool = (int)pool_ll;
    const int per_row = o ? o->per_row : 0;
    if (per_row < 0 || per_row > 32 || (per_row > 0 && (P > 1024 || per_row > P))) {
        snprintf(M->err, sizeof M->err, "bm_learned_sweep: per_row must be 0..min(32, pool) and pool <= 1024");
        return BM_E_INPUT;
    }
    const int top = per_row > 0 ? n * per_row : std::max(1, std::min(pool, (int)std::ceil(frac * pool)));
    *fell_back = 0;
    const long long before = ctx->score;
    MK(M->pa.need((size_t)pool * sizeof(int)));
    MK(M->pb.need((size_t)pool * sizeof(int)));
    MK(M->ys.need((size_t)pool * sizeof(float)));
    MK(M->key.need((size_t)pool * sizeof(unsigned)));
    MK(M->key2.need((size_t)pool * sizeof(unsigned)));
    MK(M->idx.need((size_t)pool * sizeof(int)));
    MK(M->idx2.need((size_t)pool * sizeof(int)));
    MK(M->qa.need((size_t)top * sizeof(int)));
    MK(M->qb.need((size_t)top * sizeof(int)));
    MK(M->dd.need((size_t)top * sizeof(int)));
    MK(M->ckeys.need((size_t)top * 2 * sizeof(unsigned long long)));
    MK(M->cinfo.need((size_t)top * 2 * sizeof(int4)));
    int *pa = M->pa.as<int>(), *pb = M->pb.as<int>(), *idx = M->idx.as<int>(), *idx2 = M->idx2.as<int>();
    int *qa = M->qa.as<int>(), *qb = M->qb.as<int>(), *dd = M->dd.as<int>();
    unsigned *key = M->key.as<unsigned>(), *key2 = M->key2.as<unsigned>();
    unsigned long long* ck = M->ckeys.as<unsigned long long>();
    float* ys = M->ys.as<float>();
    size_t tb1 = 0, tb2 = 0;
    MK(cub::DeviceRadixSort::SortPairsDescending(nullptr, tb1, key, key2, idx, idx2, pool));
    MK(cub::DeviceRadixSort::SortKeys(nullptr, tb2, ck, ck + top, top));
    MK(M->tmp.need(std::max(tb1, tb2)));
    bm_status r = BM_OK;
    const int attempts = 1 + std::max(0, o ? o->retries : 0);
    DevView<W16> g = view<W16>(ctx);
    CommitStats cs;
    memset(&cs, 0, sizeof cs);
    if (stats) memset(stats, 0, sizeof *stats);
    for (int at = 0; at < attempts; at++) {
        // a failed attempt commits nothing, so the features and U, V stay valid
        MK(cudaEventRecord(M->e0, M->cs));
        if (at == 0 && (r = features<W16>(ctx, M))) return r;
        const unsigned long long seed = (o ? o->seed : 0) + 0x9E3779B97F4A7C15ull * (unsigned long long)at;
        k_pool<W16><<<ctx->num_sms * 8, 256, 0, M->cs>>>(g, P, seed, pa, pb);
        MK(cudaGetLastError());
        MK(cudaEventRecord(M->ea, M->cs));
        // rank the pool with the network (factorised first layer + fused kernel)
        if ((r = rank_pairs_dev(ctx, M, pa, pb, pool, ys, at > 0))) return r;
        MK(cudaEventRecord(M->eb, M->cs));
        size_t tb = M->tmp.cap;
        if (per_row > 0) {  // each vertex's best-ranked partners
            k_row_topr<<<(n + 7) / 8, 256, 0, M->cs>>>(ys, pb, n, P, per_row, qa, qb);
        } else {            // the best-ranked fraction of the whole pool
            k_score_keys<<<(pool + 255) / 256, 256, 0, M->cs>>>(ys, pool, key, idx);
            MK(cub::DeviceRadixSort::SortPairsDescending(M->tmp.p, tb, key, key2, idx, idx2, pool, 0, 32, M->cs));
            k_gather_pairs<<<(top + 255) / 256, 256, 0, M->cs>>>(idx2, top, pa, pb, qa, qb);
        }
        // exact deltas of the selected pairs on the current matching
        const long long blocks = std::min<long long>(top, (long long)ctx->num_sms * 8);
        k_pair_deltas_block<W16><<<(int)blocks, 256, 0, M->cs>>>(g, qa, qb, top, dd);
        MK(cudaEventRecord(M->ec, M->cs));
        k_learned_keys<<<(top + 255) / 256, 256, 0, M->cs>>>(qa, qb, dd, top, ck);
        tb = M->tmp.cap;
        MK(cub::DeviceRadixSort::SortKeys(M->tmp.p, tb, ck, ck + top, top, 0, 64, M->cs));
        MK(cudaGetLastError());
        // exact set commit of the improving ones, in (delta desc, lo, hi) order
        k_cand_info<W16><<<(top + 255) / 256, 256, 0, M->cs>>>(g, ck + top, top, M->cinfo.as<int4>());
        const size_t smem = commit_group_smem(n);
        if (smem + 4096 > ctx->smem_optin) {
            snprintf(M->err, sizeof M->err, "set commit needs %zu bytes of shared memory for n=%d: n too large",
                     smem, n);
            return BM_E_INPUT;
        }
        if (!ctx->cgrid) {
            MK(cudaMalloc(&ctx->cgrid, commit_grid_ints() * sizeof(int)));
            MK(cudaMemset(ctx->cgrid, 0, commit_grid_ints() * sizeof(int)));
        }
        const int ctas = std::min(kCommitDefaultCtas, ctx->num_sms);
        MK(launch_commit_group<W16>(g, ck + top, top, -1, ctx->cstats, M->cinfo.as<int4>(), ctas, ctx->cgrid, smem,
                                    M->cs));
        MK(cudaMemcpyAsync(&cs, ctx->cstats, sizeof cs, cudaMemcpyDeviceToHost, M->cs));
        int cerr = 0;
        MK(cudaMemcpyAsync(&cerr, ctx->cgrid, sizeof cerr, cudaMemcpyDeviceToHost, M->cs));
        MK(cudaEventRecord(M->e1, M->cs));
        if ((r = check_err(M))) return r;
        if (cerr) { snprintf(M->err, sizeof M->err, "set commit grid barrier wait timed out"); return BM_E_TIMEOUT; }
        if (stats) {
            float t[5];
            cudaEventElapsedTime(&t[0], M->e0, M->ea);
            cudaEventElapsedTime(&t[1], M->ea, M->eb);
            cudaEventElapsedTime(&t[2], M->eb, M->ec);
            cudaEventElapsedTime(&t[3], M->ec, M->e1);
            cudaEventElapsedTime(&t[4], M->e0, M->e1);
            stats->ms_prep += t[0];
            stats->ms_hub += t[1];
            stats->ms_combine += t[2];
            stats->ms_commit += t[3];
            stats->ms_total += t[4];
            stats->deltas_evaluated += top;
            stats->candidates += pool;
            stats->scanned += cs.scanned;
            stats->verified += cs.verified;
        }
        if (cs.committed > 0) break;
    }
    ctx->score = before + cs.total_delta;
    if (stats) {
        stats->score_before = before;
        stats->score_after = ctx->score;
        stats->committed = cs.committed;
        stats->commit_steps = cs.steps;
        stats->commit_carried = cs.carried;
    }
    if (cs.committed == 0 && allow_fallback) {  // nothing improving among the proposals: exhaustive sweep
        *fell_back = 1;
        bm_sweep_stats fs;
        r = bm_sweep(ctx, &kIncremental, &fs);
        if (r) { snprintf(M->err, sizeof M->err, "%s", ctx->err); return r; }
        if (stats) {
            stats->score_after = fs.score_after;
            stats->committed = fs.committed;
            stats->deltas_evaluated += fs.deltas_evaluated;
            stats->ms_total += fs.ms_total;
        }
    }
    return BM_OK;
}

extern "C" bm_status bm_learned_sweep(bm_ctx* ctx, bm_mlp* M, const bm_learned_opts* opts, bm_sweep_stats* stats,
                                      int32_t* fell_back) {
    if (!ctx || !M) return BM_E_INPUT;
    if (!ctx->mapped) { snprintf(M->err, sizeof M->err, "bm_learned_sweep: no mapping set"); return BM_E_STATE; }
    int fb = 0;
    M->cs = ctx->st;  // one stream with the engine: the commit changes its matching
    bm_status s = ctx->w16 ? learned_impl<true>(ctx, M, opts, stats, &fb) : learned_impl<false>(ctx, M, opts, stats, &fb);
    cudaStreamSynchronize(M->cs);
    M->cs = M->st;
    if (fell_back) *fell_back = fb;
    return s;
}

extern "C" bm_status bm_learned_run(bm_ctx* ctx, bm_mlp* M, const bm_learned_opts* opts, int32_t max_sweeps,
                                    int64_t target_score, int32_t probe_every, bm_learned_run_stats* out,
                                    int64_t* trace_score, float* trace_ms, int8_t* trace_kind) {
    if (!ctx || !M || max_sweeps < 0 || probe_every < 0) return BM_E_INPUT;
    if (!ctx->mapped) { snprintf(M->err, sizeof M->err, "bm_learned_run: no mapping set"); return BM_E_STATE; }
    bm_learned_run_stats rs;
    memset(&rs, 0, sizeof rs);
    rs.score_before = ctx->score;
    const int probe = probe_every > 0 ? probe_every : 8;
    double rate_learned = -1.0, rate_full = -1.0;  // score gained per device-ms, last of each kind
    int since_learned = 0;
    bool converged = false;
    bm_status s = BM_OK;
    M->cs = ctx->st;
    for (int step = 0; step < max_sweeps; step++) {
        if (target_score > 0 && ctx->score >= target_score) { rs.reached = 1; break; }
        // learned while it gains at least as fast as the exhaustive sweep; the
        // first step is learned, the second measures the exhaustive rate
        const bool learned = rate_learned < 0 || (rate_full >= 0 && (rate_learned >= rate_full || since_learned >= probe));
        bm_sweep_stats st;
        int kind = 0;
        if (learned) {
            int fb = 0;
            s = ctx->w16 ? learned_impl<true>(ctx, M, opts, &st, &fb, false)
                         : learned_impl<false>(ctx, M, opts, &st, &fb, false);
            if (s) break;
            rate_learned = (double)(st.score_after - st.score_before) / std::max(st.ms_total, 1e-3f);
            rs.learned++;
            rs.ms_learned += st.ms_total;
            since_learned = 0;
            kind = 1;
        }
        if (!learned || st.committed == 0) {  // exhaustive sweep (also the fallback of a fruitless learned one)
            const long long before = ctx->score;
            bm_sweep_stats fs;
            s = bm_sweep(ctx, &kIncremental, &fs);
            if (s) { snprintf(M->err, sizeof M->err, "%s", ctx->err); break; }
            rate_full = (double)(fs.score_after - before) / std::max(fs.ms_total, 1e-3f);
            rs.exhaustive++;
            rs.ms_exhaustive += fs.ms_total;
            if (!learned) since_learned++;
            if (kind == 1) { st.committed = fs.committed; st.ms_total += fs.ms_total; kind = 2; }
            else { st = fs; kind = 0; }
            if (fs.committed == 0) converged = true;
        }
        rs.committed += st.committed;
        rs.ms_total += st.ms_total;
        if (trace_score) trace_score[rs.sweeps] = ctx->score;
        if (trace_ms) trace_ms[rs.sweeps] = rs.ms_total;
        if (trace_kind) trace_kind[rs.sweeps] = (int8_t)kind;
        rs.sweeps++;
        if (converged) break;
    }
    if (!s && target_score > 0 && ctx->score >= target_score) rs.reached = 1;
    rs.converged = converged ? 1 : 0;
    rs.score_after = ctx->score;
    cudaStreamSynchronize(M->cs);
    M->cs = M->st;
    if (out) *out = rs;
    return s;
}
