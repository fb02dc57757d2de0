// bm_engine.cu -- context, preprocessing and the C ABI of the swap-delta engine.
//
// Boundary: include/bm.h.  Every entry point returns a bm_status and records
// a message retrievable with bm_last_error; nothing here calls exit().
// All device work of a context runs on one non-blocking stream.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cstdarg>
#include <vector>
#include <atomic>
#include <algorithm>
#include <utility>
#include <mutex>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include "bm.h"
#include "bm_internal.cuh"
#include "bm_triples.cuh"
#include "bm_quads.cuh"
#include "bm_select.cuh"
#include "bm_combine_tma.cuh"
#include "bm_hub.cuh"
#include "bm_hub_ws.cuh"
#include "bm_incr.cuh"

using namespace bm;

static thread_local char g_create_err[512];

static bool hub_ws_setup(bm_ctx* ctx);

// Test hook: the site set by bm_test_stall, taken (and cleared) by the next
// launch at that site.
static std::atomic<int> g_stall{0};

int take_stall(int site) {
    int want = site;
    return g_stall.compare_exchange_strong(want, 0) ? 1 : 0;
}

extern "C" bm_status bm_test_stall(int32_t site) {
    if (site < 0 || site > BM_STALL_BATCH) return BM_E_INPUT;
    g_stall.store(site);
    return BM_OK;
}

void set_err(bm_ctx* c, const char* fmt, ...) {
    char* dst = c ? c->err : g_create_err;
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(dst, 512, fmt, ap);
    va_end(ap);
}

extern "C" const char* bm_last_error(const bm_ctx* ctx) { return ctx ? ctx->err : g_create_err; }

// ---------------------------------------------------------------------------
// Host preprocessing: CSR/CSC build with the reference's graph semantics.
namespace {

struct HostCSR {
    std::vector<int> off;        // n+2 (off[n+1] = off[n]: empty NONE row)
    std::vector<int> id, w;      // entries
};

// Builds a CSR keyed by `key` (src for out-lists, dst for in-lists); entries
// within a row are sorted by the other endpoint, ties kept in input order.
static void build_csr(int n, const std::vector<int>& key, const std::vector<int>& other,
                      const std::vector<int>& w, HostCSR& out) {
    const size_t m = key.size();
    out.off.assign((size_t)n + 2, 0);
    for (size_t i = 0; i < m; i++) out.off[key[i] + 1]++;
    for (int v = 0; v < n; v++) out.off[v + 1] += out.off[v];
    out.off[n + 1] = out.off[n];
    std::vector<int> pos(out.off.begin(), out.off.begin() + n);
    std::vector<int> idx(m);
    for (size_t i = 0; i < m; i++) idx[pos[key[i]]++] = (int)i;
    for (int v = 0; v < n; v++) {
        auto b = idx.begin() + out.off[v], e = idx.begin() + out.off[v + 1];
        std::stable_sort(b, e, [&](int x, int y) { return other[x] < other[y]; });
    }
    out.id.resize(m);
    out.w.resize(m);
    for (size_t i = 0; i < m; i++) { out.id[i] = other[idx[i]]; out.w[i] = w[idx[i]]; }
}

}  // namespace

template <bool W16>
static bm_status upload_lists(bm_ctx* ctx, const HostCSR& g1o, const HostCSR& g1i,
                              const HostCSR& g2o, const HostCSR& g2i, int clamp1, int clamp2) {
    typedef Ent<W16> EN;
    typedef typename EN::T E;
    auto pack = [&](const HostCSR& h, int clampw, void** dst, void** dstP) -> bm_status {
        std::vector<E> v(h.id.size());
        for (size_t i = 0; i < v.size(); i++) v[i] = EN::make(h.id[i], std::min(h.w[i], clampw));
        CK(dalloc(ctx, (E**)dst, v.size() * sizeof(E)));
        CK(dalloc(ctx, (E**)dstP, v.size() * sizeof(E)));
        if (!v.empty()) CK(cudaMemcpy(*dst, v.data(), v.size() * sizeof(E), cudaMemcpyHostToDevice));
        return BM_OK;
    };
    bm_status s;
    if ((s = pack(g1o, clamp1, &ctx->ent1o, &ctx->ent1oP)) != BM_OK) return s;
    if ((s = pack(g1i, clamp1, &ctx->ent1i, &ctx->ent1iP)) != BM_OK) return s;
    if ((s = pack(g2o, clamp2, &ctx->ent2o, &ctx->ent2oP)) != BM_OK) return s;
    if ((s = pack(g2i, clamp2, &ctx->ent2i, &ctx->ent2iP)) != BM_OK) return s;
    return BM_OK;
}

template <bool W16>
static bm_status upload_entries(bm_ctx* ctx, const HostCSR& h, void** dst, void** dstP) {
    typedef Ent<W16> EN;
    typedef typename EN::T E;
    std::vector<E> v(h.id.size());
    for (size_t i = 0; i < v.size(); i++) v[i] = EN::make(h.id[i], h.w[i]);
    CK(dalloc(ctx, (E**)dst, v.size() * sizeof(E)));
    CK(dalloc(ctx, (E**)dstP, v.size() * sizeof(E)));
    if (!v.empty()) CK(cudaMemcpy(*dst, v.data(), v.size() * sizeof(E), cudaMemcpyHostToDevice));
    return BM_OK;
}

template <bool W16>
static bm_status upload_dense(bm_ctx* ctx, const HostCSR& g2o, const HostCSR& g2i, int clamp2) {
    typedef typename Dense<W16>::T D;
    const size_t n1 = (size_t)ctx->n + 1;
    const int n = ctx->n;
    CK(dalloc(ctx, (D**)&ctx->W2, n1 * n1 * sizeof(D)));
    CK(dalloc(ctx, (D**)&ctx->W2T, n1 * n1 * sizeof(D)));
    CK(cudaMemset(ctx->W2, 0, n1 * n1 * sizeof(D)));
    CK(cudaMemset(ctx->W2T, 0, n1 * n1 * sizeof(D)));
    // fill row by row (and the transpose column by column) through a staging buffer
    const size_t chunk_rows = 256;
    std::vector<D> buf(chunk_rows * n1);
    for (int t = 0; t < 2; t++) {
        for (int f0 = 0; f0 < n; f0 += (int)chunk_rows) {
            const int f1 = std::min(n, f0 + (int)chunk_rows);
            std::fill(buf.begin(), buf.end(), (D)0);
            const HostCSR& h = t == 0 ? g2o : g2i;  // in-lists are the rows of the transpose
            for (int f = f0; f < f1; f++)
                for (int i = h.off[f]; i < h.off[f + 1]; i++)
                    buf[(size_t)(f - f0) * n1 + h.id[i]] = (D)std::min(h.w[i], clamp2);
            D* out = (D*)(t == 0 ? ctx->W2 : ctx->W2T);
            CK(cudaMemcpy(out + (size_t)f0 * n1, buf.data(), (size_t)(f1 - f0) * n1 * sizeof(D),
                          cudaMemcpyHostToDevice));
        }
    }
    std::vector<int> diag(n1, 0);   // G2 self-loops: W2[f][f]
    for (int f = 0; f < n; f++)
        for (int i = g2o.off[f]; i < g2o.off[f + 1]; i++)
            if (g2o.id[i] == f) diag[f] = std::min(g2o.w[i], clamp2);
    CK(dalloc(ctx, &ctx->W2D, n1 * sizeof(int)));
    CK(cudaMemcpy(ctx->W2D, diag.data(), n1 * sizeof(int), cudaMemcpyHostToDevice));
    return BM_OK;
}

static void free_ctx(bm_ctx* c) {
    if (!c) return;
    for (void* b : {(void*)c->off2oH, c->ent2oH, c->ent2oHP}) if (b) cudaFree(b);
    if (c->W2T) cudaFree(c->W2T);
    if (c->W2D) cudaFree(c->W2D);
    void* bufs[] = {c->off1o, c->off1i, c->off2o, c->off2i, c->offs, c->selfw, c->ent1o, c->ent1i,
                    c->ent2o, c->ent2i, c->ent1oP, c->ent1iP, c->ent2oP, c->ent2iP, c->W2, c->p,
                    c->pinv, c->S, c->rowbest, c->ckeys, c->ckeys_sorted, c->wkeys, c->wkeys_sorted,
                    c->wvals, c->order, c->cub_tmp, c->small, c->score_acc, c->cstats, c->scratch_pairs,
                    c->adj, c->rowd, c->first, c->fi_acc, c->tcount};
    for (void* b : bufs) if (b) cudaFree(b);
    for (auto& e : c->ev) if (e) cudaEventDestroy(e);
    for (auto& e : c->uev) if (e) cudaEventDestroy(e);
    if (c->work_sum) cudaFree(c->work_sum);
    if (c->part) cudaFree(c->part);
    if (c->diagS) cudaFree(c->diagS);
    for (void* b : {(void*)c->hubs, (void*)c->is_hub, (void*)c->hubA, (void*)c->hubB, (void*)c->hub_err})
        if (b) cudaFree(b);
    if (c->cinfo) cudaFree(c->cinfo);
    if (c->cgrid) cudaFree(c->cgrid);
    for (void* b : {(void*)c->pS, (void*)c->pinvS, (void*)c->moved, (void*)c->minfo, (void*)c->mwork})
        if (b) cudaFree(b);
    if (c->ev_hub) cudaEventDestroy(c->ev_hub);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
}

extern "C" void bm_destroy(bm_ctx* ctx) { free_ctx(ctx); }

extern "C" bm_status bm_create(bm_ctx** out, int32_t n, int64_t e1, const int32_t* src1,
                               const int32_t* dst1, const int32_t* w1, int64_t e2,
                               const int32_t* src2, const int32_t* dst2, const int32_t* w2,
                               uint32_t flags) {
    if (!out) { set_err(nullptr, "bm_create: out is NULL"); return BM_E_INPUT; }
    *out = nullptr;
    if (n < 2 || n > 65535) { set_err(nullptr, "bm_create: n=%d outside 2..65535", n); return BM_E_INPUT; }
    if (e1 < 0 || e2 < 0 || e1 > 0x7fffffff || e2 > 0x7fffffff ||
        (e1 && (!src1 || !dst1 || !w1)) || (e2 && (!src2 || !dst2 || !w2))) {
        set_err(nullptr, "bm_create: bad edge arrays");
        return BM_E_INPUT;
    }
    // ---- validate and split G1 (self-loops apart, zero weights dropped) ----
    std::vector<int> s1, d1, ww1, selfv, selfwt;
    s1.reserve(e1); d1.reserve(e1); ww1.reserve(e1);
    long long maxw1 = 0;
    for (int64_t i = 0; i < e1; i++) {
        const int a = src1[i], b = dst1[i], w = w1[i];
        if (a < 1 || a > n || b < 1 || b > n) { set_err(nullptr, "bm_create: G1 edge %lld has id outside 1..%d", (long long)i, n); return BM_E_INPUT; }
        if (w < 0) { set_err(nullptr, "bm_create: G1 edge %lld has negative weight %d", (long long)i, w); return BM_E_INPUT; }
        if (w == 0) continue;
        maxw1 = std::max<long long>(maxw1, w);
        if (a == b) { selfv.push_back(a - 1); selfwt.push_back(w); continue; }
        s1.push_back(a - 1); d1.push_back(b - 1); ww1.push_back(w);
    }
    // ---- G2: last weight per (src,dst) wins, as the dense reference matrix does ----
    std::vector<std::pair<long long, int>> keys2;   // ((src,dst) pair, input index)
    keys2.reserve(e2);
    for (int64_t i = 0; i < e2; i++) {
        const int a = src2[i], b = dst2[i], w = w2[i];
        if (a < 1 || a > n || b < 1 || b > n) { set_err(nullptr, "bm_create: G2 edge %lld has id outside 1..%d", (long long)i, n); return BM_E_INPUT; }
        if (w < 0) { set_err(nullptr, "bm_create: G2 edge %lld has negative weight %d", (long long)i, w); return BM_E_INPUT; }
        keys2.emplace_back((long long)(a - 1) * n + (b - 1), (int)i);
    }
    std::sort(keys2.begin(), keys2.end());
    std::vector<int> s2, d2, ww2;
    long long maxw2 = 0;
    for (size_t k = 0; k < keys2.size(); k++) {
        const long long pair = keys2[k].first;
        if (k + 1 < keys2.size() && keys2[k + 1].first == pair) continue;  // a later copy wins
        const int i = keys2[k].second;
        if (w2[i] == 0) continue;
        s2.push_back((int)(pair / n)); d2.push_back((int)(pair % n)); ww2.push_back(w2[i]);
        maxw2 = std::max<long long>(maxw2, w2[i]);
    }
    // ---- storage mode: 16-bit when one side's weights fit (min(w1,w2) is unchanged
    //      by clamping the other side at 65535) ----
    const bool w16 = !(flags & BM_FLAG_FORCE_I32) && std::min(maxw1, maxw2) <= 65535;
    const int clamp1 = (w16 && maxw1 > 65535) ? 65535 : 0x7fffffff;
    const int clamp2 = (w16 && maxw2 > 65535) ? 65535 : 0x7fffffff;
    // ---- overflow guard: every delta is bounded by 8 x the heaviest vertex load ----
    {
        std::vector<long long> load(n, 0);
        for (size_t i = 0; i < s1.size(); i++) { load[s1[i]] += std::min(ww1[i], clamp1); load[d1[i]] += std::min(ww1[i], clamp1); }
        for (size_t i = 0; i < selfv.size(); i++) load[selfv[i]] += 2LL * std::min(selfwt[i], clamp1);
        long long mx = 0;
        for (int v = 0; v < n; v++) mx = std::max(mx, load[v]);
        if (mx > 0x7fffffffLL / 8) {
            set_err(nullptr, "bm_create: vertex weight load %lld could overflow int32 deltas", mx);
            return BM_E_OVERFLOW;
        }
    }
    HostCSR g1o, g1i, g2o, g2i, gs;
    build_csr(n, s1, d1, ww1, g1o);
    build_csr(n, d1, s1, ww1, g1i);
    build_csr(n, s2, d2, ww2, g2o);
    build_csr(n, d2, s2, ww2, g2i);
    {
        std::vector<int> zero(selfv.size(), 0);
        build_csr(n, selfv, zero, selfwt, gs);
        for (auto& x : gs.w) x = std::min(x, clamp1);
    }

    static std::atomic<unsigned long long> next_serial{1};
    bm_ctx* ctx = new (std::nothrow) bm_ctx();
    if (ctx) ctx->serial = next_serial.fetch_add(1);
    if (!ctx) { set_err(nullptr, "bm_create: out of host memory"); return BM_E_NOMEM; }
    ctx->n = n;
    ctx->w16 = w16;
    ctx->e1 = (long long)s1.size();
    ctx->e2 = (long long)s2.size();
    ctx->nself = (long long)selfv.size();
    for (int v = 0; v < n; v++)
        ctx->max_deg1 = std::max(ctx->max_deg1, (g1o.off[v + 1] - g1o.off[v]) + (g1i.off[v + 1] - g1i.off[v]));
    auto fail = [&](bm_status s) {
        snprintf(g_create_err, sizeof g_create_err, "%s", ctx->err);
        free_ctx(ctx);
        return s;
    };
    {
        cudaError_t e = cudaGetDevice(&ctx->dev);
        if (e != cudaSuccess) { set_err(ctx, "bm_create: no CUDA device: %s", cudaGetErrorString(e)); return fail(BM_E_CUDA); }
        cudaDeviceProp prop;
        e = cudaGetDeviceProperties(&prop, ctx->dev);
        if (e != cudaSuccess) { set_err(ctx, "bm_create: %s", cudaGetErrorString(e)); return fail(BM_E_CUDA); }
        ctx->num_sms = prop.multiProcessorCount;
        ctx->smem_optin = prop.sharedMemPerBlockOptin;
    }
    auto body = [&]() -> bm_status {
        CK(cudaStreamCreateWithFlags(&ctx->st, cudaStreamNonBlocking));
        for (auto& e : ctx->ev) CK(cudaEventCreate(&e));
        for (auto& e : ctx->uev) CK(cudaEventCreate(&e));
        CK(dalloc(ctx, &ctx->work_sum, sizeof(unsigned long long)));
        auto up_off = [&](const HostCSR& h, int** d) -> bm_status {
            CK(dalloc(ctx, d, h.off.size() * sizeof(int)));
            CK(cudaMemcpy(*d, h.off.data(), h.off.size() * sizeof(int), cudaMemcpyHostToDevice));
            return BM_OK;
        };
        bm_status s;
        if ((s = up_off(g1o, &ctx->off1o)) || (s = up_off(g1i, &ctx->off1i)) ||
            (s = up_off(g2o, &ctx->off2o)) || (s = up_off(g2i, &ctx->off2i)) || (s = up_off(gs, &ctx->offs)))
            return s;
        CK(dalloc(ctx, &ctx->selfw, gs.w.size() * sizeof(int)));
        if (!gs.w.empty()) CK(cudaMemcpy(ctx->selfw, gs.w.data(), gs.w.size() * sizeof(int), cudaMemcpyHostToDevice));
        s = w16 ? upload_lists<true>(ctx, g1o, g1i, g2o, g2i, clamp1, clamp2)
                : upload_lists<false>(ctx, g1o, g1i, g2o, g2i, clamp1, clamp2);
        if (s) return s;
        s = w16 ? upload_dense<true>(ctx, g2o, g2i, clamp2) : upload_dense<false>(ctx, g2o, g2i, clamp2);
        if (s) return s;
        {   // G2 out-entries above the hub threshold (hub residual terms)
            HostCSR hv;
            hv.off.assign((size_t)n + 2, 0);
            for (int f = 0; f < n; f++) {
                int c = 0;
                for (int i = g2o.off[f]; i < g2o.off[f + 1]; i++) c += g2o.w[i] > kHubT;
                hv.off[f + 1] = hv.off[f] + c;
            }
            hv.off[n + 1] = hv.off[n];
            for (int f = 0; f < n; f++)
                for (int i = g2o.off[f]; i < g2o.off[f + 1]; i++)
                    if (g2o.w[i] > kHubT) { hv.id.push_back(g2o.id[i]); hv.w.push_back(std::min(g2o.w[i], clamp2)); }
            ctx->e2H = (long long)hv.id.size();
            if ((s = up_off(hv, &ctx->off2oH))) return s;
            s = w16 ? upload_entries<true>(ctx, hv, &ctx->ent2oH, &ctx->ent2oHP)
                    : upload_entries<false>(ctx, hv, &ctx->ent2oH, &ctx->ent2oHP);
            if (s) return s;
        }
        CK(dalloc(ctx, &ctx->p, (n + 1) * sizeof(int)));
        CK(dalloc(ctx, &ctx->pinv, (n + 1) * sizeof(int)));
        CK(cudaEventCreate(&ctx->ev_hub));
        CK(dalloc(ctx, &ctx->hub_err, sizeof(int)));
        CK(cudaMemset(ctx->hub_err, 0, sizeof(int)));
        if (!(flags & BM_FLAG_NO_HUB_GEMM)) {
            // hubs: G1 vertices of out-degree >= max(64, n/9), at most kHubMaxHubs,
            // topped up by the next-largest out-degrees to a multiple of 16 so the
            // GEMM depth (hubs x thresholds) is a multiple of 128 bytes.  A hub
            // adds n^2 x kHubT operations to the GEMM and takes out about
            // deg^2 scattered terms once hubs are matched to hubs; at
            // n = 18,524 the sweep is fastest near 256 hubs (out-degree >= n/9)
            std::vector<int> byd(n);
            for (int v = 0; v < n; v++) byd[v] = v;
            std::stable_sort(byd.begin(), byd.end(), [&](int x, int y) {
                return (g1o.off[x + 1] - g1o.off[x]) > (g1o.off[y + 1] - g1o.off[y]);
            });
            const int thr = std::max(64, n / 9);
            int nh = 0;
            while (nh < std::min(n, kHubMaxHubs) && g1o.off[byd[nh] + 1] - g1o.off[byd[nh]] >= thr) nh++;
            if (nh > 0) {
                nh = std::min(std::min(n, kHubMaxHubs), (nh + 15) / 16 * 16);
                if (nh % 16 == 0) {
                    std::vector<unsigned char> flag(n, 0);
                    std::vector<int> hv(byd.begin(), byd.begin() + nh);
                    for (int v : hv) flag[v] = 1;
                    ctx->nh = nh;
                    ctx->hubK = nh * kHubT;
                    ctx->Mpad = (n + 2 * kGemmM - 1) / (2 * kGemmM) * (2 * kGemmM);  // whole 256-row tiles
                    ctx->Npad = (n + kGemmN - 1) / kGemmN * kGemmN;
                    CK(dalloc(ctx, &ctx->hubs, nh * sizeof(int)));
                    CK(cudaMemcpy(ctx->hubs, hv.data(), nh * sizeof(int), cudaMemcpyHostToDevice));
                    CK(dalloc(ctx, &ctx->is_hub, n));
                    CK(cudaMemcpy(ctx->is_hub, flag.data(), n, cudaMemcpyHostToDevice));
                    CK(dalloc(ctx, &ctx->hubA, (size_t)ctx->Mpad * ctx->hubK));
                    CK(dalloc(ctx, &ctx->hubB, (size_t)ctx->Npad * ctx->hubK));
                }
            }
        }
        CK(dalloc(ctx, &ctx->rowbest, n * sizeof(unsigned long long)));
        CK(dalloc(ctx, &ctx->ckeys, n * sizeof(unsigned long long)));
        CK(dalloc(ctx, &ctx->ckeys_sorted, n * sizeof(unsigned long long)));
        CK(dalloc(ctx, &ctx->wkeys, n * sizeof(unsigned long long)));
        CK(dalloc(ctx, &ctx->wkeys_sorted, n * sizeof(unsigned long long)));
        CK(dalloc(ctx, &ctx->wvals, n * sizeof(int)));
        CK(dalloc(ctx, &ctx->order, n * sizeof(int)));
        CK(dalloc(ctx, &ctx->small, 16 * sizeof(int)));
        CK(dalloc(ctx, &ctx->score_acc, sizeof(unsigned long long)));
        CK(dalloc(ctx, &ctx->cstats, sizeof(CommitStats)));
        size_t b1 = 0, b2 = 0;
        CK(cub::DeviceRadixSort::SortKeys(nullptr, b1, ctx->ckeys, ctx->ckeys_sorted, n));
        CK(cub::DeviceRadixSort::SortPairsDescending(nullptr, b2, ctx->wkeys, ctx->wkeys_sorted,
                                                     ctx->wvals, ctx->order, n));
        ctx->cub_bytes = std::max(b1, b2);
        CK(dalloc(ctx, &ctx->cub_tmp, ctx->cub_bytes));
        CK(cudaDeviceSynchronize());
        return BM_OK;
    };
    bm_status s = body();
    if (s != BM_OK) return fail(s);
    *out = ctx;
    return BM_OK;
}

extern "C" bm_status bm_get_info(const bm_ctx* ctx, bm_info* info) {
    if (!ctx || !info) return BM_E_INPUT;
    info->n = ctx->n;
    info->entry_bits = ctx->w16 ? 16 : 32;
    info->e1 = ctx->e1;
    info->e2 = ctx->e2;
    info->g1_self_loops = ctx->nself;
    info->device_bytes = ctx->dev_bytes;
    info->device = ctx->dev;
    info->num_sms = ctx->num_sms;
    info->hubs = ctx->nh;
    info->hub_k = ctx->hubK;
    return BM_OK;
}

// ---------------------------------------------------------------------------
static bm_status compute_score(bm_ctx* ctx, long long* out) {
    CK(cudaMemsetAsync(ctx->score_acc, 0, sizeof(unsigned long long), ctx->st));
    const int blocks = ctx->num_sms * 4;
    if (ctx->w16) k_score<true><<<blocks, 256, 0, ctx->st>>>(view<true>(ctx), ctx->score_acc);
    else k_score<false><<<blocks, 256, 0, ctx->st>>>(view<false>(ctx), ctx->score_acc);
    CK(cudaGetLastError());
    unsigned long long v = 0;
    CK(cudaMemcpyAsync(&v, ctx->score_acc, sizeof v, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    *out = (long long)v;
    return BM_OK;
}

extern "C" bm_status bm_set_mapping(bm_ctx* ctx, const int32_t* map) {
    if (!ctx) return BM_E_INPUT;
    if (!map) { set_err(ctx, "bm_set_mapping: map is NULL"); return BM_E_INPUT; }
    const int n = ctx->n;
    std::vector<int> p(n + 1), pinv(n + 1, n);
    for (int a = 0; a < n; a++) {
        const int f = map[a + 1];
        if (f < 0 || f > n) { set_err(ctx, "bm_set_mapping: map[%d]=%d outside 0..%d", a + 1, f, n); return BM_E_INPUT; }
        if (f == 0) { p[a] = n; continue; }
        if (pinv[f - 1] != n) { set_err(ctx, "bm_set_mapping: G2 vertex %d matched twice (m%d and m%d)", f, pinv[f - 1] + 1, a + 1); return BM_E_INPUT; }
        p[a] = f - 1;
        pinv[f - 1] = a;
    }
    p[n] = n;
    pinv[n] = n;
    CK(cudaMemcpyAsync(ctx->p, p.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(ctx->pinv, pinv.data(), (n + 1) * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    ctx->mapped = true;
    ctx->work_valid = false;   // row scheduling keys are estimated afresh for a new matching
    return compute_score(ctx, &ctx->score);
}

extern "C" bm_status bm_get_mapping(bm_ctx* ctx, int32_t* map) {
    if (!ctx || !map) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_get_mapping: no mapping set"); return BM_E_STATE; }
    const int n = ctx->n;
    std::vector<int> p(n + 1);
    CK(cudaMemcpyAsync(p.data(), ctx->p, (n + 1) * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    map[0] = 0;
    for (int a = 0; a < n; a++) map[a + 1] = p[a] == n ? 0 : p[a] + 1;
    return BM_OK;
}

extern "C" bm_status bm_score(bm_ctx* ctx, int64_t* score) {
    if (!ctx || !score) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_score: no mapping set"); return BM_E_STATE; }
    long long s = 0;
    bm_status r = compute_score(ctx, &s);
    if (r) return r;
    *score = s;
    return BM_OK;
}

static bm_status ensure_scratch(bm_ctx* ctx, long long ints) {
    if (ints <= ctx->scratch_cap) return BM_OK;
    if (ctx->scratch_pairs) { cudaFree(ctx->scratch_pairs); ctx->dev_bytes -= ctx->scratch_cap * (long long)sizeof(int); }
    ctx->scratch_pairs = nullptr;
    ctx->scratch_cap = 0;
    CK(dalloc(ctx, &ctx->scratch_pairs, (size_t)ints * sizeof(int)));
    ctx->scratch_cap = ints;
    return BM_OK;
}

extern "C" bm_status bm_pair_deltas(bm_ctx* ctx, int64_t k, const int32_t* m1, const int32_t* m2,
                                    int32_t* out) {
    if (!ctx) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_pair_deltas: no mapping set"); return BM_E_STATE; }
    if (k < 0 || (k && (!m1 || !m2 || !out))) { set_err(ctx, "bm_pair_deltas: bad arguments"); return BM_E_INPUT; }
    if (k == 0) return BM_OK;
    const int n = ctx->n;
    std::vector<int> a(k), b(k);
    for (int64_t i = 0; i < k; i++) {
        if (m1[i] < 1 || m1[i] > n || m2[i] < 1 || m2[i] > n || m1[i] == m2[i]) {
            set_err(ctx, "bm_pair_deltas: pair %lld = (%d,%d) invalid", (long long)i, m1[i], m2[i]);
            return BM_E_INPUT;
        }
        a[i] = m1[i] - 1;
        b[i] = m2[i] - 1;
    }
    bm_status s = ensure_scratch(ctx, 3 * k);
    if (s) return s;
    int* da = ctx->scratch_pairs;
    int* db = da + k;
    int* dout = db + k;
    CK(cudaMemcpyAsync(da, a.data(), k * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    CK(cudaMemcpyAsync(db, b.data(), k * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    const long long blocks = std::min<long long>((k + 7) / 8, (long long)ctx->num_sms * 16);
    if (ctx->w16) k_pair_deltas<true><<<(int)blocks, 256, 0, ctx->st>>>(view<true>(ctx), da, db, k, dout);
    else k_pair_deltas<false><<<(int)blocks, 256, 0, ctx->st>>>(view<false>(ctx), da, db, k, dout);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, dout, k * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return BM_OK;
}

// ---------------------------------------------------------------------------
// Sweep stages.
// S is now exact for the current matching: remember which one.
static cudaError_t record_exact_mapping(bm_ctx* ctx) {
    const size_t bytes = (size_t)(ctx->n + 1) * sizeof(int);
    cudaError_t e = cudaSuccess;
    if (!ctx->pS) e = dalloc(ctx, &ctx->pS, bytes);
    if (e == cudaSuccess && !ctx->pinvS) e = dalloc(ctx, &ctx->pinvS, bytes);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->pS, ctx->p, bytes, cudaMemcpyDeviceToDevice, ctx->st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(ctx->pinvS, ctx->pinv, bytes, cudaMemcpyDeviceToDevice, ctx->st);
    ctx->S_exact = e == cudaSuccess;
    return e;
}

bm_status ensure_S(bm_ctx* ctx) {
    if (ctx->S) return BM_OK;
    CK(dalloc(ctx, &ctx->S, (size_t)ctx->n * ctx->n * sizeof(int)));
    return BM_OK;
}

template <bool W16>
bm_status stage_profit(bm_ctx* ctx) {
    typedef typename Ent<W16>::T E;
    DevView<W16> g = view<W16>(ctx);
    const int n = ctx->n;
    ctx->S_exact = false;
    const int rb = ctx->num_sms * 8;
    k_relabel<W16><<<rb, 256, 0, ctx->st>>>((const E*)ctx->ent1o, (E*)ctx->ent1oP, ctx->e1, ctx->p);
    k_relabel<W16><<<rb, 256, 0, ctx->st>>>((const E*)ctx->ent1i, (E*)ctx->ent1iP, ctx->e1, ctx->p);
    k_relabel<W16><<<rb, 256, 0, ctx->st>>>((const E*)ctx->ent2o, (E*)ctx->ent2oP, ctx->e2, ctx->pinv);
    k_relabel<W16><<<rb, 256, 0, ctx->st>>>((const E*)ctx->ent2i, (E*)ctx->ent2iP, ctx->e2, ctx->pinv);
    if (ctx->nh && ctx->e2H)
        k_relabel<W16><<<rb, 256, 0, ctx->st>>>((const E*)ctx->ent2oH, (E*)ctx->ent2oHP, ctx->e2H, ctx->pinv);
    CK(cudaGetLastError());
    // heaviest rows first: each rebuild records its rows' work for the next
    // one; after a new matching the estimate is computed afresh
    if (!ctx->work_valid) {
        k_row_work<W16><<<(n + 7) / 8, 256, 0, ctx->st>>>(g, ctx->is_hub, ctx->wkeys, ctx->wvals, nullptr);
        CK(cudaGetLastError());
    }
    CK(cudaMemsetAsync(ctx->work_sum, 0, sizeof(unsigned long long), ctx->st));
    size_t tb = ctx->cub_bytes;
    CK(cub::DeviceRadixSort::SortPairsDescending(ctx->cub_tmp, tb, ctx->wkeys, ctx->wkeys_sorted,
                                                 ctx->wvals, ctx->order, n, 0, 32, ctx->st));
    CK(cudaMemsetAsync(ctx->small, 0, sizeof(int), ctx->st));
    CK(cudaEventRecord(ctx->ev_hub, ctx->st));
    if (ctx->nh) {
        // hub in-edge terms up to the threshold: one exact u8 GEMM on the tensor cores into S
        const int K = ctx->hubK;
        if (!ctx->hubA_built) {
            CK(cudaMemsetAsync(ctx->hubA, 0, (size_t)ctx->Mpad * K, ctx->st));
            k_hub_build_A<W16><<<ctx->nh, 256, 0, ctx->st>>>(g, ctx->hubs, ctx->nh, K, ctx->hubA);
            CK(cudaGetLastError());
            ctx->hubA_built = true;
        }
        CK(cudaMemsetAsync(ctx->hubB, 0, (size_t)ctx->Npad * K, ctx->st));
        k_hub_build_B<W16><<<dim3(ctx->nh, 8), 256, 0, ctx->st>>>(g, ctx->hubs, ctx->nh, K, ctx->hubB);
        CK(cudaGetLastError());
        if (!ctx->hub_ws_ready) {
            ctx->hub_ws_ready = true;
            ctx->hub_ws = hub_ws_setup(ctx);
        }
        const int mt = ctx->Mpad / kGemmM, nt = ctx->Npad / kGemmN;
        if (ctx->hub_ws) {
            const int mw = ctx->Mpad / kWsM;
            const int grid = std::min(ctx->num_sms, mw * nt);
            k_hub_gemm_ws<<<grid, kWsThreads, kWsSmem, ctx->st>>>(ctx->tmHubA, ctx->tmHubB, K, n, mw, nt, ctx->S,
                                                                 ctx->hub_err, take_stall(BM_STALL_HUB_GEMM));
        } else {
            CK(cudaFuncSetAttribute(k_hub_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kGemmSmem));
            k_hub_gemm<<<dim3(nt, mt), kGemmThreads, kGemmSmem, ctx->st>>>(ctx->hubA, ctx->hubB, K, n, ctx->S,
                                                                         ctx->hub_err, take_stall(BM_STALL_HUB_GEMM));
        }
        CK(cudaGetLastError());
    }
    const size_t smem = (size_t)(n + 1) * sizeof(int);
    CK(cudaFuncSetAttribute(k_profit<W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_profit<W16>, 512, smem));
    if (per_sm < 1) { set_err(ctx, "profit kernel does not fit (n=%d)", n); return BM_E_INPUT; }
    CK(cudaEventRecord(ctx->ev[4], ctx->st));
    k_profit<W16><<<ctx->num_sms * per_sm, 512, smem, ctx->st>>>(g, ctx->order, ctx->small,
                                                                ctx->nh ? ctx->is_hub : nullptr, kHubT,
                                                                ctx->wkeys, ctx->work_sum);
    CK(cudaGetLastError());
    ctx->work_valid = true;
    CK(record_exact_mapping(ctx));
    CK(cudaEventRecord(ctx->ev[5], ctx->st));
    return BM_OK;
}

template bm_status stage_profit<true>(bm_ctx*);
template bm_status stage_profit<false>(bm_ctx*);

static bm_status ensure_moved(bm_ctx* ctx) {
    if (ctx->moved) return BM_OK;
    CK(dalloc(ctx, &ctx->moved, (size_t)ctx->n * sizeof(int)));
    CK(dalloc(ctx, &ctx->minfo, 4 * sizeof(int)));
    CK(dalloc(ctx, &ctx->mwork, 3 * sizeof(unsigned long long)));
    return BM_OK;
}

// Step 3's row path (k_terms_rows): up to 256 edge slots per moved vertex.
template <bool W16>
static cudaError_t launch_terms_rows(bm_ctx* ctx, const DevView<W16>& g, int count, const int* dcount, int maxd) {
    const size_t smem = (size_t)(ctx->n + 1) * sizeof(int);
    cudaError_t e = cudaFuncSetAttribute(k_terms_rows<W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    dim3 grid(count, std::min(maxd, 256));
    k_terms_rows<W16><<<grid, kIncrRowThreads, smem, ctx->st>>>(g, ctx->pS, ctx->moved, count, dcount);
    return cudaGetLastError();
}

template <bool W16>
bm_status stage_refresh(bm_ctx* ctx, int* mode) {
    *mode = 0;
    if (!ctx->S_exact) return stage_profit<W16>(ctx);
    const int n = ctx->n;
    {
        const bm_status sm = ensure_moved(ctx);
        if (sm) return sm;
    }
    DevView<W16> g = view<W16>(ctx);
    CK(cudaMemsetAsync(ctx->minfo, 0, 4 * sizeof(int), ctx->st));
    CK(cudaMemsetAsync(ctx->mwork, 0, 3 * sizeof(unsigned long long), ctx->st));
    k_moved<W16><<<ctx->num_sms * 2, 256, 0, ctx->st>>>(g, ctx->pS, ctx->pinvS, ctx->moved, ctx->minfo, ctx->mwork);
    CK(cudaGetLastError());
    int info[4];
    unsigned long long work[3] = {0, 0, 0}, full = 0;
    CK(cudaMemcpyAsync(info, ctx->minfo, sizeof info, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(work, ctx->mwork, sizeof work, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&full, ctx->work_sum, sizeof full, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    CK(cudaEventRecord(ctx->ev_hub, ctx->st));
    CK(cudaEventRecord(ctx->ev[4], ctx->st));
    const int count = info[0];
    ctx->upd_work = (long long)work[2];
    if (count == 0) {
        *mode = 2;
        CK(cudaEventRecord(ctx->ev[5], ctx->st));
        return BM_OK;
    }
    // an atomic into S costs about kIncrAtomicCost shared-memory terms of a
    // rebuild, a row written whole kIncrRowCost per column, a permuted column
    // entry kIncrPermCost
    const double est = kIncrAtomicCost * (double)work[0] + kIncrRowCost * (double)n * (double)work[1] +
                       kIncrPermCost * (double)n * count;
    const bool rows_fit = (size_t)(n + 1) * sizeof(int) + 1024 <= ctx->smem_optin;
    if (info[1] || count > kIncrMaxMoved || est >= (double)full || (work[1] && !rows_fit))
        return stage_profit<W16>(ctx);
    const int maxd = std::max(info[2], 1);
    ctx->S_exact = false;
    {
        dim3 grid(count, (maxd + kIncrCornerEdges - 1) / kIncrCornerEdges);
        k_corner<W16><<<grid, kIncrCornerEdges, 0, ctx->st>>>(g, ctx->pS, ctx->pS, ctx->moved, count, nullptr, -1);
        CK(cudaGetLastError());
    }
    {
        const size_t smem = 3 * (size_t)count * sizeof(int);
        CK(cudaFuncSetAttribute(k_perm_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        const int blocks = std::min(n, ctx->num_sms * (smem <= 48 * 1024 ? 4 : 1));
        k_perm_cols<<<blocks, 512, smem, ctx->st>>>(ctx->S, n, ctx->moved, count, ctx->p, ctx->pinvS);
        CK(cudaGetLastError());
    }
    {
        dim3 grid(count, (maxd + kIncrEdgesPerBlock - 1) / kIncrEdgesPerBlock);
        k_terms<W16><<<grid, 256, 0, ctx->st>>>(g, ctx->pS, ctx->moved, count, nullptr);
        CK(cudaGetLastError());
        if (work[1]) CK(launch_terms_rows<W16>(ctx, g, count, nullptr, maxd));
    }
    {
        dim3 grid(count, (maxd + kIncrCornerEdges - 1) / kIncrCornerEdges);
        k_corner<W16><<<grid, kIncrCornerEdges, 0, ctx->st>>>(g, ctx->p, ctx->pS, ctx->moved, count, nullptr, 1);
        CK(cudaGetLastError());
    }
    CK(record_exact_mapping(ctx));
    CK(cudaEventRecord(ctx->ev[5], ctx->st));
    *mode = 1;
    return BM_OK;
}

template bm_status stage_refresh<true>(bm_ctx*, int*);
template bm_status stage_refresh<false>(bm_ctx*, int*);

// The tensor map of S for the TMA-fed combine: rows of n int32, 64x64 boxes,
// zero fill outside the matrix.  Needs the row stride (4n bytes) to be a
// multiple of 16; returns false (the caller keeps k_combine64) otherwise.
static PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    });
    return encode;
}

// Tensor maps of the hub GEMM's u8 operands (rows of K bytes; boxes of one
// 128-byte K-chunk of 256 A rows or 256 B rows, 128-byte swizzle) for the
// persistent warp-specialised kernel; false keeps the one-tile-per-CTA kernel.
static bool hub_ws_setup(bm_ctx* ctx) {
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode || ctx->hubK % kGemmKC != 0) return false;
    const cuuint32_t estr[2] = {1, 1};
    const cuuint64_t dA[2] = {(cuuint64_t)ctx->hubK, (cuuint64_t)ctx->Mpad};
    const cuuint64_t dB[2] = {(cuuint64_t)ctx->hubK, (cuuint64_t)ctx->Npad};
    const cuuint64_t st[1] = {(cuuint64_t)ctx->hubK};
    const cuuint32_t bA[2] = {kGemmKC, kWsM}, bB[2] = {kGemmKC, kGemmN};
    if (encode(&ctx->tmHubA, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, ctx->hubA, dA, st, bA, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    if (encode(&ctx->tmHubB, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, ctx->hubB, dB, st, bB, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    if (cudaFuncSetAttribute(k_hub_gemm_ws, cudaFuncAttributeMaxDynamicSharedMemorySize, kWsSmem) != cudaSuccess)
        return false;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_hub_gemm_ws, kWsThreads, kWsSmem) != cudaSuccess ||
        per_sm != 1)
        return false;
    return true;
}

static bool combine_tma_setup(bm_ctx* ctx) {
    const int n = ctx->n;
    if ((n & 3) != 0 || n < kCmbT) return false;
    PFN_cuTensorMapEncodeTiled_v12000 encode = tensor_map_encoder();
    if (!encode) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)n, (cuuint64_t)n};
    const cuuint64_t strides[1] = {(cuuint64_t)n * sizeof(int)};
    const cuuint32_t box[2] = {kCmbT, kCmbT};
    const cuuint32_t estr[2] = {1, 1};
    if (encode(&ctx->tmS, CU_TENSOR_MAP_DATA_TYPE_INT32, 2, ctx->S, dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return false;
    if (cudaFuncSetAttribute(k_combine_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, kCmbSmem) != cudaSuccess)
        return false;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_combine_tma, kCmbThreads, kCmbSmem) != cudaSuccess ||
        per_sm < 1)
        return false;
    if (dalloc(ctx, &ctx->diagS, (size_t)n * sizeof(int)) != cudaSuccess) return false;
    ctx->cmb_grid = ctx->num_sms * per_sm;
    return true;
}

bm_status stage_combine(bm_ctx* ctx, int* all_out) {
    const int n = ctx->n;
    const int t = (n + kTile - 1) / kTile;
    if (!ctx->part) CK(dalloc(ctx, &ctx->part, (size_t)t * n * sizeof(unsigned long long)));
    if (!ctx->cmb_ready) {
        ctx->cmb_ready = true;
        if (!combine_tma_setup(ctx)) ctx->cmb_grid = 0;
    }
    if (!all_out && ctx->cmb_grid > 0) {
        k_diag<<<(n + 255) / 256, 256, 0, ctx->st>>>(ctx->S, n, ctx->diagS);
        const long long pairs = (long long)t * (t + 1) / 2;
        const int grid = (int)std::min<long long>(ctx->cmb_grid, pairs);
        k_combine_tma<<<grid, kCmbThreads, kCmbSmem, ctx->st>>>(ctx->tmS, ctx->diagS, n, t, ctx->part,
                                                                 ctx->hub_err, take_stall(BM_STALL_COMBINE));
    } else {
        dim3 grid(t, t);
        k_combine64<<<grid, 256, 0, ctx->st>>>(ctx->S, n, ctx->part, all_out);
    }
    CK(cudaGetLastError());
    k_best_reduce<<<(n + 255) / 256, 256, 0, ctx->st>>>(ctx->part, n, t, ctx->rowbest);
    CK(cudaGetLastError());
    return BM_OK;
}

// G1 adjacency bitmap (x -> y), built once on first use.
template <bool W16>
static bm_status ensure_adj(bm_ctx* ctx) {
    if (ctx->adj) return BM_OK;
    const int n = ctx->n;
    ctx->adj_words = (n + 31) / 32;
    const size_t bytes = (size_t)n * ctx->adj_words * sizeof(unsigned);
    CK(dalloc(ctx, &ctx->adj, bytes));
    CK(cudaMemsetAsync(ctx->adj, 0, bytes, ctx->st));
    k_adj_bits<W16><<<(n + 7) / 8, 256, 0, ctx->st>>>(view<W16>(ctx), ctx->adj, ctx->adj_words);
    CK(cudaGetLastError());
    return BM_OK;
}

template <bool W16>
static bm_status stage_commit(bm_ctx* ctx, const bm_sweep_opts* o) {
    const int n = ctx->n;
    CK(cudaMemsetAsync(ctx->small + 1, 0, 2 * sizeof(int), ctx->st));
    k_candidates<<<(n + 255) / 256, 256, 0, ctx->st>>>(ctx->rowbest, n, ctx->ckeys, ctx->small + 1, ctx->small + 2);
    CK(cudaGetLastError());
    size_t tb = ctx->cub_bytes;
    CK(cub::DeviceRadixSort::SortKeys(ctx->cub_tmp, tb, ctx->ckeys, ctx->ckeys_sorted, n, 0, 64, ctx->st));
    const int max_scan = o ? o->max_candidates : 0;
    const int max_verify = o ? o->max_verify : -1;
    const int lim = (max_scan > 0 && max_scan < n) ? max_scan : n;
    {   // G1 lists and offsets into L2 for the commit's scattered list reads
        const size_t es = W16 ? 4 : 8;
        k_prefetch_l2<<<ctx->num_sms * 4, 256, 0, ctx->st>>>((const char*)ctx->ent1o, (size_t)ctx->e1 * es);
        k_prefetch_l2<<<ctx->num_sms * 4, 256, 0, ctx->st>>>((const char*)ctx->ent1i, (size_t)ctx->e1 * es);
        k_prefetch_l2<<<ctx->num_sms, 256, 0, ctx->st>>>((const char*)ctx->off1o, (size_t)(n + 2) * sizeof(int));
        k_prefetch_l2<<<ctx->num_sms, 256, 0, ctx->st>>>((const char*)ctx->off1i, (size_t)(n + 2) * sizeof(int));
        CK(cudaGetLastError());
    }
    if (!ctx->cinfo) CK(dalloc(ctx, &ctx->cinfo, (size_t)n * 2 * sizeof(int4)));
    k_cand_info<W16><<<(lim + 255) / 256, 256, 0, ctx->st>>>(view<W16>(ctx), ctx->ckeys_sorted, lim, ctx->cinfo);
    CK(cudaGetLastError());
    const size_t smem = commit_group_smem(n);
    if (smem + 4096 > ctx->smem_optin) {
        set_err(ctx, "set commit needs %zu bytes of shared memory for n=%d (limit %zu): n too large for a sweep",
                smem, n, ctx->smem_optin);
        return BM_E_INPUT;
    }
    int ctas = o && o->commit_ctas > 0 ? o->commit_ctas : kCommitDefaultCtas;
    ctas = std::min(std::min(ctas, kCommitMaxCtas), ctx->num_sms);
    if (!ctx->cgrid) {
        CK(dalloc(ctx, &ctx->cgrid, commit_grid_ints() * sizeof(int)));
        CK(cudaMemset(ctx->cgrid, 0, commit_grid_ints() * sizeof(int)));
    }
    CK(launch_commit_group<W16>(view<W16>(ctx), ctx->ckeys_sorted, lim, max_verify, ctx->cstats, ctx->cinfo, ctas,
                                ctx->cgrid, smem, ctx->st, ctas > 1 ? take_stall(BM_STALL_COMMIT) : 0));
    return BM_OK;
}

extern "C" bm_status bm_all_deltas(bm_ctx* ctx, int32_t* out) {
    if (!ctx || !out) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_all_deltas: no mapping set"); return BM_E_STATE; }
    bm_status s = ensure_S(ctx);
    if (s) return s;
    const long long np = (long long)ctx->n * (ctx->n - 1) / 2;
    int* d = nullptr;
    CK(cudaMalloc(&d, np * sizeof(int)));
    s = ctx->w16 ? stage_profit<true>(ctx) : stage_profit<false>(ctx);
    if (!s) s = stage_combine(ctx, d);
    if (!s) {
        cudaError_t e = cudaMemcpyAsync(out, d, np * sizeof(int), cudaMemcpyDeviceToHost, ctx->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
        if (e != cudaSuccess) { set_err(ctx, "bm_all_deltas: %s", cudaGetErrorString(e)); s = BM_E_CUDA; }
    }
    cudaFree(d);
    return s;
}

extern "C" bm_status bm_profit_row(bm_ctx* ctx, int32_t a, int32_t* out) {
    if (!ctx || !out) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_profit_row: no mapping set"); return BM_E_STATE; }
    if (a < 1 || a > ctx->n) { set_err(ctx, "bm_profit_row: a=%d outside 1..%d", a, ctx->n); return BM_E_INPUT; }
    bm_status s = ensure_S(ctx);
    if (s) return s;
    s = ctx->w16 ? stage_profit<true>(ctx) : stage_profit<false>(ctx);
    if (s) return s;
    CK(cudaMemcpyAsync(out, ctx->S + (size_t)(a - 1) * ctx->n, ctx->n * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return BM_OK;
}

extern "C" bm_status bm_sweep(bm_ctx* ctx, const bm_sweep_opts* opts, bm_sweep_stats* stats) {
    if (!ctx) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_sweep: no mapping set"); return BM_E_STATE; }
    bm_status s = ensure_S(ctx);
    if (s) return s;
    const long long before = ctx->score;
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    int mode = 0;
    if (opts && opts->incremental)
        s = ctx->w16 ? stage_refresh<true>(ctx, &mode) : stage_refresh<false>(ctx, &mode);
    else
        s = ctx->w16 ? stage_profit<true>(ctx) : stage_profit<false>(ctx);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    s = stage_combine(ctx, nullptr);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    s = ctx->w16 ? stage_commit<true>(ctx, opts) : stage_commit<false>(ctx, opts);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[3], ctx->st));
    CommitStats cs;
    int small[3];
    unsigned long long terms = 0;
    int herr = 0, cerr = 0;
    CK(cudaMemcpyAsync(&cs, ctx->cstats, sizeof cs, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(small, ctx->small, 3 * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&terms, ctx->work_sum, sizeof terms, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(&herr, ctx->hub_err, sizeof herr, cudaMemcpyDeviceToHost, ctx->st));
    if (ctx->cgrid)
        CK(cudaMemcpyAsync(&cerr, ctx->cgrid, sizeof cerr, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    if (herr || cerr) {
        // the matching may be partly committed and S is not trusted: the
        // caller sets a matching again before the next call
        set_err(ctx, "bm_sweep: %s wait timed out",
                (herr & (1 << kCmbErrBit)) ? "pair combine tile" : herr ? "tensor-core hub GEMM"
                                                                        : "set commit cluster barrier");
        if (herr) CK(cudaMemset(ctx->hub_err, 0, sizeof(int)));
        ctx->mapped = false;
        ctx->S_exact = false;
        return BM_E_TIMEOUT;
    }
    ctx->score = before + cs.total_delta;
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->score_before = before;
        stats->score_after = ctx->score;
        stats->deltas_evaluated = (long long)ctx->n * (ctx->n - 1) / 2;
        stats->candidates = small[1];
        stats->best_delta = small[2];
        stats->profit_mode = mode;
        stats->scanned = cs.scanned;
        stats->verified = cs.verified;
        stats->committed = cs.committed;
        cudaEventElapsedTime(&stats->ms_prep, ctx->ev[0], ctx->ev_hub);
        cudaEventElapsedTime(&stats->ms_hub, ctx->ev_hub, ctx->ev[4]);
        cudaEventElapsedTime(&stats->ms_profit, ctx->ev[4], ctx->ev[5]);
        cudaEventElapsedTime(&stats->ms_combine, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&stats->ms_commit, ctx->ev[2], ctx->ev[3]);
        cudaEventElapsedTime(&stats->ms_total, ctx->ev[0], ctx->ev[3]);
        stats->min_terms = mode == 1 ? ctx->upd_work : mode == 2 ? 0 : (long long)terms;
        stats->commit_entries = cs.entries;
        stats->commit_steps = cs.steps;
        stats->commit_carried = cs.carried;
    }
    return BM_OK;
}

// ---------------------------------------------------------------------------
// Exact swap-lookup table (src/best-swap/create-score-lookup.c:289-296,
// src/best-swap/score-lookup.c:514-640): the table is the profit matrix, kept
// exact by the moved-vertex update; the heap is the per-row best partners.

extern "C" bm_status bm_lookup_rows(bm_ctx* ctx, int32_t a0, int32_t rows, int32_t* out) {
    if (!ctx || !out || rows < 0) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_lookup_rows: no mapping set"); return BM_E_STATE; }
    if (a0 < 1 || (long long)a0 + rows - 1 > ctx->n) {
        set_err(ctx, "bm_lookup_rows: rows %d..%lld outside 1..%d", a0, (long long)a0 + rows - 1, ctx->n);
        return BM_E_INPUT;
    }
    if (rows == 0) return BM_OK;
    bm_status s = ensure_S(ctx);
    if (s) return s;
    int mode = 0;
    s = ctx->w16 ? stage_refresh<true>(ctx, &mode) : stage_refresh<false>(ctx, &mode);
    if (s) return s;
    const long long total = (long long)rows * ctx->n;
    if ((s = ensure_scratch(ctx, total))) return s;
    k_delta_rows<<<ctx->num_sms * 8, 256, 0, ctx->st>>>(ctx->S, ctx->n, a0 - 1, rows, ctx->scratch_pairs);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, ctx->scratch_pairs, total * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return BM_OK;
}

template <bool W16>
static bm_status lookup_descent_impl(bm_ctx* ctx, int max_swaps, bm_lookup_stats* st) {
    const int n = ctx->n;
    if ((size_t)(n + 1) * sizeof(int) + 1024 > ctx->smem_optin) {
        set_err(ctx, "bm_lookup_descent: n=%d needs a %zu-byte shared-memory row (limit %zu)", n,
                (size_t)(n + 1) * sizeof(int), ctx->smem_optin);
        return BM_E_INPUT;
    }
    bm_status s = ensure_S(ctx);
    if (!s) s = ensure_moved(ctx);
    if (s) return s;
    if (!ctx->fi_acc) CK(dalloc(ctx, &ctx->fi_acc, 2 * sizeof(long long)));
    const long long before = ctx->score;
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    int mode = 0;
    s = stage_refresh<W16>(ctx, &mode);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    CK(cudaMemsetAsync(ctx->minfo, 0, 4 * sizeof(int), ctx->st));
    CK(cudaMemsetAsync(ctx->fi_acc, 0, 2 * sizeof(long long), ctx->st));
    DevView<W16> g = view<W16>(ctx);
    const int maxd = std::max(ctx->max_deg1, 1);
    const dim3 gc(2, (maxd + kIncrCornerEdges - 1) / kIncrCornerEdges);
    const dim3 gt(2, (maxd + kIncrEdgesPerBlock - 1) / kIncrEdgesPerBlock);
    const int pblocks = std::max(1, std::min((n + 255) / 256, ctx->num_sms * 4));
    int info[4] = {0, 0, 0, 0};
    long long acc[2] = {0, 0};
    int done = 0;
    while (done < max_swaps && !info[3]) {
        const int batch = std::min(kLookupBatch, max_swaps - done);
        for (int k = 0; k < batch; k++) {
            s = stage_combine(ctx, nullptr);
            if (s) return s;
            k_pick_commit<<<1, 1024, 0, ctx->st>>>(ctx->rowbest, n, ctx->p, ctx->pinv, ctx->moved, ctx->minfo,
                                                   ctx->fi_acc);
            k_corner<W16><<<gc, kIncrCornerEdges, 0, ctx->st>>>(g, ctx->pS, ctx->pS, ctx->moved, 2, ctx->minfo, -1);
            k_perm_cols_small<<<pblocks, 256, 0, ctx->st>>>(ctx->S, n, ctx->moved, ctx->minfo, ctx->p, ctx->pinvS);
            k_terms<W16><<<gt, 256, 0, ctx->st>>>(g, ctx->pS, ctx->moved, 2, ctx->minfo);
            CK(launch_terms_rows<W16>(ctx, g, 2, ctx->minfo, maxd));
            k_corner<W16><<<gc, kIncrCornerEdges, 0, ctx->st>>>(g, ctx->p, ctx->pS, ctx->moved, 2, ctx->minfo, 1);
            k_sync_exact<<<1, 32, 0, ctx->st>>>(ctx->moved, ctx->minfo, ctx->p, ctx->pS, ctx->pinvS, n);
            CK(cudaGetLastError());
        }
        done += batch;
        CK(cudaMemcpyAsync(info, ctx->minfo, sizeof info, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaMemcpyAsync(acc, ctx->fi_acc, sizeof acc, cudaMemcpyDeviceToHost, ctx->st));
        CK(cudaStreamSynchronize(ctx->st));
    }
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    CK(cudaEventSynchronize(ctx->ev[2]));
    {
        int herr = 0;
        CK(cudaMemcpy(&herr, ctx->hub_err, sizeof herr, cudaMemcpyDeviceToHost));
        if (herr & (1 << kCmbErrBit)) {
            set_err(ctx, "bm_lookup_descent: pair combine tile wait timed out");
            CK(cudaMemset(ctx->hub_err, 0, sizeof(int)));
            ctx->mapped = false;
            ctx->S_exact = false;
            return BM_E_TIMEOUT;
        }
    }
    ctx->score = before + acc[0];
    if (st) {
        memset(st, 0, sizeof *st);
        st->score_before = before;
        st->score_after = ctx->score;
        st->swaps = (int32_t)acc[1];
        st->converged = info[3] ? 1 : 0;
        st->refresh_mode = mode;
        cudaEventElapsedTime(&st->ms_refresh, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&st->ms_total, ctx->ev[0], ctx->ev[2]);
    }
    return BM_OK;
}

extern "C" bm_status bm_lookup_descent(bm_ctx* ctx, int32_t max_swaps, bm_lookup_stats* stats) {
    if (!ctx || max_swaps < 0) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_lookup_descent: no mapping set"); return BM_E_STATE; }
    return ctx->w16 ? lookup_descent_impl<true>(ctx, max_swaps, stats) : lookup_descent_impl<false>(ctx, max_swaps, stats);
}

extern "C" bm_status bm_timer_mark(bm_ctx* ctx, int32_t slot) {
    if (!ctx || slot < 0 || slot >= 8) return BM_E_INPUT;
    CK(cudaEventRecord(ctx->uev[slot], ctx->st));
    return BM_OK;
}

extern "C" bm_status bm_timer_elapsed(bm_ctx* ctx, int32_t a, int32_t b, float* ms) {
    if (!ctx || !ms || a < 0 || a >= 8 || b < 0 || b >= 8) return BM_E_INPUT;
    CK(cudaEventSynchronize(ctx->uev[b]));
    CK(cudaEventElapsedTime(ms, ctx->uev[a], ctx->uev[b]));
    return BM_OK;
}

extern "C" bm_status bm_hillclimb(bm_ctx* ctx, int32_t max_sweeps, const bm_sweep_opts* opts,
                                  bm_sweep_stats* per_sweep, int32_t* sweeps_done) {
    if (!ctx || max_sweeps < 0) return BM_E_INPUT;
    int done = 0;
    for (; done < max_sweeps; done++) {
        bm_sweep_stats st;
        bm_status s = bm_sweep(ctx, opts, &st);
        if (s) { if (sweeps_done) *sweeps_done = done; return s; }
        if (per_sweep) per_sweep[done] = st;
        if (st.committed == 0) { done++; break; }
    }
    if (sweeps_done) *sweeps_done = done;
    return BM_OK;
}

// ---------------------------------------------------------------------------
// Reference-order first improvement (src/graph-alignment-optimized.c:515-577).
__global__ void k_first_reset(int* first, int n) { first[0] = n; }
__global__ void k_first_publish(int* first, int n) { first[1] = first[0]; first[0] = n; }

template <bool W16>
static bm_status first_improvement_impl(bm_ctx* ctx, int max_passes, long long* commits, int* passes) {
    const int n = ctx->n;
    if (!ctx->rowd) CK(dalloc(ctx, &ctx->rowd, n * sizeof(int)));
    if (!ctx->first) CK(dalloc(ctx, &ctx->first, 2 * sizeof(int)));
    if (!ctx->fi_acc) CK(dalloc(ctx, &ctx->fi_acc, 2 * sizeof(long long)));
    CK(cudaMemsetAsync(ctx->fi_acc, 0, 2 * sizeof(long long), ctx->st));
    k_first_reset<<<1, 1, 0, ctx->st>>>(ctx->first, n);
    DevView<W16> g = view<W16>(ctx);
    long long total = 0;
    int pass = 0;
    const int blocks = std::min((n + 7) / 8, ctx->num_sms * 16);
    for (; pass < max_passes; pass++) {
        long long in_pass = 0;
        for (int m1 = 0; m1 < n; m1++) {
            int start = 0;
            while (start < n) {
                k_row_first<W16><<<blocks, 256, 0, ctx->st>>>(g, m1, start, ctx->rowd, ctx->first);
                k_apply_first<<<1, 1, 0, ctx->st>>>(ctx->p, ctx->pinv, n, m1, ctx->first, ctx->rowd, ctx->fi_acc);
                k_first_publish<<<1, 1, 0, ctx->st>>>(ctx->first, n);
                CK(cudaGetLastError());
                int m2 = n;
                CK(cudaMemcpyAsync(&m2, ctx->first + 1, sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
                CK(cudaStreamSynchronize(ctx->st));
                if (m2 >= n) break;
                in_pass++;
                start = m2 + 1;
            }
        }
        total += in_pass;
        if (in_pass == 0) { pass++; break; }
    }
    long long acc[2] = {0, 0};
    CK(cudaMemcpyAsync(acc, ctx->fi_acc, sizeof acc, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->score += acc[0];
    *commits = total;
    *passes = pass;
    return BM_OK;
}

extern "C" bm_status bm_first_improvement(bm_ctx* ctx, int32_t max_passes, int64_t* commits,
                                          int32_t* passes_done) {
    if (!ctx || max_passes < 0) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_first_improvement: no mapping set"); return BM_E_STATE; }
    long long c = 0;
    int p = 0;
    bm_status s = ctx->w16 ? first_improvement_impl<true>(ctx, max_passes, &c, &p)
                           : first_improvement_impl<false>(ctx, max_passes, &c, &p);
    if (commits) *commits = c;
    if (passes_done) *passes_done = p;
    return s;
}

// ---------------------------------------------------------------------------
// 3-cycles.
extern "C" bm_status bm_triple_deltas(bm_ctx* ctx, int64_t k, const int32_t* a, const int32_t* b,
                                      const int32_t* c, int32_t* out) {
    if (!ctx) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_triple_deltas: no mapping set"); return BM_E_STATE; }
    if (k < 0 || (k && (!a || !b || !c || !out))) { set_err(ctx, "bm_triple_deltas: bad arguments"); return BM_E_INPUT; }
    if (k == 0) return BM_OK;
    const int n = ctx->n;
    std::vector<int> h(3 * k);
    for (int64_t i = 0; i < k; i++) {
        const int x = a[i], y = b[i], z = c[i];
        if (x < 1 || x > n || y < 1 || y > n || z < 1 || z > n || x == y || y == z || x == z) {
            set_err(ctx, "bm_triple_deltas: triple %lld = (%d,%d,%d) invalid", (long long)i, x, y, z);
            return BM_E_INPUT;
        }
        h[i] = x - 1; h[k + i] = y - 1; h[2 * k + i] = z - 1;
    }
    bm_status s = ensure_scratch(ctx, 5 * k);
    if (s) return s;
    int* d = ctx->scratch_pairs;
    CK(cudaMemcpyAsync(d, h.data(), 3 * k * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    const long long blocks = std::min<long long>((k + 7) / 8, (long long)ctx->num_sms * 16);
    if (ctx->w16) k_triple_deltas<true><<<(int)blocks, 256, 0, ctx->st>>>(view<true>(ctx), d, d + k, d + 2 * k, k, d + 3 * k);
    else k_triple_deltas<false><<<(int)blocks, 256, 0, ctx->st>>>(view<false>(ctx), d, d + k, d + 2 * k, k, d + 3 * k);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, d + 3 * k, 2 * k * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return BM_OK;
}

template <bool W16>
static bm_status triple_round_impl(bm_ctx* ctx, const bm_triple_opts* o, bm_triple_stats* stats) {
    const int n = ctx->n;
    const int partners = o->partners > 0 ? o->partners : 256;
    if (partners > 32768) { set_err(ctx, "bm_triple_round: partners=%d above 32768", partners); return BM_E_INPUT; }
    bm_status s = ensure_S(ctx);
    if (s) return s;
    s = ensure_adj<W16>(ctx);
    if (s) return s;
    if (!ctx->tcount) CK(dalloc(ctx, &ctx->tcount, 2 * sizeof(unsigned long long)));
    const long long before = ctx->score;
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    int mode = 0;
    s = (o && o->incremental) ? stage_refresh<W16>(ctx, &mode) : stage_profit<W16>(ctx);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    CK(cudaMemsetAsync(ctx->tcount, 0, 2 * sizeof(unsigned long long), ctx->st));
    const int blocks = std::min(n, ctx->num_sms * 8);
    k_triple_eval<W16><<<blocks, 256, 0, ctx->st>>>(view<W16>(ctx), ctx->adj, ctx->adj_words, partners,
                                                    o->seed, ctx->ckeys, ctx->tcount);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    size_t tb = ctx->cub_bytes;
    CK(cub::DeviceRadixSort::SortKeys(ctx->cub_tmp, tb, ctx->ckeys, ctx->ckeys_sorted, n, 0, 64, ctx->st));
    const size_t smem = 2 * (size_t)n;
    CK(cudaFuncSetAttribute(k_triple_commit<W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_triple_commit<W16><<<1, 1024, smem, ctx->st>>>(view<W16>(ctx), ctx->ckeys_sorted, n, o->max_candidates,
                                                      o->max_verify, o->seed, ctx->cstats);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[3], ctx->st));
    CommitStats cs;
    unsigned long long cnt[2];
    std::vector<unsigned long long> keys(n);
    CK(cudaMemcpyAsync(&cs, ctx->cstats, sizeof cs, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(cnt, ctx->tcount, sizeof cnt, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(keys.data(), ctx->ckeys_sorted, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->score = before + cs.total_delta;
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->score_before = before;
        stats->score_after = ctx->score;
        stats->triples = (long long)cnt[0];
        stats->rotations = 2 * (long long)cnt[0];
        int nc = 0;
        while (nc < n && keys[nc] != ~0ull) nc++;
        stats->candidates = nc;
        stats->best_delta = nc ? (int)(0x7fffffffu - (unsigned)(keys[0] >> 32)) : 0;
        stats->scanned = cs.scanned;
        stats->verified = cs.verified;
        stats->committed = cs.committed;
        cudaEventElapsedTime(&stats->ms_sample, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&stats->ms_eval, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&stats->ms_commit, ctx->ev[2], ctx->ev[3]);
        cudaEventElapsedTime(&stats->ms_total, ctx->ev[0], ctx->ev[3]);
    }
    return BM_OK;
}

extern "C" bm_status bm_triple_round(bm_ctx* ctx, const bm_triple_opts* opts, bm_triple_stats* stats) {
    if (!ctx || !opts) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_triple_round: no mapping set"); return BM_E_STATE; }
    return ctx->w16 ? triple_round_impl<true>(ctx, opts, stats) : triple_round_impl<false>(ctx, opts, stats);
}

extern "C" bm_status bm_quad_deltas(bm_ctx* ctx, int64_t k, const int32_t* sets, const int32_t* perms,
                                    int32_t* out) {
    if (!ctx) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_quad_deltas: no mapping set"); return BM_E_STATE; }
    if (k < 0 || (k && (!sets || !perms || !out))) { set_err(ctx, "bm_quad_deltas: bad arguments"); return BM_E_INPUT; }
    if (k == 0) return BM_OK;
    const int n = ctx->n;
    std::vector<int> h(5 * k);
    for (int64_t i = 0; i < k; i++) {
        const int* v = sets + 4 * i;
        bool ok = perms[i] >= 1 && perms[i] <= 23;
        for (int t = 0; t < 4 && ok; t++) {
            if (v[t] < 1 || v[t] > n) ok = false;
            for (int u = 0; u < t; u++) if (v[u] == v[t]) ok = false;
        }
        if (!ok) {
            set_err(ctx, "bm_quad_deltas: set %lld = (%d,%d,%d,%d) with permutation %d invalid", (long long)i,
                    v[0], v[1], v[2], v[3], perms[i]);
            return BM_E_INPUT;
        }
        for (int t = 0; t < 4; t++) h[4 * i + t] = v[t] - 1;
        h[4 * k + i] = perms[i];
    }
    bm_status s = ensure_scratch(ctx, 6 * k);
    if (s) return s;
    int* d = ctx->scratch_pairs;
    CK(cudaMemcpyAsync(d, h.data(), 5 * k * sizeof(int), cudaMemcpyHostToDevice, ctx->st));
    const long long blocks = std::min<long long>((k + 7) / 8, (long long)ctx->num_sms * 16);
    if (ctx->w16) k_quad_deltas<true><<<(int)blocks, 256, 0, ctx->st>>>(view<true>(ctx), d, d + 4 * k, k, d + 5 * k);
    else k_quad_deltas<false><<<(int)blocks, 256, 0, ctx->st>>>(view<false>(ctx), d, d + 4 * k, k, d + 5 * k);
    CK(cudaGetLastError());
    CK(cudaMemcpyAsync(out, d + 5 * k, k * sizeof(int), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    return BM_OK;
}

template <bool W16>
static bm_status quad_round_impl(bm_ctx* ctx, const bm_quad_opts* o, bm_quad_stats* stats) {
    const int n = ctx->n;
    const int partners = o->partners > 0 ? o->partners : 64;
    if (partners > 2048) { set_err(ctx, "bm_quad_round: partners=%d above 2048", partners); return BM_E_INPUT; }
    bm_status s = ensure_S(ctx);
    if (s) return s;
    s = ensure_adj<W16>(ctx);
    if (s) return s;
    if (!ctx->tcount) CK(dalloc(ctx, &ctx->tcount, 2 * sizeof(unsigned long long)));
    const long long before = ctx->score;
    CK(cudaEventRecord(ctx->ev[0], ctx->st));
    int mode = 0;
    s = (o && o->incremental) ? stage_refresh<W16>(ctx, &mode) : stage_profit<W16>(ctx);
    if (s) return s;
    CK(cudaEventRecord(ctx->ev[1], ctx->st));
    CK(cudaMemsetAsync(ctx->tcount, 0, 2 * sizeof(unsigned long long), ctx->st));
    const int blocks = std::min(n, ctx->num_sms * 8);
    k_quad_eval<W16><<<blocks, 256, 0, ctx->st>>>(view<W16>(ctx), ctx->adj, ctx->adj_words, partners, o->seed,
                                                  ctx->ckeys, ctx->tcount);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[2], ctx->st));
    size_t tb = ctx->cub_bytes;
    CK(cub::DeviceRadixSort::SortKeys(ctx->cub_tmp, tb, ctx->ckeys, ctx->ckeys_sorted, n, 0, 64, ctx->st));
    const size_t smem = 2 * (size_t)n;
    CK(cudaFuncSetAttribute(k_quad_commit<W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_quad_commit<W16><<<1, 1024, smem, ctx->st>>>(view<W16>(ctx), ctx->ckeys_sorted, n, o->max_candidates,
                                                    o->max_verify, o->seed, ctx->cstats);
    CK(cudaGetLastError());
    CK(cudaEventRecord(ctx->ev[3], ctx->st));
    CommitStats cs;
    unsigned long long cnt[2];
    std::vector<unsigned long long> keys(n);
    CK(cudaMemcpyAsync(&cs, ctx->cstats, sizeof cs, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(cnt, ctx->tcount, sizeof cnt, cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaMemcpyAsync(keys.data(), ctx->ckeys_sorted, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->st));
    CK(cudaStreamSynchronize(ctx->st));
    ctx->score = before + cs.total_delta;
    if (stats) {
        memset(stats, 0, sizeof *stats);
        stats->score_before = before;
        stats->score_after = ctx->score;
        stats->quads = (long long)cnt[0];
        stats->permutations = 23 * (long long)cnt[0];
        int nc = 0;
        while (nc < n && keys[nc] != ~0ull) nc++;
        stats->candidates = nc;
        stats->best_delta = nc ? (int)(0x7fffffffu - (unsigned)(keys[0] >> 32)) : 0;
        stats->scanned = cs.scanned;
        stats->verified = cs.verified;
        stats->committed = cs.committed;
        cudaEventElapsedTime(&stats->ms_sample, ctx->ev[0], ctx->ev[1]);
        cudaEventElapsedTime(&stats->ms_eval, ctx->ev[1], ctx->ev[2]);
        cudaEventElapsedTime(&stats->ms_commit, ctx->ev[2], ctx->ev[3]);
        cudaEventElapsedTime(&stats->ms_total, ctx->ev[0], ctx->ev[3]);
    }
    return BM_OK;
}

extern "C" bm_status bm_quad_round(bm_ctx* ctx, const bm_quad_opts* opts, bm_quad_stats* stats) {
    if (!ctx || !opts) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_quad_round: no mapping set"); return BM_E_STATE; }
    return ctx->w16 ? quad_round_impl<true>(ctx, opts, stats) : quad_round_impl<false>(ctx, opts, stats);
}

// ---------------------------------------------------------------------------
// bm_pair_deltas_static: staging in a fixed library array instead of memory
// the context allocates.  Layout: [0,K) first vertices, [K,2K) second
// vertices (both 1-based, as the caller passed them), [2K,3K) deltas, with
// K = BM_STATIC_MAX_PAIRS.  The host only ever uses the array's device address
// obtained from cudaGetSymbolAddress; the symbol itself is a host-side stand-in.
static __device__ __align__(256) int g_static_pairs[3 * BM_STATIC_MAX_PAIRS];

namespace {
constexpr int kStaticMaxDevices = 64;
std::mutex g_static_mu;
int* g_static_addr[kStaticMaxDevices] = {};
}  // namespace

// One warp per pair; ids arrive 1-based straight from the caller's arrays.
template <bool W16>
__global__ void k_pair_deltas_static(DevView<W16> g, const int* __restrict__ m1,
                                     const int* __restrict__ m2, long long k, int* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
    for (; w < k; w += nw) {
        int d = swap_delta_part<W16>(g, m1[w] - 1, m2[w] - 1, lane, 32);
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
        if (lane == 0) out[w] = d;
    }
}

// Device address of g_static_pairs on the context's device, looked up once per
// device with that device current.
static bm_status static_pairs_addr(bm_ctx* ctx, int** out) {
    if (ctx->dev < 0 || ctx->dev >= kStaticMaxDevices) {
        set_err(ctx, "bm_pair_deltas_static: device %d outside 0..%d", ctx->dev, kStaticMaxDevices - 1);
        return BM_E_INPUT;
    }
    std::lock_guard<std::mutex> lock(g_static_mu);
    if (!g_static_addr[ctx->dev]) {   // the caller made ctx->dev current
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_static_pairs);
        if (e != cudaSuccess) {
            set_err(ctx, "bm_pair_deltas_static: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
            return BM_E_CUDA;
        }
        g_static_addr[ctx->dev] = static_cast<int*>(p);
    }
    *out = g_static_addr[ctx->dev];
    return BM_OK;
}

extern "C" bm_status bm_pair_deltas_static(bm_ctx* ctx, int64_t k, const int32_t* m1, const int32_t* m2,
                                           int32_t* out) {
    if (!ctx) return BM_E_INPUT;
    if (!ctx->mapped) { set_err(ctx, "bm_pair_deltas_static: no mapping set"); return BM_E_STATE; }
    if (k < 0 || (k && (!m1 || !m2 || !out))) { set_err(ctx, "bm_pair_deltas_static: bad arguments"); return BM_E_INPUT; }
    if (k > BM_STATIC_MAX_PAIRS) {
        set_err(ctx, "bm_pair_deltas_static: k=%lld pairs exceeds the fixed staging size %d; split the call",
                (long long)k, BM_STATIC_MAX_PAIRS);
        return BM_E_INPUT;
    }
    if (k == 0) return BM_OK;
    const int n = ctx->n;
    for (int64_t i = 0; i < k; i++) {
        if (m1[i] < 1 || m1[i] > n || m2[i] < 1 || m2[i] > n || m1[i] == m2[i]) {
            set_err(ctx, "bm_pair_deltas_static: pair %lld = (%d,%d) invalid", (long long)i, m1[i], m2[i]);
            return BM_E_INPUT;
        }
    }
    // the copies and the launch run with the context's device current, whatever
    // device the caller has current; the caller's device is restored on return
    int cur = -1;
    CK(cudaGetDevice(&cur));
    if (cur != ctx->dev) CK(cudaSetDevice(ctx->dev));
    int* base = nullptr;
    bm_status s = static_pairs_addr(ctx, &base);
    if (!s) {
        int* da = base;
        int* db = base + BM_STATIC_MAX_PAIRS;
        int* dout = base + 2 * BM_STATIC_MAX_PAIRS;
        cudaError_t e = cudaMemcpyAsync(da, m1, k * sizeof(int), cudaMemcpyHostToDevice, ctx->st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(db, m2, k * sizeof(int), cudaMemcpyHostToDevice, ctx->st);
        if (e == cudaSuccess) {
            const long long blocks = std::min<long long>((k + 7) / 8, (long long)ctx->num_sms * 16);
            if (ctx->w16) k_pair_deltas_static<true><<<(int)blocks, 256, 0, ctx->st>>>(view<true>(ctx), da, db, k, dout);
            else k_pair_deltas_static<false><<<(int)blocks, 256, 0, ctx->st>>>(view<false>(ctx), da, db, k, dout);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) e = cudaMemcpyAsync(out, dout, k * sizeof(int), cudaMemcpyDeviceToHost, ctx->st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->st);
        if (e != cudaSuccess) {
            set_err(ctx, "bm_pair_deltas_static: %s", cudaGetErrorString(e));
            s = BM_E_CUDA;
        }
    }
    if (cur != ctx->dev) cudaSetDevice(cur);
    return s;
}
