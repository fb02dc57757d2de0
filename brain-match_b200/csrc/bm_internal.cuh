// bm_internal.cuh -- engine context shared by the single-instance and the
// batched entry points (internal; not part of the C ABI).
#pragma once
#include <cstdio>
#include <cstdarg>
#include <cuda.h>
#include <cuda_runtime.h>
#include "bm.h"
#include "bm_kernels.cuh"

using namespace bm;

// Test hook (bm_test_stall): 1 if the next launch at `site` is to make one of
// its bounded waits run out, clearing the request.
int take_stall(int site);

struct bm_ctx {
    int n = 0;
    bool w16 = true;
    int dev = 0, num_sms = 0;
    size_t smem_optin = 0;  // opt-in shared memory per block
    long long e1 = 0, e2 = 0, nself = 0;
    int max_deg1 = 0;       // largest G1 degree (in + out, self-loops apart)
    cudaStream_t st = nullptr;
    char err[512] = {0};
    bool mapped = false;
    long long score = 0;  // score of the current matching (kept exact across commits)
    unsigned long long serial = 0;  // unique per context in the process (caches keyed on a context)
    // device buffers
    int *off1o = nullptr, *off1i = nullptr, *off2o = nullptr, *off2i = nullptr, *offs = nullptr, *selfw = nullptr;
    void *ent1o = nullptr, *ent1i = nullptr, *ent2o = nullptr, *ent2i = nullptr;
    void *ent1oP = nullptr, *ent1iP = nullptr, *ent2oP = nullptr, *ent2iP = nullptr;
    int* off2oH = nullptr;                  // G2 out-entries with weight above the hub threshold
    void *ent2oH = nullptr, *ent2oHP = nullptr;
    long long e2H = 0;
    void* W2 = nullptr;
    void* W2T = nullptr;
    int* W2D = nullptr;            // W2's diagonal, n+1 entries (entry n = 0)
    int *p = nullptr, *pinv = nullptr;
    int* S = nullptr;
    unsigned long long* rowbest = nullptr;
    unsigned long long *ckeys = nullptr, *ckeys_sorted = nullptr;
    unsigned long long *wkeys = nullptr, *wkeys_sorted = nullptr;
    int *wvals = nullptr, *order = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int* small = nullptr;          // [0]=row counter [1]=ncand [2]=best delta
    unsigned long long* score_acc = nullptr;
    CommitStats* cstats = nullptr;
    int4* cinfo = nullptr;  // list extents of the sorted candidates (2 per candidate)
    int* cgrid = nullptr;   // set commit across CTAs: partial sums [2][32][8][3], barrier [2], error [1]
    // S kept exact across commits: the matching it is exact for, and the moved-vertex update
    bool S_exact = false;
    int *pS = nullptr, *pinvS = nullptr;  // n+1 entries each
    int* moved = nullptr;                 // moved vertices (n)
    int* minfo = nullptr;                 // [0] count [1] needs rebuild [2] max degree
    unsigned long long* mwork = nullptr;  // list entries the update touches
    long long upd_work = 0;               // ... in the last update (host copy)
    int* scratch_pairs = nullptr;  // pair/triple inputs and outputs (ints)
    long long scratch_cap = 0;
    unsigned* adj = nullptr;       // G1 adjacency bitmap (3-cycles)
    int adj_words = 0;
    int* rowd = nullptr;           // reference-order row deltas
    int* first = nullptr;          // [0] = first improving partner, [1] = copy for the host
    long long* fi_acc = nullptr;   // [0] = delta sum, [1] = commits
    unsigned long long* tcount = nullptr;
    long long dev_bytes = 0;
    cudaEvent_t ev[6] = {};
    cudaEvent_t uev[8] = {};       // bm_timer_* slots
    unsigned long long* work_sum = nullptr;   // min terms of the last rebuild
    bool work_valid = false;                  // wkeys hold the last rebuild's row work (scheduling keys)
    unsigned long long* part = nullptr;   // per-tile best partners (combine)
    // TMA-fed combine (n % 4 == 0): tensor map over S, S's diagonal, grid size
    alignas(64) CUtensorMap tmS;
    // persistent warp-specialised hub GEMM: tensor maps of its operands
    alignas(64) CUtensorMap tmHubA;
    alignas(64) CUtensorMap tmHubB;
    bool hub_ws_ready = false, hub_ws = false;
    bool cmb_ready = false;
    int cmb_grid = 0;
    int* diagS = nullptr;
    // tensor-core hub terms
    int nh = 0, hubK = 0, Mpad = 0, Npad = 0;
    bool hubA_built = false;
    int* hubs = nullptr;
    unsigned char* is_hub = nullptr;
    uint8_t *hubA = nullptr, *hubB = nullptr;
    int* hub_err = nullptr;
    cudaEvent_t ev_hub = nullptr;
};

// Records an error message on the context (or, with c == NULL, in the
// thread's slot read by bm_last_error(NULL)).
void set_err(bm_ctx* c, const char* fmt, ...);

#define CK(call)                                                                   \
    do {                                                                           \
        cudaError_t e_ = (call);                                                   \
        if (e_ != cudaSuccess) {                                                   \
            set_err(ctx, "%s:%d: %s: %s", __FILE__, __LINE__, #call,               \
                    cudaGetErrorString(e_));                                       \
            return BM_E_CUDA;                                                      \
        }                                                                          \
    } while (0)

template <typename T>
static cudaError_t dalloc(bm_ctx* ctx, T** ptr, size_t bytes) {
    cudaError_t e = cudaMalloc((void**)ptr, bytes ? bytes : 16);
    if (e == cudaSuccess) ctx->dev_bytes += (long long)bytes;
    return e;
}

template <bool W16>
inline DevView<W16> view(bm_ctx* c) {
    DevView<W16> g;
    typedef typename Ent<W16>::T E;
    typedef typename Dense<W16>::T D;
    g.n = c->n;
    g.off1o = c->off1o; g.ent1o = (const E*)c->ent1o;
    g.off1i = c->off1i; g.ent1i = (const E*)c->ent1i;
    g.off2o = c->off2o; g.ent2o = (const E*)c->ent2o;
    g.off2i = c->off2i; g.ent2i = (const E*)c->ent2i;
    g.offs = c->offs; g.selfw = c->selfw;
    g.ent1oP = (E*)c->ent1oP; g.ent1iP = (E*)c->ent1iP;
    g.ent2oP = (E*)c->ent2oP; g.ent2iP = (E*)c->ent2iP;
    g.off2oH = c->off2oH; g.ent2oHP = (E*)c->ent2oHP;
    g.W2 = (const D*)c->W2;
    g.W2T = (const D*)c->W2T;
    g.W2D = c->W2D;
    g.p = c->p; g.pinv = c->pinv;
    g.S = c->S;
    return g;
}

// Allocates the n x n profit matrix on first use.
bm_status ensure_S(bm_ctx* ctx);
// Sweep stages shared by the exhaustive and the learned sweep (bm_engine.cu):
// the profit matrix S of the current matching, then each row's best partner.
template <bool W16> bm_status stage_profit(bm_ctx* ctx);
// S made exact for the current matching: an update from the vertices whose
// image changed since S was last exact when that is cheaper, else
// stage_profit.  *mode: 0 rebuilt, 1 updated, 2 already exact.
template <bool W16> bm_status stage_refresh(bm_ctx* ctx, int* mode);
bm_status stage_combine(bm_ctx* ctx, int* all_out);
