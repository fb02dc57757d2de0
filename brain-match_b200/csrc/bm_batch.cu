// bm_batch.cu -- many independent alignment instances of uneven size swept
// together.
//
// Each instance is an ordinary context (bm_create: same preprocessing, same
// storage, same exact arithmetic); the batch adds device tables of the
// instances' buffers and runs the shared per-row, per-tile and per-instance
// bodies of the single-instance path in one of two schedules:
//   * the launch sequence: relabel (all lists of all instances) -> row work +
//     one LPT sort over all (instance, row) items -> one persistent
//     profit-row launch over every item -> one combine launch over every
//     (instance, tile) item -> reduce -> candidates -> one segmented sort ->
//     one commit launch (a CTA per instance);
//   * one persistent launch (k_b_sweep): the same phases in one cooperative
//     grid behind grid barriers, the candidate sort in shared memory.
// One sweep of the whole batch is captured once as a CUDA graph and replayed.
// The schedule and its launch shapes (profit-row block size, combine tile)
// are picked by bm_batch_autotune, which times the candidates on the batch
// itself; results do not depend on the choice.  Hub tensor-core terms are
// not used here: the instances are built with BM_FLAG_NO_HUB_GEMM.
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_segmented_radix_sort.cuh>
#include <cub/block/block_radix_sort.cuh>
#include "bm.h"
#include "bm_internal.cuh"
#include "bm_select.cuh"

namespace {

// Per-instance device record of the batch.
struct BatchInst {
    int n;
    int tiles;            // combine tiles per side for the current tile size
    long long tile_base;  // first global (instance, tile) item
    int row_base;         // first global (instance, row) item / candidate slot
    int* S;
    unsigned long long* rowbest;
    unsigned long long* part;
    unsigned long long* keys;
    unsigned long long* keys_sorted;
};

__device__ __forceinline__ int find_inst(const int* __restrict__ base, int nb, long long it) {
    int lo = 0, hi = nb;  // base[lo] <= it < base[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (base[mid] <= it) lo = mid; else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ int find_inst_ll(const long long* __restrict__ base, int nb, long long it) {
    int lo = 0, hi = nb;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (base[mid] <= it) lo = mid; else hi = mid;
    }
    return lo;
}

template <bool W16>
__global__ void k_b_relabel(const DevView<W16>* __restrict__ views, const long long* __restrict__ e1,
                            const long long* __restrict__ e2, const typename Ent<W16>::T* const* __restrict__ src,
                            int nb) {
    typedef Ent<W16> EN;
    const int b = blockIdx.y;
    const DevView<W16> g = views[b];
    // lists: 0 G1 out, 1 G1 in (through p); 2 G2 out, 3 G2 in (through pinv)
    const int lst = blockIdx.z;
    const long long m = lst < 2 ? e1[b] : e2[b];
    const typename EN::T* in = src[4 * b + lst];
    typename EN::T* out = lst == 0 ? g.ent1oP : lst == 1 ? g.ent1iP : lst == 2 ? g.ent2oP : g.ent2iP;
    const int* map = lst < 2 ? g.p : g.pinv;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (long long)gridDim.x * blockDim.x) {
        const typename EN::T e = in[i];
        out[i] = EN::make(map[EN::id(e)], EN::w(e));
    }
}

template <bool W16>
__global__ void k_b_row_work(const DevView<W16>* __restrict__ views, const int* __restrict__ row_base, int nb,
                             int total, unsigned long long* __restrict__ key, int* __restrict__ val) {
    typedef Ent<W16> EN;
    const int lane = threadIdx.x & 31;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int it = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; it < total; it += nwarps) {
        const int b = find_inst(row_base, nb, it);
        const DevView<W16>& g = views[b];
        const int a = it - row_base[b];
        long long w = 0;
        for (int i = g.off1o[a] + lane; i < g.off1o[a + 1]; i += 32) {
            const int f = EN::id(g.ent1oP[i]);
            w += g.off2i[f + 1] - g.off2i[f];
        }
        for (int i = g.off1i[a] + lane; i < g.off1i[a + 1]; i += 32) {
            const int f = EN::id(g.ent1iP[i]);
            w += g.off2o[f + 1] - g.off2o[f];
        }
        for (int o = 16; o; o >>= 1) w += __shfl_xor_sync(0xffffffffu, w, o);
        if (lane == 0) {
            w += (g.off1o[a + 1] - g.off1o[a]) + (g.off1i[a + 1] - g.off1i[a]) + 64;
            if (g.offs[a + 1] > g.offs[a]) w += g.n;
            key[it] = (unsigned long long)w;
            val[it] = it;
        }
    }
}

template <bool W16>
__global__ void __launch_bounds__(512)
k_b_profit(const DevView<W16>* __restrict__ views, const int* __restrict__ row_base, int nb, int total,
           const int* __restrict__ order, int* __restrict__ counter) {
    extern __shared__ int acc[];
    __shared__ int s_item, s_nlong;
    __shared__ int2 s_long[kLongQueue];
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int r = s_item;
        if (r >= total) break;
        const int it = order[r];
        const int b = find_inst(row_base, nb, it);
        const DevView<W16> g = views[b];
        profit_row<W16>(g, it - row_base[b], acc, s_long, &s_nlong, nullptr, 0);
    }
}

// (instance, tile) items: the upper triangle of each instance, row-major.
template <int T>
__global__ void __launch_bounds__(256)
k_b_combine(const BatchInst* __restrict__ inst, const long long* __restrict__ tile_base, int nb, long long total) {
    for (long long it = blockIdx.x; it < total; it += gridDim.x) {
        const int b = find_inst_ll(tile_base, nb, it);
        const BatchInst I = inst[b];
        long long t = it - tile_base[b];
        int ti = 0;
        while (t >= I.tiles - ti) { t -= I.tiles - ti; ti++; }
        const int tj = ti + (int)t;
        combine_tile<T>(I.S, I.n, ti, tj, I.part, nullptr);
        __syncthreads();
    }
}

__global__ void k_b_reduce(const BatchInst* __restrict__ inst, int nb) {
    const int b = blockIdx.y;
    const BatchInst I = inst[b];
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < I.n; x += gridDim.x * blockDim.x) {
        unsigned long long k = 0;
        for (int t = 0; t < I.tiles; t++) k = kmax(k, I.part[(size_t)t * I.n + x]);
        I.rowbest[x] = k;
    }
}

// Candidate keys of every instance (the single-instance rule, k_candidates).
__global__ void k_b_candidates(const BatchInst* __restrict__ inst, int nb) {
    const int b = blockIdx.y;
    const BatchInst I = inst[b];
    for (int a = blockIdx.x * blockDim.x + threadIdx.x; a < I.n; a += gridDim.x * blockDim.x) {
        const unsigned long long k = I.rowbest[a];
        unsigned long long out = ~0ull;
        if (k) {
            const int d = (int)((unsigned)(k >> 32) - 0x80000000u);
            const int p = (int)(~(unsigned)(k & 0xffffffffu));
            if (d > 0) {
                const unsigned long long kb = I.rowbest[p];
                const int pp = (int)(~(unsigned)(kb & 0xffffffffu));
                const bool mutual = (kb != 0) && (pp == a);
                if (!mutual || a < p) {
                    const int lo = a < p ? a : p, hi = a < p ? p : a;
                    out = ((unsigned long long)(0x7fffffffu - (unsigned)d) << 32) |
                          ((unsigned long long)lo << 16) | (unsigned long long)hi;
                }
            }
        }
        I.keys[a] = out;
    }
}

template <bool W16>
__global__ void __launch_bounds__(1024)
k_b_commit(const DevView<W16>* __restrict__ views, const BatchInst* __restrict__ inst, int max_scan,
           int max_verify, CommitStats* __restrict__ st, long long* __restrict__ acc_delta,
           long long* __restrict__ acc_commits) {
    extern __shared__ unsigned char smem[];
    const int b = blockIdx.x;
    const DevView<W16> g = views[b];
    const BatchInst I = inst[b];
    const int lim = (max_scan > 0 && max_scan < I.n) ? max_scan : I.n;
    commit_group<W16, kCGBatch>(g, I.keys_sorted, lim, max_verify, &st[b], smem);
    __syncthreads();
    if (threadIdx.x == 0) {
        acc_delta[b] += st[b].total_delta;
        acc_commits[b] += st[b].committed;
    }
}

// ---------------------------------------------------------------------------
// One batch sweep as one persistent launch: a cooperative grid of one
// 1024-thread CTA per SM.  The relabel of every list of every instance comes
// first, behind one bounded grid barrier; then a dataflow over the instances
// (no further grid barrier, see the kernel): four 256-thread groups per CTA
// take profit rows and combine tile pairs from one task counter, and each
// instance's row bests, candidates, in-kernel candidate sort and set commit
// run on the CTA that owns it as soon as its own tile pairs are done.  Row
// order does not matter for the result (integer sums).
constexpr int kBThreads = 1024;
constexpr int kBSortItems = 8;                           // candidate keys per thread
constexpr int kBSortMax = kBThreads * kBSortItems;       // instances up to 8,192 vertices
constexpr unsigned kBSpinLimit = 1u << 24;               // polls of one grid-barrier wait (~1 s)
typedef cub::BlockRadixSort<unsigned long long, kBThreads, kBSortItems> BSort;

template <bool W16>
struct BSweepArgs {
    const DevView<W16>* views;
    const BatchInst* inst;
    const long long* ebase;   // 4 count + 1: list segments laid end to end
    const typename Ent<W16>::T* const* lists;
    int nb;
    const int* iorder;     // instances, largest first: the order of their tasks
    const int* rpt;        // rows per row task: 2 when two of the instance's rows fit a group's shared memory
    const long long* tbase;   // 2 (count + 1): first row task, then first tile-pair task (from the
                              // first tile-pair task) of each instance in that order
    int total_tasks;       // every instance's rows and tile pairs
    size_t group_bytes;    // shared memory of one 256-thread group (a row accumulator or a tile stage)
    int* counter;          // tasks taken
    int* done;             // 2 count: rows and tile pairs finished, per instance
    unsigned* bar;         // grid barrier: arrivals, generation, error
    int max_scan, max_verify;
    int stall;             // test hook: the first grid barrier never completes
    CommitStats* st;
    long long* acc_delta;
    long long* acc_commits;
};

__device__ __forceinline__ unsigned b_ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Grid-wide barrier of the co-resident CTAs.  A wait that runs out sets the
// error word (bar[2]); every CTA leaves at its next barrier.  Returns false
// once the error word is set.  With `stall` (the bm_test_stall hook) CTA 0
// does not arrive and every CTA polls only a few thousand times, so the
// barrier never completes and every CTA leaves at it.
__device__ bool b_grid_barrier(unsigned* bar, bool stall = false) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        const unsigned gen = b_ld_acquire(&bar[1]);
        const unsigned limit = stall ? (1u << 12) : kBSpinLimit;
        if (!(stall && blockIdx.x == 0) && atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
            atomicExch(&bar[0], 0u);
            __threadfence();
            atomicAdd(&bar[1], 1u);
        } else {
            unsigned it = 0;
            while (b_ld_acquire(&bar[1]) == gen) {
                if (b_ld_acquire(&bar[2]) || ++it > limit) {
                    atomicExch(&bar[2], 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = ok && !b_ld_acquire(&bar[2]);
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ void b_group_sync(int grp) {
    asm volatile("bar.sync %0, 256;" :: "r"(grp + 1) : "memory");
}

template <bool W16, int T>
__global__ void __launch_bounds__(kBThreads, 1) k_b_sweep(BSweepArgs<W16> a) {
    typedef Ent<W16> EN;
    extern __shared__ __align__(16) unsigned char bsm[];
    const int tid = threadIdx.x;
    // relabel every instance's lists (G1 through p, G2 through pinv): the
    // lists laid end to end (segment 4b + lst starts at ebase[4b + lst]), each
    // CTA one contiguous range of that
    {
        const long long tot = a.ebase[4 * a.nb];
        const long long per = (tot + gridDim.x - 1) / gridDim.x;
        const long long lo = (long long)blockIdx.x * per, hi = min(tot, lo + per);
        for (int sg = 0; sg < 4 * a.nb && lo < hi; sg++) {
            const long long s0 = max(lo, a.ebase[sg]), s1 = min(hi, a.ebase[sg + 1]);
            if (s0 >= s1) continue;
            const int b = sg >> 2, lst = sg & 3;
            const DevView<W16>& g = a.views[b];
            const typename EN::T* in = a.lists[sg];
            typename EN::T* out = lst == 0 ? g.ent1oP : lst == 1 ? g.ent1iP : lst == 2 ? g.ent2oP : g.ent2iP;
            const int* map = lst < 2 ? g.p : g.pinv;
            for (long long i = s0 - a.ebase[sg] + tid; i < s1 - a.ebase[sg]; i += blockDim.x) {
                const typename EN::T e = in[i];
                out[i] = EN::make(map[EN::id(e)], EN::w(e));
            }
        }
    }
    // the dataflow's counters start from zero (read only after the barrier)
    if (blockIdx.x == 0) {
        if (tid == 0) *a.counter = 0;
        for (int i = tid; i < 2 * a.nb; i += blockDim.x) a.done[i] = 0;
    }
    if (!b_grid_barrier(a.bar, a.stall != 0)) return;
    // Dataflow over the instances, with no further grid barrier: the tasks are
    // every instance's rows, then every instance's tile pairs, each part with
    // the largest instance first (iorder), and the four 256-thread groups of
    // every CTA take them one at a time from a global counter.  A tile pair of
    // instance i waits until all of i's rows are written (they were taken
    // long before); the CTA that owns i (CTA i mod grid) stops taking tasks
    // once all of i's tile pairs are done and runs i's row bests, candidates,
    // candidate sort and set commit with all its threads -- so the largest
    // instances' commits overlap the other instances' tile pairs.
    // Dependencies point only to earlier tasks, which the groups that took
    // them finish without waiting on later ones.
    int* rows_done = a.done;
    int* tiles_done = a.done + a.nb;
    const int grp = tid >> 8, gtid = tid & 255;
    unsigned char* gsm = bsm + (size_t)grp * a.group_bytes;     // the group's row accumulator or tile stage
    int* acc = reinterpret_cast<int*>(gsm);
    CombineSmem<T>& cs = *reinterpret_cast<CombineSmem<T>*>(gsm);
    __shared__ int s_task[4], s_go[4];
    __shared__ int s_nlong[8];
    __shared__ int2 s_long[8][kLongQueue];   // per group, or per half-group for paired rows
    __shared__ int s_stop;
    for (int own = blockIdx.x;; own += gridDim.x) {
        const int target = own < a.nb ? a.inst[own].tiles * (a.inst[own].tiles + 1) / 2 : 0;
        for (;;) {
            if (gtid == 0) {
                int go = !b_ld_acquire(&a.bar[2]);
                if (go && own < a.nb && (int)b_ld_acquire((const unsigned*)&tiles_done[own]) >= target) go = 0;
                int t = -1;
                if (go && (t = atomicAdd(a.counter, 1)) >= a.total_tasks) go = 0;
                s_task[grp] = t;
                s_go[grp] = go;
            }
            b_group_sync(grp);
            if (!s_go[grp]) break;
            const int t = s_task[grp];
            const bool row = t < a.tbase[a.nb];
            const long long* base = row ? a.tbase : a.tbase + a.nb + 1;
            const int k = find_inst_ll(base, a.nb, row ? t : t - a.tbase[a.nb]);
            const int i = a.iorder[k];
            const BatchInst I = a.inst[i];
            const int local = (row ? t : t - (int)a.tbase[a.nb]) - (int)base[k] + (row ? 0 : I.n);
            if (row) {
                const DevView<W16> g = a.views[i];
                if (a.rpt[i] == 1) {   // profit row `local` of instance i by the whole group
                    // (the long-list queue of the group's first half: halves of other groups use theirs)
                    profit_row_on<W16, 256>(g, local, acc, s_long[2 * grp], &s_nlong[2 * grp], nullptr, 0, nullptr,
                                            nullptr, nullptr, [grp] { b_group_sync(grp); });
                    __threadfence();     // every thread's part of the row is visible before it counts
                    b_group_sync(grp);
                    if (gtid == 0) atomicAdd(&rows_done[i], 1);
                } else {               // rows 2 local and 2 local + 1, a 128-thread half and accumulator each
                    const int half = gtid >> 7, r = 2 * local + half;
                    const int hb = 2 * grp + half;   // the half's barrier: 5 + hb, 128 threads
                    if (r < I.n)
                        profit_row_on<W16, 128>(g, r, acc + half * ((I.n + 1 + 3) & ~3), s_long[hb], &s_nlong[hb],
                                                nullptr, 0, nullptr, nullptr, nullptr, [hb] {
                                                    asm volatile("bar.sync %0, 128;" :: "r"(5 + hb) : "memory");
                                                });
                    __threadfence();
                    b_group_sync(grp);
                    if (gtid == 0) atomicAdd(&rows_done[i], min(2, I.n - 2 * local));
                }
            } else {             // tile pair of instance i, once its rows are written
                if (gtid == 0) {
                    unsigned it = 0;
                    while ((int)b_ld_acquire((const unsigned*)&rows_done[i]) < I.n) {
                        if (b_ld_acquire(&a.bar[2]) || ++it > kBSpinLimit) { atomicExch(&a.bar[2], 1u); break; }
                        __nanosleep(64);
                    }
                    __threadfence();
                }
                b_group_sync(grp);
                long long q = local - I.n;
                int ti = 0;
                while (q >= I.tiles - ti) { q -= I.tiles - ti; ti++; }
                const int tj = ti + (int)q;
                combine_tile_on<T>(I.S, I.n, ti, tj, I.part, nullptr, cs, gtid, [grp] { b_group_sync(grp); });
                __threadfence();     // the tile's partial bests are visible before it counts
                b_group_sync(grp);   // (and cs is rewritten by the group's next task)
                if (gtid == 0) atomicAdd(&tiles_done[i], 1);
            }
        }
        __syncthreads();   // all four groups have stopped
        if (own >= a.nb) break;
        // ---- instance `own`: wait for its tile pairs, then its bests, candidates, sort and commit
        if (tid == 0) {
            unsigned it = 0;
            while ((int)b_ld_acquire((const unsigned*)&tiles_done[own]) < target) {
                if (b_ld_acquire(&a.bar[2]) || ++it > kBSpinLimit) { atomicExch(&a.bar[2], 1u); break; }
                __nanosleep(64);
            }
            __threadfence();
            s_stop = b_ld_acquire(&a.bar[2]) != 0;
        }
        __syncthreads();
        if (s_stop) break;
        const BatchInst I = a.inst[own];
        for (int x = tid; x < I.n; x += blockDim.x) {
            unsigned long long k = 0;
            for (int tt = 0; tt < I.tiles; tt++) k = kmax(k, __ldcg(&I.part[(size_t)tt * I.n + x]));
            I.rowbest[x] = k;
        }
        __syncthreads();
        // candidate keys (the single-instance rule, k_candidates)
        for (int xa = tid; xa < I.n; xa += blockDim.x) {
            const unsigned long long k = I.rowbest[xa];
            unsigned long long out = ~0ull;
            if (k) {
                const int d = (int)((unsigned)(k >> 32) - 0x80000000u);
                const int q = (int)(~(unsigned)(k & 0xffffffffu));
                if (d > 0) {
                    const unsigned long long kb = I.rowbest[q];
                    const int qq = (int)(~(unsigned)(kb & 0xffffffffu));
                    const bool mutual = (kb != 0) && (qq == xa);
                    if (!mutual || xa < q) {
                        const int lo = xa < q ? xa : q, hi = xa < q ? q : xa;
                        out = ((unsigned long long)(0x7fffffffu - (unsigned)d) << 32) |
                              ((unsigned long long)lo << 16) | (unsigned long long)hi;
                    }
                }
            }
            I.keys[xa] = out;
        }
        __syncthreads();
        {   // sort the candidate keys in shared memory
            typename BSort::TempStorage& ts = *reinterpret_cast<typename BSort::TempStorage*>(bsm);
            unsigned long long kk[kBSortItems];
#pragma unroll
            for (int q = 0; q < kBSortItems; q++) {
                const int x = tid * kBSortItems + q;
                kk[q] = x < I.n ? I.keys[x] : ~0ull;
            }
            BSort(ts).Sort(kk);
#pragma unroll
            for (int q = 0; q < kBSortItems; q++) {
                const int x = tid * kBSortItems + q;
                if (x < I.n) I.keys_sorted[x] = kk[q];
            }
        }
        __syncthreads();
        const DevView<W16> g = a.views[own];
        const int lim = (a.max_scan > 0 && a.max_scan < I.n) ? a.max_scan : I.n;
        commit_group<W16, kCGBatch>(g, I.keys_sorted, lim, a.max_verify, &a.st[own], bsm);
        __syncthreads();
        if (tid == 0) {
            a.acc_delta[own] += a.st[own].total_delta;
            a.acc_commits[own] += a.st[own].committed;
        }
        __syncthreads();
    }
}

}  // namespace

struct bm_batch {
    int count = 0, max_n = 0, total = 0;
    bool w16 = true;
    std::vector<bm_ctx*> ctx;
    cudaStream_t st = nullptr;
    char err[512] = {0};
    // tuning
    int profit_threads = 512, tile = 64;
    bool tuned = false;
    // device tables
    void* views = nullptr;                // DevView<W16>[count]
    BatchInst* inst = nullptr;
    int* row_base = nullptr;              // count+1
    long long* tile_base = nullptr;       // count+1
    long long *e1 = nullptr, *e2 = nullptr;
    long long* ebase = nullptr;           // 4 count + 1: the lists laid end to end (persistent relabel)
    // the persistent schedule's dataflow: instances largest first, the first
    // row task and tile-pair task of each in that order, per-instance
    // finished rows and tile pairs
    int* iorder = nullptr;
    int* rpt = nullptr;                   // rows per row task of each instance (1 or 2)
    long long* tbase = nullptr;
    long long total_tasks = 0;
    int* done = nullptr;
    void** lists = nullptr;               // 4 per instance: ent1o, ent1i, ent2o, ent2i
    unsigned long long *wkeys = nullptr, *wkeys_sorted = nullptr, *ckeys = nullptr, *ckeys_sorted = nullptr;
    int *wvals = nullptr, *order = nullptr;
    unsigned long long *rowbest = nullptr, *part = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    int* counter = nullptr;
    CommitStats* cstats = nullptr;
    long long *acc_delta = nullptr, *acc_commits = nullptr;
    long long total_tiles = 0;
    std::vector<BatchInst> hinst;
    // schedules: one persistent launch per sweep (k_b_sweep, possible when
    // every instance's candidates fit its in-kernel sort) or the launch
    // sequence above; the autotuner times both and keeps the faster
    bool can_persist = false, use_persist = false;
    size_t psmem = 0;
    unsigned* gbar = nullptr;             // its grid barrier
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int graph_max_scan = 0, graph_max_verify = -1;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
};

static thread_local char g_batch_create_err[512];

template <bool W16>
static bm_status persistent_setup(bm_batch* B);
template <int T>
static size_t persistent_group_bytes(int max_n);

#define BK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess) {                                                         \
            snprintf(B->err, sizeof B->err, "%s:%d: %s: %s", __FILE__, __LINE__, #call,  \
                     cudaGetErrorString(e_));                                            \
            return BM_E_CUDA;                                                            \
        }                                                                                \
    } while (0)

static void batch_free(bm_batch* B) {
    if (!B) return;
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    void* bufs[] = {B->views, B->inst, B->row_base, B->tile_base, B->e1, B->e2, B->lists, B->wkeys,
                    B->wkeys_sorted, B->ckeys, B->ckeys_sorted, B->wvals, B->order, B->rowbest, B->part,
                    B->cub_tmp, B->counter, B->cstats, B->acc_delta, B->acc_commits, B->gbar, B->ebase,
                    B->iorder, B->tbase, B->done, B->rpt};
    for (void* p : bufs) if (p) cudaFree(p);
    if (B->ev0) cudaEventDestroy(B->ev0);
    if (B->ev1) cudaEventDestroy(B->ev1);
    if (B->st) cudaStreamDestroy(B->st);
    for (bm_ctx* c : B->ctx) bm_destroy(c);
    delete B;
}

extern "C" void bm_batch_destroy(bm_batch* B) { batch_free(B); }
extern "C" const char* bm_batch_last_error(const bm_batch* B) { return B ? B->err : g_batch_create_err; }

// (Re)builds the per-instance tile tables for the current tile size.
static bm_status batch_tiles(bm_batch* B) {
    std::vector<long long> tb(B->count + 1, 0);
    for (int i = 0; i < B->count; i++) {
        const int T = (B->hinst[i].n + B->tile - 1) / B->tile;
        B->hinst[i].tiles = T;
        B->hinst[i].tile_base = tb[i];
        tb[i + 1] = tb[i] + (long long)T * (T + 1) / 2;
    }
    B->total_tiles = tb[B->count];
    BK(cudaMemcpy(B->tile_base, tb.data(), tb.size() * sizeof(long long), cudaMemcpyHostToDevice));
    if (B->iorder) {   // the persistent schedule's task layout: per instance, largest first, rows then tile pairs
        std::vector<int> ord(B->count);
        for (int i = 0; i < B->count; i++) ord[i] = i;
        std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) { return B->hinst[x].n > B->hinst[y].n; });
        // two rows per row task where both accumulators fit a group's shared memory
        const size_t gb = B->tile == 32 ? persistent_group_bytes<32>(B->max_n) : persistent_group_bytes<64>(B->max_n);
        std::vector<int> rpt(B->count);
        for (int i = 0; i < B->count; i++)
            rpt[i] = 2 * (size_t)((B->hinst[i].n + 1 + 3) & ~3) * sizeof(int) <= gb ? 2 : 1;
        // [rows prefix (count + 1)][tile-pair prefix (count + 1)]
        std::vector<long long> tbase(2 * (size_t)B->count + 2, 0);
        for (int k = 0; k < B->count; k++) {
            const BatchInst& I = B->hinst[ord[k]];
            tbase[k + 1] = tbase[k] + (I.n + rpt[ord[k]] - 1) / rpt[ord[k]];
            tbase[B->count + 1 + k + 1] = tbase[B->count + 1 + k] + (long long)I.tiles * (I.tiles + 1) / 2;
        }
        B->total_tasks = tbase[B->count] + tbase[2 * (size_t)B->count + 1];
        if (B->total_tasks > 0x7fffffffLL) B->can_persist = B->use_persist = false;   // 32-bit task indices
        BK(cudaMemcpy(B->iorder, ord.data(), ord.size() * sizeof(int), cudaMemcpyHostToDevice));
        BK(cudaMemcpy(B->rpt, rpt.data(), rpt.size() * sizeof(int), cudaMemcpyHostToDevice));
        BK(cudaMemcpy(B->tbase, tbase.data(), tbase.size() * sizeof(long long), cudaMemcpyHostToDevice));
    }
    BK(cudaMemcpy(B->inst, B->hinst.data(), B->hinst.size() * sizeof(BatchInst), cudaMemcpyHostToDevice));
    return BM_OK;
}

template <bool W16>
static bm_status batch_tables(bm_batch* B) {
    std::vector<DevView<W16>> v(B->count);
    std::vector<void*> lists(4 * B->count);
    std::vector<long long> e1(B->count), e2(B->count);
    for (int i = 0; i < B->count; i++) {
        v[i] = view<W16>(B->ctx[i]);
        lists[4 * i + 0] = B->ctx[i]->ent1o;
        lists[4 * i + 1] = B->ctx[i]->ent1i;
        lists[4 * i + 2] = B->ctx[i]->ent2o;
        lists[4 * i + 3] = B->ctx[i]->ent2i;
        e1[i] = B->ctx[i]->e1;
        e2[i] = B->ctx[i]->e2;
    }
    BK(cudaMalloc(&B->views, v.size() * sizeof(DevView<W16>)));
    BK(cudaMemcpy(B->views, v.data(), v.size() * sizeof(DevView<W16>), cudaMemcpyHostToDevice));
    BK(cudaMalloc(&B->lists, lists.size() * sizeof(void*)));
    BK(cudaMemcpy(B->lists, lists.data(), lists.size() * sizeof(void*), cudaMemcpyHostToDevice));
    BK(cudaMalloc(&B->e1, B->count * sizeof(long long)));
    BK(cudaMalloc(&B->e2, B->count * sizeof(long long)));
    BK(cudaMemcpy(B->e1, e1.data(), B->count * sizeof(long long), cudaMemcpyHostToDevice));
    BK(cudaMemcpy(B->e2, e2.data(), B->count * sizeof(long long), cudaMemcpyHostToDevice));
    std::vector<long long> eb(4 * (size_t)B->count + 1, 0);
    for (int i = 0; i < B->count; i++)
        for (int l = 0; l < 4; l++) eb[4 * i + l + 1] = eb[4 * i + l] + (l < 2 ? e1[i] : e2[i]);
    BK(cudaMalloc(&B->ebase, eb.size() * sizeof(long long)));
    BK(cudaMemcpy(B->ebase, eb.data(), eb.size() * sizeof(long long), cudaMemcpyHostToDevice));
    return BM_OK;
}

extern "C" bm_status bm_batch_create(bm_batch** out, int32_t count, const int32_t* n, const int64_t* e1,
                                     const int32_t* const* src1, const int32_t* const* dst1,
                                     const int32_t* const* w1, const int64_t* e2, const int32_t* const* src2,
                                     const int32_t* const* dst2, const int32_t* const* w2, uint32_t flags) {
    if (!out || count < 1 || !n || !e1 || !src1 || !dst1 || !w1 || !e2 || !src2 || !dst2 || !w2)
        return BM_E_INPUT;
    *out = nullptr;
    bm_batch* B = new (std::nothrow) bm_batch();
    if (!B) return BM_E_NOMEM;
    B->count = count;
    // every instance in one storage mode
    const uint32_t f = (flags | BM_FLAG_NO_HUB_GEMM);
    bool any32 = (flags & BM_FLAG_FORCE_I32) != 0;
    for (int pass = 0; pass < 2; pass++) {
        for (bm_ctx* c : B->ctx) bm_destroy(c);
        B->ctx.clear();
        for (int i = 0; i < count; i++) {
            bm_ctx* c = nullptr;
            bm_status s = bm_create(&c, n[i], e1[i], src1[i], dst1[i], w1[i], e2[i], src2[i], dst2[i], w2[i],
                                    f | (any32 ? BM_FLAG_FORCE_I32 : 0u));
            if (s != BM_OK) {
                snprintf(g_batch_create_err, sizeof g_batch_create_err, "instance %d: %s", i, bm_last_error(nullptr));
                batch_free(B);
                return s;
            }
            B->ctx.push_back(c);
        }
        bool mixed = false;
        for (bm_ctx* c : B->ctx) mixed |= !c->w16;
        if (!mixed || any32) break;
        any32 = true;  // some instance needs 32-bit entries: rebuild all that way
    }
    B->w16 = B->ctx[0]->w16;
    bm_status s;
    for (bm_ctx* c : B->ctx) {
        if ((s = ensure_S(c)) != BM_OK) {
            snprintf(g_batch_create_err, sizeof g_batch_create_err, "%s", c->err);
            batch_free(B);
            return s;
        }
        B->max_n = std::max(B->max_n, c->n);
        B->total += c->n;
    }
    auto body = [&]() -> bm_status {
        BK(cudaStreamCreateWithFlags(&B->st, cudaStreamNonBlocking));
        BK(cudaEventCreate(&B->ev0));
        BK(cudaEventCreate(&B->ev1));
        // concatenated per-instance buffers, sized for the smallest tile (32)
        std::vector<int> rb(count + 1, 0);
        long long part_total = 0;
        for (int i = 0; i < count; i++) {
            rb[i + 1] = rb[i] + B->ctx[i]->n;
            part_total += (long long)((B->ctx[i]->n + 31) / 32) * B->ctx[i]->n;
        }
        BK(cudaMalloc(&B->row_base, rb.size() * sizeof(int)));
        BK(cudaMemcpy(B->row_base, rb.data(), rb.size() * sizeof(int), cudaMemcpyHostToDevice));
        BK(cudaMalloc(&B->tile_base, (count + 1) * sizeof(long long)));
        BK(cudaMalloc(&B->inst, count * sizeof(BatchInst)));
        const size_t tot = (size_t)B->total;
        BK(cudaMalloc(&B->wkeys, tot * sizeof(unsigned long long)));
        BK(cudaMalloc(&B->wkeys_sorted, tot * sizeof(unsigned long long)));
        BK(cudaMalloc(&B->ckeys, tot * sizeof(unsigned long long)));
        BK(cudaMalloc(&B->ckeys_sorted, tot * sizeof(unsigned long long)));
        BK(cudaMalloc(&B->wvals, tot * sizeof(int)));
        BK(cudaMalloc(&B->order, tot * sizeof(int)));
        BK(cudaMalloc(&B->rowbest, tot * sizeof(unsigned long long)));
        BK(cudaMalloc(&B->part, (size_t)part_total * sizeof(unsigned long long)));
        BK(cudaMalloc(&B->counter, sizeof(int)));
        BK(cudaMalloc(&B->cstats, count * sizeof(CommitStats)));
        BK(cudaMalloc(&B->acc_delta, count * sizeof(long long)));
        BK(cudaMalloc(&B->acc_commits, count * sizeof(long long)));
        size_t b1 = 0, b2 = 0;
        BK(cub::DeviceRadixSort::SortPairsDescending(nullptr, b1, B->wkeys, B->wkeys_sorted, B->wvals, B->order,
                                                     B->total));
        BK(cub::DeviceSegmentedRadixSort::SortKeys(nullptr, b2, B->ckeys, B->ckeys_sorted, B->total, count,
                                                   B->row_base, B->row_base + 1));
        B->cub_bytes = std::max(b1, b2);
        BK(cudaMalloc(&B->cub_tmp, B->cub_bytes));
        B->hinst.resize(count);
        long long poff = 0;
        for (int i = 0; i < count; i++) {
            BatchInst& I = B->hinst[i];
            I.n = B->ctx[i]->n;
            I.row_base = rb[i];
            I.S = B->ctx[i]->S;
            I.rowbest = B->rowbest + rb[i];
            I.part = B->part + poff;
            poff += (long long)((I.n + 31) / 32) * I.n;
            I.keys = B->ckeys + rb[i];
            I.keys_sorted = B->ckeys_sorted + rb[i];
        }
        bm_status s2 = B->w16 ? batch_tables<true>(B) : batch_tables<false>(B);
        if (s2) return s2;
        BK(cudaMalloc(&B->gbar, 4 * sizeof(unsigned)));
        BK(cudaMemset(B->gbar, 0, 4 * sizeof(unsigned)));
        BK(cudaMalloc(&B->iorder, count * sizeof(int)));
        BK(cudaMalloc(&B->rpt, count * sizeof(int)));
        BK(cudaMalloc(&B->tbase, 2 * (count + 1) * sizeof(long long)));
        BK(cudaMalloc(&B->done, 2 * count * sizeof(int)));
        s2 = B->w16 ? persistent_setup<true>(B) : persistent_setup<false>(B);
        if (s2) return s2;
        return batch_tiles(B);
    };
    s = body();
    if (s != BM_OK) {
        snprintf(g_batch_create_err, sizeof g_batch_create_err, "%s", B->err);
        batch_free(B);
        return s;
    }
    *out = B;
    return BM_OK;
}

extern "C" bm_status bm_batch_set_mappings(bm_batch* B, const int32_t* const* maps) {
    if (!B || !maps) return BM_E_INPUT;
    for (int i = 0; i < B->count; i++) {
        bm_status s = bm_set_mapping(B->ctx[i], maps[i]);
        if (s) { snprintf(B->err, sizeof B->err, "instance %d: %.480s", i, B->ctx[i]->err); return s; }
    }
    return BM_OK;
}

extern "C" bm_status bm_batch_get_mappings(bm_batch* B, int32_t* const* maps) {
    if (!B || !maps) return BM_E_INPUT;
    for (int i = 0; i < B->count; i++) {
        bm_status s = bm_get_mapping(B->ctx[i], maps[i]);
        if (s) { snprintf(B->err, sizeof B->err, "instance %d: %.480s", i, B->ctx[i]->err); return s; }
    }
    return BM_OK;
}

extern "C" bm_status bm_batch_scores(bm_batch* B, int64_t* scores) {
    if (!B || !scores) return BM_E_INPUT;
    for (int i = 0; i < B->count; i++) {
        bm_status s = bm_score(B->ctx[i], &scores[i]);
        if (s) { snprintf(B->err, sizeof B->err, "instance %d: %.480s", i, B->ctx[i]->err); return s; }
    }
    return BM_OK;
}

// Shared memory of k_b_sweep: the largest of its phases' needs.
// Shared memory of one 256-thread group of k_b_sweep: a row accumulator or a
// tile stage, whichever is larger.
template <int T>
static size_t persistent_group_bytes(int max_n) {
    const size_t row = (size_t)((max_n + 1 + 3) & ~3) * sizeof(int);
    return (std::max(row, sizeof(CombineSmem<T>)) + 15) & ~(size_t)15;
}

template <int T>
static size_t persistent_smem(int max_n) {
    size_t m = 4 * persistent_group_bytes<T>(max_n);                      // four groups
    m = std::max(m, sizeof(typename BSort::TempStorage));                  // the candidate sort
    m = std::max(m, commit_group_smem(max_n));                             // the set commit
    return (m + 15) & ~(size_t)15;
}

template <bool W16, int T>
static bool persistent_fits(bm_batch* B, size_t* smem) {
    const size_t sm = persistent_smem<T>(B->max_n);
    if (cudaFuncSetAttribute(k_b_sweep<W16, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_b_sweep<W16, T>, kBThreads, sm) != cudaSuccess ||
        per_sm < 1) {
        cudaGetLastError();
        return false;
    }
    *smem = sm;
    return true;
}

// Whether every batch sweep can be one persistent launch: the instances'
// candidates fit the in-kernel sort and the kernel fits one CTA per SM with
// either combine tile.
template <bool W16>
static bm_status persistent_setup(bm_batch* B) {
    size_t s32 = 0, s64 = 0;
    B->can_persist = B->max_n <= kBSortMax && persistent_fits<W16, 32>(B, &s32) && persistent_fits<W16, 64>(B, &s64);
    B->psmem = std::max(s32, s64);
    return BM_OK;
}

template <bool W16>
static bm_status enqueue_persistent(bm_batch* B, int max_scan, int max_verify, int stall = 0) {
    BSweepArgs<W16> a;
    a.views = (const DevView<W16>*)B->views;
    a.inst = B->inst;
    a.ebase = B->ebase;
    a.lists = (const typename Ent<W16>::T* const*)B->lists;
    a.nb = B->count;
    a.iorder = B->iorder;
    a.rpt = B->rpt;
    a.tbase = B->tbase;
    a.total_tasks = (int)B->total_tasks;
    a.group_bytes = B->tile == 32 ? persistent_group_bytes<32>(B->max_n) : persistent_group_bytes<64>(B->max_n);
    a.counter = B->counter;
    a.done = B->done;
    a.bar = B->gbar;
    a.max_scan = max_scan;
    a.max_verify = max_verify;
    a.stall = stall;
    a.st = B->cstats;
    a.acc_delta = B->acc_delta;
    a.acc_commits = B->acc_commits;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(B->ctx[0]->num_sms);
    cfg.blockDim = dim3(kBThreads);
    cfg.dynamicSmemBytes = B->tile == 32 ? persistent_smem<32>(B->max_n) : persistent_smem<64>(B->max_n);
    cfg.stream = B->st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (B->tile == 32) BK(cudaLaunchKernelEx(&cfg, k_b_sweep<W16, 32>, a));
    else BK(cudaLaunchKernelEx(&cfg, k_b_sweep<W16, 64>, a));
    return BM_OK;
}

// Enqueues the profit and combine stages of one batch sweep on B->st.
template <bool W16>
static bm_status enqueue_eval(bm_batch* B) {
    typedef typename Ent<W16>::T E;
    const DevView<W16>* views = (const DevView<W16>*)B->views;
    long long maxe = 0;
    for (bm_ctx* c : B->ctx) maxe = std::max(maxe, std::max(c->e1, c->e2));
    dim3 rg((unsigned)std::min<long long>((maxe + 255) / 256, 256), B->count, 4);
    k_b_relabel<W16><<<rg, 256, 0, B->st>>>(views, B->e1, B->e2, (const E* const*)B->lists, B->count);
    BK(cudaGetLastError());
    k_b_row_work<W16><<<(B->total + 7) / 8, 256, 0, B->st>>>(views, B->row_base, B->count, B->total, B->wkeys,
                                                            B->wvals);
    BK(cudaGetLastError());
    size_t tb = B->cub_bytes;
    BK(cub::DeviceRadixSort::SortPairsDescending(B->cub_tmp, tb, B->wkeys, B->wkeys_sorted, B->wvals, B->order,
                                                 B->total, 0, 64, B->st));
    BK(cudaMemsetAsync(B->counter, 0, sizeof(int), B->st));
    const size_t smem = (size_t)(B->max_n + 1) * sizeof(int);
    BK(cudaFuncSetAttribute(k_b_profit<W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0, sms = B->ctx[0]->num_sms;
    BK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_b_profit<W16>, B->profit_threads, smem));
    if (per_sm < 1) { snprintf(B->err, sizeof B->err, "profit kernel does not fit (max n %d)", B->max_n); return BM_E_INPUT; }
    k_b_profit<W16><<<sms * per_sm, B->profit_threads, smem, B->st>>>(views, B->row_base, B->count, B->total,
                                                                     B->order, B->counter);
    BK(cudaGetLastError());
    const unsigned cg = (unsigned)std::min<long long>(B->total_tiles, (long long)sms * 16);
    if (B->tile == 32) k_b_combine<32><<<cg, 256, 0, B->st>>>(B->inst, B->tile_base, B->count, B->total_tiles);
    else k_b_combine<64><<<cg, 256, 0, B->st>>>(B->inst, B->tile_base, B->count, B->total_tiles);
    BK(cudaGetLastError());
    dim3 cg2((B->max_n + 255) / 256, B->count);
    k_b_reduce<<<cg2, 256, 0, B->st>>>(B->inst, B->count);
    BK(cudaGetLastError());
    return BM_OK;
}

template <bool W16>
static bm_status enqueue_select_commit(bm_batch* B, int max_scan, int max_verify) {
    dim3 cg2((B->max_n + 255) / 256, B->count);
    k_b_candidates<<<cg2, 256, 0, B->st>>>(B->inst, B->count);
    BK(cudaGetLastError());
    size_t tb = B->cub_bytes;
    BK(cub::DeviceSegmentedRadixSort::SortKeys(B->cub_tmp, tb, B->ckeys, B->ckeys_sorted, B->total, B->count,
                                               B->row_base, B->row_base + 1, 0, 64, B->st));
    const size_t smem = commit_group_smem(B->max_n);
    BK(cudaFuncSetAttribute(k_b_commit<W16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_b_commit<W16><<<B->count, 1024, smem, B->st>>>((const DevView<W16>*)B->views, B->inst, max_scan, max_verify,
                                                     B->cstats, B->acc_delta, B->acc_commits);
    BK(cudaGetLastError());
    return BM_OK;
}

static bm_status enqueue_sweep(bm_batch* B, int max_scan, int max_verify) {
    if (B->use_persist)
        return B->w16 ? enqueue_persistent<true>(B, max_scan, max_verify)
                      : enqueue_persistent<false>(B, max_scan, max_verify);
    bm_status s = B->w16 ? enqueue_eval<true>(B) : enqueue_eval<false>(B);
    if (s) return s;
    return B->w16 ? enqueue_select_commit<true>(B, max_scan, max_verify)
                  : enqueue_select_commit<false>(B, max_scan, max_verify);
}

extern "C" bm_status bm_batch_autotune(bm_batch* B, int32_t* profit_threads, int32_t* combine_tile) {
    if (!B) return BM_E_INPUT;
    for (bm_ctx* c : B->ctx)
        if (!c->mapped) { snprintf(B->err, sizeof B->err, "bm_batch_autotune: mappings not set"); return BM_E_STATE; }
    // candidate schedules: the persistent launch with either combine tile,
    // and the launch sequence with profit blocks of 256 or 512 threads and
    // either tile; each is timed on whole sweeps of the batch itself from the
    // same matchings, restored afterwards (results never depend on the choice)
    struct Sched { bool persist; int threads, tile; };
    std::vector<Sched> cand;
    if (B->can_persist) { cand.push_back({true, kBThreads, 32}); cand.push_back({true, kBThreads, 64}); }
    for (int pt : {256, 512})
        for (int tl : {32, 64}) cand.push_back({false, pt, tl});
    std::vector<std::vector<int32_t>> saved(B->count);
    for (int i = 0; i < B->count; i++) {
        saved[i].resize((size_t)B->ctx[i]->n + 1);
        bm_status s = bm_get_mapping(B->ctx[i], saved[i].data());
        if (s) return s;
    }
    auto restore = [&]() -> bm_status {
        for (int i = 0; i < B->count; i++) {
            bm_status s = bm_set_mapping(B->ctx[i], saved[i].data());
            if (s) return s;
        }
        return BM_OK;
    };
    float best = 1e30f;
    Sched pick = cand[0];
    for (const Sched& c : cand) {
        B->use_persist = c.persist;
        B->profit_threads = c.threads;
        B->tile = c.tile;
        bm_status s = batch_tiles(B);
        if (s) return s;
        // the second and third sweep from the saved matchings (the first
        // warms up and has a descent's first, commit-heavy candidate set)
        if ((s = restore())) return s;
        if ((s = enqueue_sweep(B, 0, -1))) return s;
        BK(cudaEventRecord(B->ev0, B->st));
        for (int rep = 0; rep < 2; rep++)
            if ((s = enqueue_sweep(B, 0, -1))) return s;
        BK(cudaEventRecord(B->ev1, B->st));
        BK(cudaEventSynchronize(B->ev1));
        float tot = 0;
        BK(cudaEventElapsedTime(&tot, B->ev0, B->ev1));
        if (tot < best) { best = tot; pick = c; }
    }
    bm_status s = restore();
    if (s) return s;
    B->use_persist = pick.persist;
    B->profit_threads = pick.threads;
    B->tile = pick.tile;
    if ((s = batch_tiles(B))) return s;
    B->tuned = true;
    if (B->exec) { cudaGraphExecDestroy(B->exec); B->exec = nullptr; }
    if (B->graph) { cudaGraphDestroy(B->graph); B->graph = nullptr; }
    if (profit_threads) *profit_threads = pick.threads;
    if (combine_tile) *combine_tile = pick.tile;
    return BM_OK;
}

extern "C" bm_status bm_batch_set_schedule(bm_batch* B, int32_t persistent, int32_t profit_threads,
                                           int32_t combine_tile) {
    if (!B) return BM_E_INPUT;
    if (combine_tile != 32 && combine_tile != 64) {
        snprintf(B->err, sizeof B->err, "bm_batch_set_schedule: combine_tile %d is not 32 or 64", combine_tile);
        return BM_E_INPUT;
    }
    if (persistent && !B->can_persist) {
        snprintf(B->err, sizeof B->err, "bm_batch_set_schedule: no persistent schedule (largest instance %d > %d or "
                 "the kernel does not fit)", B->max_n, kBSortMax);
        return BM_E_INPUT;
    }
    if (!persistent && profit_threads != 256 && profit_threads != 512) {
        snprintf(B->err, sizeof B->err, "bm_batch_set_schedule: profit_threads %d is not 256 or 512", profit_threads);
        return BM_E_INPUT;
    }
    B->use_persist = persistent != 0;
    B->profit_threads = persistent ? kBThreads : profit_threads;
    B->tile = combine_tile;
    bm_status s = batch_tiles(B);
    if (s) return s;
    if (B->exec) { cudaGraphExecDestroy(B->exec); B->exec = nullptr; }
    if (B->graph) { cudaGraphDestroy(B->graph); B->graph = nullptr; }
    return BM_OK;
}

extern "C" bm_status bm_batch_sweeps(bm_batch* B, int32_t sweeps, const bm_sweep_opts* opts,
                                     int64_t* committed, float* ms) {
    if (!B || sweeps < 0) return BM_E_INPUT;
    for (bm_ctx* c : B->ctx)
        if (!c->mapped) { snprintf(B->err, sizeof B->err, "bm_batch_sweeps: mappings not set"); return BM_E_STATE; }
    const int max_scan = opts ? opts->max_candidates : 0;
    const int max_verify = opts ? opts->max_verify : -1;
    // one sweep of the whole batch as a CUDA graph, captured once per option set
    if (B->exec && (max_scan != B->graph_max_scan || max_verify != B->graph_max_verify)) {
        cudaGraphExecDestroy(B->exec); B->exec = nullptr;
        cudaGraphDestroy(B->graph); B->graph = nullptr;
    }
    if (!B->exec) {
        BK(cudaStreamBeginCapture(B->st, cudaStreamCaptureModeThreadLocal));
        bm_status s = enqueue_sweep(B, max_scan, max_verify);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(B->st, &g);
        if (s) { if (g) cudaGraphDestroy(g); return s; }
        BK(ce);
        B->graph = g;
        BK(cudaGraphInstantiate(&B->exec, B->graph, 0));
        B->graph_max_scan = max_scan;
        B->graph_max_verify = max_verify;
    }
    BK(cudaMemsetAsync(B->acc_delta, 0, B->count * sizeof(long long), B->st));
    BK(cudaMemsetAsync(B->acc_commits, 0, B->count * sizeof(long long), B->st));
    // test hook (bm_test_stall): one sweep launched outside the graph whose
    // first grid barrier never completes
    const int stall = (B->use_persist && sweeps > 0) ? take_stall(BM_STALL_BATCH) : 0;
    BK(cudaEventRecord(B->ev0, B->st));
    if (stall) {
        bm_status s = B->w16 ? enqueue_persistent<true>(B, max_scan, max_verify, 1)
                             : enqueue_persistent<false>(B, max_scan, max_verify, 1);
        if (s) return s;
        sweeps = 0;
    }
    for (int i = 0; i < sweeps; i++) BK(cudaGraphLaunch(B->exec, B->st));
    BK(cudaEventRecord(B->ev1, B->st));
    std::vector<long long> dsum(B->count), csum(B->count);
    BK(cudaMemcpyAsync(dsum.data(), B->acc_delta, B->count * sizeof(long long), cudaMemcpyDeviceToHost, B->st));
    BK(cudaMemcpyAsync(csum.data(), B->acc_commits, B->count * sizeof(long long), cudaMemcpyDeviceToHost, B->st));
    unsigned gerr = 0;
    if (B->use_persist) BK(cudaMemcpyAsync(&gerr, B->gbar + 2, sizeof gerr, cudaMemcpyDeviceToHost, B->st));
    BK(cudaStreamSynchronize(B->st));
    if (gerr) {
        // a grid-barrier wait of the persistent sweep ran out: the matchings
        // may be partly committed; the caller sets them again
        BK(cudaMemset(B->gbar, 0, 4 * sizeof(unsigned)));
        for (bm_ctx* c : B->ctx) { c->mapped = false; c->S_exact = false; }
        snprintf(B->err, sizeof B->err, "bm_batch_sweeps: persistent sweep grid barrier wait timed out");
        return BM_E_TIMEOUT;
    }
    for (int i = 0; i < B->count; i++) {
        B->ctx[i]->score += dsum[i];
        if (committed) committed[i] = csum[i];
    }
    if (ms) BK(cudaEventElapsedTime(ms, B->ev0, B->ev1));
    return BM_OK;
}

extern "C" bm_status bm_batch_info(const bm_batch* B, int32_t* count, int32_t* max_n, int64_t* total_pairs,
                                   int32_t* profit_threads, int32_t* combine_tile) {
    if (!B) return BM_E_INPUT;
    long long pairs = 0;
    for (bm_ctx* c : B->ctx) pairs += (long long)c->n * (c->n - 1) / 2;
    if (count) *count = B->count;
    if (max_n) *max_n = B->max_n;
    if (total_pairs) *total_pairs = pairs;
    if (profit_threads) *profit_threads = B->profit_threads;
    if (combine_tile) *combine_tile = B->tile;
    return BM_OK;
}
