/*
 * bm.h -- C ABI of the B200 swap-delta engine for brain-match graph alignment.
 *
 * Problem: two directed, integer-weighted graphs G1 ("male", gm) and G2
 * ("female", gf) on vertex ids 1..n, and a matching map[m] = f (G1 -> G2,
 * 1-based, map[0] unused, 0 = unmatched).  The alignment score is
 *
 *     score(map) = sum over G1 edges (u,v,w):  min(w, w2(map[u], map[v]))
 *
 * (brain-match src/graph-alignment-optimized.c:292-307).  The engine computes
 * the exact change of that score for swaps map[a] <-> map[b] and for 3-cycles,
 * and hill-climbs by committing improving moves.
 *
 * Every function returns a bm_status (0 = OK, negative = error) and never
 * calls exit().  The caller owns every host array it passes; arrays are copied
 * in or out before the call returns.  The context owns all device memory.  One
 * host thread per context; contexts are independent.
 *
 * Graph semantics follow the reference loaders
 * (src/graph-alignment-optimized.c:183-204,635-679):
 *   - G1 edges are summed per list entry, so duplicate G1 edges each count
 *     (the reference keeps every copy in its edge lists);
 *   - G2 is looked up as a dense matrix, so a repeated G2 edge keeps the LAST
 *     weight given (the reference overwrites adj_matrix[from][to]);
 *   - zero-weight edges contribute nothing and are dropped; negative weights
 *     and ids outside 1..n are rejected with BM_E_INPUT.
 * Deltas are mathematically exact.  They equal the reference's
 * calculate_swap_delta whenever G1 has no self-loops and no repeated edge
 * between the two swapped vertices (the reference is inexact there), and
 * weights are <= 32767 (the reference stores weights in `short`).
 */
#ifndef BM_H
#define BM_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t bm_status;
#define BM_OK          0
#define BM_E_INPUT    -1   /* bad argument, malformed graph or mapping        */
#define BM_E_CUDA     -2   /* a CUDA call failed (no device, launch error ...) */
#define BM_E_OVERFLOW -3   /* a delta could exceed int32                       */
#define BM_E_TIMEOUT  -4   /* a bounded device wait ran out                    */
#define BM_E_NOMEM    -5   /* host or device allocation failed                 */
#define BM_E_STATE    -6   /* call out of order (e.g. no mapping set)          */
#define BM_E_IO       -7   /* file could not be opened / written               */

/* Flags for bm_create. */
#define BM_FLAG_FORCE_I32   0x1u  /* int32 entries even when 16-bit ones fit        */
#define BM_FLAG_NO_HUB_GEMM 0x2u  /* no tensor-core hub term (all terms scattered)   */

typedef struct bm_ctx bm_ctx;

/* Human-readable name of a status code (static string). */
const char* bm_status_string(bm_status s);

/* Text of the last error on this context ("" if none).  ctx may be NULL, in
 * which case the last error of a failed bm_create on this thread is returned. */
const char* bm_last_error(const bm_ctx* ctx);

/*
 * Build a context on the current CUDA device from two COO edge lists with
 * 1-based vertex ids in 1..n.
 * Replaces: load_graph_from_csv + new_graph/add_edge + the host->device copies
 * of the dense matrices (src/graph-alignment-optimized.c:125-204,635-679;
 * src/quick.cu:1047-1062).  Storage is chosen per input: 16-bit entries when
 * n <= 65536 and min(max w1, max w2) <= 65535 (results stay exact), 32-bit
 * otherwise or with BM_FLAG_FORCE_I32.
 */
bm_status bm_create(bm_ctx** out, int32_t n,
                    int64_t e1, const int32_t* src1, const int32_t* dst1, const int32_t* w1,
                    int64_t e2, const int32_t* src2, const int32_t* dst2, const int32_t* w2,
                    uint32_t flags);

void bm_destroy(bm_ctx* ctx);

/* Information about a context. */
typedef struct {
    int32_t n;
    int32_t entry_bits;      /* 16 or 32 */
    int64_t e1, e2;          /* stored list entries (after drops/dedupe)   */
    int64_t g1_self_loops;   /* G1 self-loop entries (handled exactly)     */
    int64_t device_bytes;    /* device memory held by the context          */
    int32_t device;          /* CUDA ordinal                               */
    int32_t num_sms;
    int32_t hubs;            /* G1 hubs whose in-edge terms use the tensor cores */
    int32_t hub_k;           /* GEMM depth (hubs x thresholds), 0 if none  */
} bm_info;
bm_status bm_get_info(const bm_ctx* ctx, bm_info* info);

/*
 * Set / read the matching, map[1..n] in 1..n (0 = unmatched), an injective map.
 * Mirrors the int mapping[NUM_NODES+1] of the reference
 * (src/graph-alignment-optimized.c:428-475, src/quick.cu:1163-1166).
 */
bm_status bm_set_mapping(bm_ctx* ctx, const int32_t* map);
bm_status bm_get_mapping(bm_ctx* ctx, int32_t* map);

/*
 * Alignment score of the current matching.
 * Replaces calculate_alignment_score (src/graph-alignment-optimized.c:292-307).
 */
bm_status bm_score(bm_ctx* ctx, int64_t* score);

/*
 * Exact swap deltas for k given pairs (m1[i], m2[i]), 1-based, m1 != m2.
 * Replaces calculate_swap_delta (src/graph-alignment-optimized.c:321-408).
 */
bm_status bm_pair_deltas(bm_ctx* ctx, int64_t k, const int32_t* m1, const int32_t* m2,
                         int32_t* out);

/*
 * bm_pair_deltas_static -- the same deltas as bm_pair_deltas for up to
 * BM_STATIC_MAX_PAIRS pairs, without allocating any memory.
 * No counterpart in the reference.
 *
 * bm_pair_deltas stages the pairs and their results in device memory that the
 * context allocates with cudaMalloc the first time a call needs more room.
 * Some callers cannot let that happen:
 *   - a process whose GPU memory is already handed out to another allocator
 *     (a framework's caching allocator, a fixed memory pool), where a new
 *     cudaMalloc fails or pushes the pool out of memory mid-search;
 *   - a loop that scores a few candidate swaps between other GPU work, where
 *     cudaMalloc/cudaFree can synchronize the whole device and stall the
 *     other streams.
 * This entry point stages through one fixed array compiled into the library
 * (a static __device__ array of 3 * BM_STATIC_MAX_PAIRS int32, 768 KiB).  Every
 * GPU that loads the library holds that array until the process exits.
 *
 * Limits and sharing:
 *   - k > BM_STATIC_MAX_PAIRS is rejected with BM_E_INPUT; split the work.
 *   - The first call on a device looks up the array's device address
 *     (cudaGetSymbolAddress, with that device current) and keeps it for the
 *     life of the process; make that first call before capturing any CUDA
 *     stream.  Each call makes the context's device current for its copies
 *     and launch and restores the caller's device before it returns.
 *   - The kept address belongs to the device's primary context: after a
 *     cudaDeviceReset the library (every bm_ctx included) must not be used
 *     again in that process.
 *   - All calls in the process share the one array, which keeps the last
 *     call's contents.  Nothing in it has to start at zero: each call writes
 *     every result it copies back.  Calls that overlap on the GPU (two
 *     contexts, or two host threads, at the same time on one device) race on
 *     the array; serialize them.  Each call waits for its own work before it
 *     returns.
 * Arguments and errors are those of bm_pair_deltas.
 */
#define BM_STATIC_MAX_PAIRS 65536
bm_status bm_pair_deltas_static(bm_ctx* ctx, int64_t k, const int32_t* m1, const int32_t* m2,
                                int32_t* out);

/*
 * Exact deltas of all n(n-1)/2 unordered pairs in the reference's linear pair
 * order (index 0 = (1,2), (1,3), ..., (1,n), (2,3), ...), written to the host
 * array out.  Replaces calculateSwapDeltasKernel + its D2H copy
 * (src/graph-re-alignment-gpu.cu:38-131,845-857; src/quick.cu:48-137).
 */
bm_status bm_all_deltas(bm_ctx* ctx, int32_t* out);

/*
 * Per-vertex profit row: out[b-1] = score that vertex a would contribute if it
 * took map[b] with every other vertex fixed (b = 1..n); out[a-1] is a's current
 * contribution.  Diagnostic view of the matrix the sweep is built on.
 */
bm_status bm_profit_row(bm_ctx* ctx, int32_t a, int32_t* out);

/* ---- Pairwise hill-climbing sweep (full all-pairs evaluation + commit) ---- */
typedef struct {
    int32_t max_candidates;  /* sorted candidates scanned per sweep (<=0: all)   */
    int32_t max_verify;      /* re-verifications of tainted candidates (<0: all) */
    int32_t commit_ctas;     /* CTAs (one thread-block cluster) sharing the set
                                commit's list scans: 0 = default (8), 1..8;
                                results never depend on it                      */
    int32_t incremental;     /* 1: keep the profit matrix exact across sweeps and
                                update it from the vertices the last commit moved
                                when that is cheaper than a rebuild; results never
                                depend on it                                     */
    int32_t reserved[4];
} bm_sweep_opts;

typedef struct {
    int64_t score_before;
    int64_t score_after;
    int64_t deltas_evaluated;   /* n(n-1)/2 per sweep                   */
    int32_t candidates;         /* rows whose best swap is improving     */
    int32_t scanned;            /* candidates looked at by the commit    */
    int32_t verified;           /* tainted candidates re-evaluated       */
    int32_t committed;          /* swaps applied                         */
    int32_t best_delta;         /* largest delta of the sweep            */
    int32_t profit_mode;        /* 0 rebuilt, 1 updated from the moved
                                   vertices, 2 already exact              */
    /* device time (CUDA events on the context's stream), milliseconds:      */
    float   ms_profit;          /* profit-row kernel alone                */
    float   ms_combine;         /* pair combine + per-row best            */
    float   ms_commit;          /* candidate sort + sequential commit     */
    float   ms_total;           /* whole sweep                            */
    float   ms_prep;            /* relabelling + row scheduling           */
    float   ms_hub;             /* hub operands + tensor-core GEMM        */
    int64_t min_terms;          /* nonzero min terms scattered by a rebuild,
                                   list entries applied by an update       */
    int64_t commit_entries;     /* edge-list entries read by the commit   */
    int32_t commit_steps;       /* commit steps (pairs decided per step)  */
    int32_t commit_carried;     /* pairs carried into a later step        */
} bm_sweep_stats;

/*
 * One sweep: evaluate every pair, take each vertex's best partner, sort the
 * improving ones by (delta desc, lower id asc, higher id asc), then in that
 * order commit each pair whose vertices are still untouched and whose delta,
 * re-evaluated on the updated matching, is still > 0.
 * Replaces the sweep + host argmax + commit of src/graph-re-alignment-gpu.cu:
 * 845-891 and the best-per-row loop of src/alignment-omp.c:601-658.
 */
bm_status bm_sweep(bm_ctx* ctx, const bm_sweep_opts* opts, bm_sweep_stats* stats);

/*
 * Sweeps until no improving swap remains or max_sweeps is reached.
 * per_sweep (may be NULL) receives one record per sweep.
 */
bm_status bm_hillclimb(bm_ctx* ctx, int32_t max_sweeps, const bm_sweep_opts* opts,
                       bm_sweep_stats* per_sweep, int32_t* sweeps_done);

/*
 * The reference's sequential first-improvement order
 * (src/graph-alignment-optimized.c:515-577): for m1 = 1..n, for m2 = 1..n,
 * m2 != m1, commit the swap if its delta on the current matching is > 0.
 * Runs up to max_passes full passes, stopping after a pass with no commit
 * (the reference loops forever).  Commits and passes are reported.
 */
bm_status bm_first_improvement(bm_ctx* ctx, int32_t max_passes, int64_t* commits,
                               int32_t* passes_done);

/*
 * Device timer on the context's stream: record event `slot` (0..7) now, and
 * read the elapsed milliseconds between two recorded slots (synchronizes).
 * Lets a caller time a run of calls on the device, e.g. K sweeps.
 */
bm_status bm_timer_mark(bm_ctx* ctx, int32_t slot);
bm_status bm_timer_elapsed(bm_ctx* ctx, int32_t start_slot, int32_t end_slot, float* ms);

/*
 * Microbenchmarks behind the sweep's roofline figures, on the current device:
 * *red_per_s = shared-memory atomic adds per second at random addresses of an
 * n-int array at full occupancy (the profit-row kernel's inner operation);
 * *minadd_per_s = independent int32 (min, add) pairs per second.
 * Allocates a 4-byte scratch word; diagnostic, not on the hot path.
 */
bm_status bm_measure_peaks(int32_t n, double* red_per_s, double* minadd_per_s);

/*
 * Test hook for the timeout paths; no counterpart in the reference.
 * Every wait a kernel makes on another part of the GPU (an mbarrier that the
 * tensor cores or a copy complete, a cluster or grid barrier) is bounded:
 * when it runs out the kernel records an error word, waits (bounded) for its
 * own copies in flight, releases what it holds and returns, and the call
 * reports BM_E_TIMEOUT with the site in bm_last_error.  bm_test_stall(site)
 * makes the next launch at that site take one such wait that nothing
 * completes (CTA 0 skips an arrival, or waits for a barrier phase nothing
 * opens), with a short limit -- no fault, trap or endless loop.  One site at
 * a time, process-wide; 0 clears it.  After BM_E_TIMEOUT a context's matching
 * may be partly committed: set a matching again before the next call.
 */
#define BM_STALL_HUB_GEMM   1   /* bm_sweep: tensor-core hub GEMM          */
#define BM_STALL_COMMIT     2   /* bm_sweep: set commit cluster exchange   */
#define BM_STALL_COMBINE    3   /* bm_sweep: TMA-fed pair combine          */
#define BM_STALL_GREEDY     4   /* bm_greedy_match: grid barrier           */
#define BM_STALL_MLP_GEMM   5   /* bm_mlp_*: tensor-core GEMM              */
#define BM_STALL_BATCH      6   /* bm_batch_sweeps: persistent sweep grid barrier */
bm_status bm_test_stall(int32_t site);

/* ---- Exact swap-lookup table ----
 * The reference's best-swap tools keep an n x n table of swap deltas
 * (src/best-swap/create-score-lookup.c:289-296) and a heap of its positive
 * entries; after each swap they recompute only the rows and columns of the
 * two swapped vertices (src/best-swap/score-lookup.c:514-537), so every pair
 * next to them goes stale.  Here the table is the context's profit matrix,
 * kept exact across commits by the update of bm_sweep_opts.incremental (every
 * term that the moved vertices change), and the heap is each row's best
 * partner, recomputed from the exact table at every step. */

/*
 * Rows a0 .. a0+rows-1 (1-based) of the exact delta table on the current
 * matching: out[(a-a0)*n + (b-1)] = delta of swapping map[a] and map[b],
 * 0 for b == a.  The create-score-lookup table, row-chunked so a caller can
 * stream n x n entries to a file.
 */
bm_status bm_lookup_rows(bm_ctx* ctx, int32_t a0, int32_t rows, int32_t* out);

typedef struct {
    int64_t score_before, score_after;
    int32_t swaps;          /* swaps committed                               */
    int32_t converged;      /* 1: stopped because no swap improves           */
    int32_t refresh_mode;   /* how the table was made exact first: 0 rebuilt,
                               1 updated, 2 already exact                     */
    int32_t reserved;
    float   ms_refresh;     /* device time of making the table exact        */
    float   ms_total;       /* device time of the whole call                 */
} bm_lookup_stats;

/*
 * Best-swap descent (the extract_max / swap / update loop of
 * src/best-swap/score-lookup.c:597-640) on the exact table: each step commits
 * the swap of largest delta over all pairs (ties: smallest first vertex, then
 * smallest second) while it is > 0, then updates the table, up to max_swaps
 * swaps.  Zero-delta and temperature-accepted swaps (:548-595) are not made:
 * with an exact table a zero-delta swap is followed by its own reversal.
 */
bm_status bm_lookup_descent(bm_ctx* ctx, int32_t max_swaps, bm_lookup_stats* stats);

/* ---- 3-cycles ---- */

/*
 * Exact deltas of the two cyclic rotations of each triple (a[i],b[i],c[i]),
 * distinct 1-based ids:  out[2i]   = delta of (map[a],map[b],map[c]) <- (f2,f3,f1)
 *                        out[2i+1] = delta of (map[a],map[b],map[c]) <- (f3,f1,f2)
 * i.e. permutations 3 and 4 of calculateThreeNodeSwapKernel
 * (src/triple.cu:85-92) as applied by apply_permutation (src/triple.cu:903-934).
 */
bm_status bm_triple_deltas(bm_ctx* ctx, int64_t k, const int32_t* a, const int32_t* b,
                           const int32_t* c, int32_t* out);

typedef struct {
    int32_t partners;        /* 2-hop samples per vertex (256)            */
    int32_t max_candidates;  /* sorted candidates scanned (<=0: all)      */
    int32_t max_verify;      /* re-verifications (<0: all)                */
    int32_t incremental;     /* 1: keep the profit matrix exact across rounds
                                (as bm_sweep_opts.incremental); same moves   */
    uint64_t seed;           /* round seed for the 2-hop sampler          */
    int32_t reserved[4];
} bm_triple_opts;

typedef struct {
    int64_t score_before, score_after;
    int64_t triples;            /* valid sampled triples               */
    int64_t rotations;          /* 2 per triple                        */
    int32_t candidates, scanned, verified, committed;
    int32_t best_delta, reserved;
    float   ms_sample, ms_eval, ms_commit, ms_total;
} bm_triple_stats;

/*
 * One 3-cycle round: sample `partners` 2-hop paths (a -> b -> c, undirected
 * G1 neighbourhoods) per vertex a, evaluate both rotations of each triple
 * exactly, and commit the best vertex-disjoint improving set under the same
 * re-verification rule as bm_sweep.  Replaces the batch loop of
 * src/triple.cu:1074-1157 (which visits only a few batches per pass).
 */
bm_status bm_triple_round(bm_ctx* ctx, const bm_triple_opts* opts, bm_triple_stats* stats);

/* ---- 4-set permutations ---- */

/*
 * Exact deltas of permuting the images of 4-vertex sets: set i is
 * sets[4i..4i+3] (distinct 1-based ids), perms[i] in 1..23 is the q-th
 * permutation of (0,1,2,3) in lexicographic order (0 would be the identity),
 * and vertex sets[4i+t] takes the image of vertex sets[4i+perm_q[t]].  The
 * k = 4 case of generate_permutations (src/permutation.c:700-744), scored
 * like calculate_permutation_delta (:623-696).
 */
bm_status bm_quad_deltas(bm_ctx* ctx, int64_t k, const int32_t* sets, const int32_t* perms, int32_t* out);

typedef struct {
    int32_t partners;        /* 3-step walk samples per vertex (64, at most 2048) */
    int32_t max_candidates;  /* sorted candidates scanned (<=0: all)              */
    int32_t max_verify;      /* re-verifications (<0: all)                        */
    int32_t incremental;     /* as in bm_triple_opts                       */
    uint64_t seed;           /* round seed for the sampler                        */
    int32_t reserved[4];
} bm_quad_opts;

typedef struct {
    int64_t score_before, score_after;
    int64_t quads;              /* valid sampled 4-sets                 */
    int64_t permutations;       /* 23 per 4-set                         */
    int32_t candidates, scanned, verified, committed;
    int32_t best_delta, reserved;
    float   ms_sample, ms_eval, ms_commit, ms_total;
} bm_quad_stats;

/*
 * One 4-set round: sample `partners` connected 4-sets per vertex a (a 3-step
 * walk a -> b -> c -> d along undirected G1 edges), evaluate all 23
 * non-identity permutations of their images exactly (from the profit matrix
 * plus the set's internal edges), keep each vertex's best, and commit the best
 * vertex-disjoint improving sets under the re-verification rule of
 * bm_triple_round.  The reference enumerates all k-subsets for this
 * (src/permutation.c:746-800); sampling connected sets keeps it exact per
 * move and linear in n per round.
 */
bm_status bm_quad_round(bm_ctx* ctx, const bm_quad_opts* opts, bm_quad_stats* stats);

/* ---- Batches of independent instances ---- */

/*
 * Many independent graph pairs of uneven size swept together: every
 * instance keeps the single-instance semantics (bm_create, bm_sweep), and a
 * batch sweep runs all of them together, captured once as a CUDA graph and
 * replayed, in one of two schedules: one persistent cooperative launch that
 * runs every phase of the sweep for every instance behind grid barriers
 * (instances up to 8,192 vertices), or a launch sequence -- one persistent
 * profit-row launch over every (instance, row), one combine launch over
 * every (instance, tile), one commit launch with a CTA per instance.  The
 * reference runs
 * independent instances as separate processes (MPI replicas,
 * src/mpi-omp.c:76-122) each with the sweep of
 * src/graph-re-alignment-gpu.cu:845-891.  The tensor-core hub term is not
 * used in batches.
 */
typedef struct bm_batch bm_batch;

/* Instance i has n[i] vertices and the edge arrays src1[i][0..e1[i]) etc. */
bm_status bm_batch_create(bm_batch** out, int32_t count, const int32_t* n,
                          const int64_t* e1, const int32_t* const* src1, const int32_t* const* dst1,
                          const int32_t* const* w1,
                          const int64_t* e2, const int32_t* const* src2, const int32_t* const* dst2,
                          const int32_t* const* w2, uint32_t flags);
void bm_batch_destroy(bm_batch* b);
/* Last error of the batch (b may be NULL after a failed bm_batch_create). */
const char* bm_batch_last_error(const bm_batch* b);
bm_status bm_batch_set_mappings(bm_batch* b, const int32_t* const* maps);
bm_status bm_batch_get_mappings(bm_batch* b, int32_t* const* maps);
bm_status bm_batch_scores(bm_batch* b, int64_t* scores);
/*
 * Times the candidate schedules on whole sweeps of the batch itself (the
 * second and third sweep from the current matchings, which it restores) and
 * keeps the fastest: the persistent
 * launch (reported as profit_threads = 1024) with combine tile 32 or 64, and
 * the launch sequence with profit-row blocks of 256 or 512 threads and tile
 * 32 or 64.  Results never depend on the choice.
 */
bm_status bm_batch_autotune(bm_batch* b, int32_t* profit_threads, int32_t* combine_tile);
/*
 * Sets the schedule directly: persistent != 0 for the one-launch sweep
 * (BM_E_INPUT if the batch's largest instance exceeds 8,192 vertices), else
 * the launch sequence with profit_threads 256 or 512; combine_tile 32 or 64.
 */
bm_status bm_batch_set_schedule(bm_batch* b, int32_t persistent, int32_t profit_threads, int32_t combine_tile);
/*
 * Runs `sweeps` sweeps of every instance (graph replays).  committed (may be
 * NULL) receives per-instance swap counts; *ms the device time.
 * BM_E_TIMEOUT if a grid-barrier wait of the persistent schedule ran out
 * (the matchings must then be set again).
 */
bm_status bm_batch_sweeps(bm_batch* b, int32_t sweeps, const bm_sweep_opts* opts, int64_t* committed,
                          float* ms);
bm_status bm_batch_info(const bm_batch* b, int32_t* count, int32_t* max_n, int64_t* total_pairs,
                        int32_t* profit_threads, int32_t* combine_tile);

/* ---- Learned swap proposal ----
 *
 * A small network ranks candidate swaps so that only the top-ranked ones are
 * evaluated exactly; the exact integer delta (bm_pair_deltas' arithmetic)
 * judges every move and the engine's set commit applies them, so scores stay
 * exact whatever the network says.  The reference has no learned component;
 * its exhaustive sweep (src/graph-re-alignment-gpu.cu:845-891) is the
 * fallback.
 *
 * Network: 128 -> 256 -> 256 -> 1, ReLU, bf16 weights and activations with
 * fp32 accumulation on the tensor cores, fp32 master weights, plain SGD on the
 * mean squared error.  Input of a pair (a, b) with images p(a), p(b):
 * [f1(a), f1(b), f2(p(a)), f2(p(b))], 32 features per vertex (see
 * bm_mlp_features).  Target: sign(d) log1p|d| of the exact delta d.
 *
 * Parameter layout (fp32, bm_mlp_param_count() values): W1[256][128], b1[256],
 * W2[256][256], b2[256], w3[256], b3.  Layer l computes
 * h_l = relu(W_l h_{l-1} + b_l); y = w3 . h2 + b3.
 */
typedef struct bm_mlp bm_mlp;

typedef struct {
    int64_t samples;    /* training rows seen (over epochs)        */
    int64_t steps;      /* SGD steps (batches of 1024 rows)        */
    float first_loss;   /* mean batch loss over the first epoch    */
    float last_loss;    /* mean batch loss over the last epoch     */
} bm_mlp_train_stats;

typedef struct {
    int32_t pool;          /* partners ranked per vertex (default 64)            */
    int32_t per_row;       /* > 0: each vertex's per_row best-ranked partners are
                              evaluated (n * per_row pairs; pool <= 1024,
                              per_row <= 32); 0: the top_fraction below       */
    double top_fraction;   /* fraction of the whole ranked pool evaluated exactly
                              when per_row == 0 (default 0.02)                 */
    uint64_t seed;         /* pool sampling seed                                 */
    int32_t retries;       /* further attempts with a fresh pool before the
                              exhaustive fallback (default 0)                  */
    int32_t reserved;
} bm_learned_opts;

int64_t bm_mlp_param_count(void);
/* He-uniform weights from a seeded generator, zero biases; on the current device. */
bm_status bm_mlp_create(bm_mlp** out, uint64_t seed);
void bm_mlp_destroy(bm_mlp* m);
/* Last error of the network (m may be NULL after a failed bm_mlp_create). */
const char* bm_mlp_last_error(const bm_mlp* m);
bm_status bm_mlp_get_params(bm_mlp* m, float* params);
bm_status bm_mlp_set_params(bm_mlp* m, const float* params);
/*
 * The per-vertex features of ctx's graphs under its current matching, as the
 * network sees them: f1[a*32 + c] for G1 vertex a, f2[f*32 + c] for G2 vertex
 * f (0-based ids).  Columns before normalisation: 0/1 out/in degree, 2/3
 * out/in weight sums, 4/5 2-hop out/in counts, 6/7 max out/in weight, 8 G1
 * self-loop weight, 9 current overlap contribution (G2: of the G1 vertex
 * matched to it), all through log1p; 10 that contribution / (incident
 * weight + 1); 11..31 zero.  Each column is then z-scored over the vertices
 * (population std; 0 for a constant column).
 */
bm_status bm_mlp_features(bm_mlp* m, bm_ctx* ctx, float* f1, float* f2);
/*
 * Network scores of k vertex pairs (m1[i], m2[i]), 1-based, on ctx's current
 * matching: the ranking the learned sweep uses, computed with the factorised
 * first layer and the fused tensor-core kernel.
 */
bm_status bm_mlp_rank_pairs(bm_mlp* m, bm_ctx* ctx, int64_t k, const int32_t* m1, const int32_t* m2, float* out);
/* out[i] = network(x[i]) for k rows of 128 fp32 inputs (rounded to bf16). */
bm_status bm_mlp_forward(bm_mlp* m, int64_t k, const float* x, float* out);
/*
 * One forward and backward pass over k rows: loss = mean (y - t)^2, grads
 * (may be NULL) receive dloss/dparams in the parameter layout, then
 * params -= lr * grads unless lr == 0.
 */
bm_status bm_mlp_train_step(bm_mlp* m, int64_t k, const float* x, const float* target, float lr,
                            float* loss, float* grads);
/*
 * Trains on data the engine generates.  First it logs `sweeps` rounds: each
 * builds the exact profit matrix of ctx's current matching, records per
 * vertex its best partner plus `extra_partners` candidate-pool partners with
 * their exact deltas (and the round's features), then advances the matching
 * with one ordinary bm_sweep.  Then it runs `epochs` passes of SGD (batches
 * of 1024, learning rate lr) over all logged samples, shuffled afresh each
 * epoch.  ctx's matching is left where the last logged sweep put it.
 */
bm_status bm_mlp_train_from(bm_mlp* m, bm_ctx* ctx, int32_t sweeps, int32_t extra_partners, int32_t epochs,
                            float lr, uint64_t seed, bm_mlp_train_stats* stats);
/*
 * One learned sweep.  The candidate pool holds opts->pool partners per
 * vertex a, each a vertex b whose image a's G1 neighbours' images point at
 * (b = pinv(f) for f a G2 neighbour of p(v), v a G1 neighbour of a, on the
 * matching side of the edge).  The network ranks the pool; exactly evaluated
 * are either the top opts->top_fraction of the whole pool or each vertex's
 * opts->per_row best-ranked partners; the improving ones are committed in
 * (delta desc, lo, hi) order with the exact set commit of bm_sweep.  When none
 * improves, opts->retries more attempts draw fresh pools, and when those fail
 * too an exhaustive bm_sweep runs instead (*fell_back = 1).
 * Stats: deltas_evaluated = exact evaluations, candidates = pool pairs ranked;
 * phase times ms_prep (features and pool), ms_hub (network ranking),
 * ms_combine (selection and exact deltas), ms_commit (candidate sort and set
 * commit); after a fallback ms_total also holds the exhaustive sweep.
 */
bm_status bm_learned_sweep(bm_ctx* ctx, bm_mlp* m, const bm_learned_opts* opts, bm_sweep_stats* stats,
                           int32_t* fell_back);

/*
 * The learned-proposal descent: hill-climbs ctx's matching with learned and
 * exhaustive sweeps until its score reaches target_score (> 0), an exhaustive
 * sweep commits nothing (a local optimum of the whole swap neighbourhood), or
 * max_sweeps steps have run.  Schedule: the first step is a learned sweep,
 * the second an exhaustive one; after that a learned sweep runs while the
 * last learned sweep gained at least as much score per device-millisecond as
 * the last exhaustive one, and otherwise exhaustive sweeps run, with one
 * learned probe after every probe_every (0: 8) exhaustive sweeps in a row.  A
 * learned sweep that finds nothing is followed by an exhaustive sweep within
 * the same step.  Every move is judged and committed exactly.
 * Optional traces (max_sweeps entries each): the score after each step, the
 * cumulative device milliseconds, the step's kind (0 exhaustive, 1 learned,
 * 2 learned then exhaustive).
 */
typedef struct {
    int32_t sweeps;       /* steps run                                         */
    int32_t learned;      /* learned sweeps                                    */
    int32_t exhaustive;   /* exhaustive sweeps (fallbacks included)            */
    int32_t reached;      /* 1: the score reached target_score                 */
    int32_t converged;    /* 1: stopped at a local optimum                     */
    int32_t reserved;
    int64_t score_before, score_after;
    int64_t committed;    /* swaps applied                                     */
    float ms_total;       /* device time of all steps                          */
    float ms_learned;     /* of which learned sweeps                           */
    float ms_exhaustive;  /* of which exhaustive sweeps                        */
    float reserved2;
} bm_learned_run_stats;
bm_status bm_learned_run(bm_ctx* ctx, bm_mlp* m, const bm_learned_opts* opts, int32_t max_sweeps,
                         int64_t target_score, int32_t probe_every, bm_learned_run_stats* stats,
                         int64_t* trace_score, float* trace_ms, int8_t* trace_kind);

/* ---- Initial matching: the greedy feature matcher ----
 * src/greedy-feature-match.c:527-712.  G1 vertices, in order of their
 * feature total (in-degree + out-degree + distinct 2-hop out-reach + distinct
 * 2-hop in-reach; descending, ties by id), each take the unmatched G2 vertex of
 * largest 0.3 * -distance + 0.7 * align: distance = (int)(1000 * sum |r1 - r2|)
 * over the four feature / total ratios, align = sum of min(w1, w2) over the
 * vertex's G1 edges to already matched neighbours and the corresponding G2
 * edges of the candidate; equal scores go to the candidate first in G2's
 * feature order.  Degrees count every edge given (repeats and self-loops); W2
 * is the last weight given for a G2 pair.  A vertex without edges has ratios 0
 * (the reference divides 0/0 there), and align compares G2 vertices with G2
 * vertices (the reference compares ids with indices).  Independent of any
 * bm_ctx; runs on the current device. */
typedef struct {
    float ms_features;   /* device time of both graphs' adjacency lists,
                            features and orders                            */
    float ms_match;      /* device time of the sequential matching          */
    int32_t reserved[2];
} bm_greedy_stats;

/* map (n+1 entries) receives the matching, 1-based, map[0] = 0.  Errors are
 * reported by bm_last_error(NULL). */
bm_status bm_greedy_match(int32_t n, int64_t e1, const int32_t* src1, const int32_t* dst1, const int32_t* w1,
                          int64_t e2, const int32_t* src2, const int32_t* dst2, const int32_t* w2,
                          int32_t* map, bm_greedy_stats* stats);

/* The features of one graph (compute_vertex_features, :527-566):
 * out[4(v-1) + k] for v = 1..n, k = in-degree, out-degree, distinct 2-hop
 * out-reach, distinct 2-hop in-reach. */
bm_status bm_greedy_features(int32_t n, int64_t e, const int32_t* src, const int32_t* dst, const int32_t* w,
                             int32_t* out);

/* ---- Host utilities: file formats and the synthetic generator ---- */

/* Free memory returned by the readers below. */
void bm_free(void* p);

/*
 * Graph CSV: one header line, then "from,to,weight" integers.  Malformed lines
 * are skipped with a message on stderr, as load_graph_from_csv does
 * (src/graph-alignment-optimized.c:635-679).  Arrays are malloc'd; release
 * them with bm_free.
 */
bm_status bm_read_graph_csv(const char* path, int64_t* e, int32_t** src, int32_t** dst,
                            int32_t** w, int32_t* max_id);

/*
 * Matching CSV: one header line, then "m<id>,f<id>" or "<id>,<id>" lines, as
 * load_benchmark_mapping reads them (src/graph-alignment-optimized.c:428-475).
 * map must hold n+1 entries; it is zeroed first.  Ids outside 1..n are
 * rejected.  *count receives the number of lines read.
 */
bm_status bm_read_mapping_csv(const char* path, int32_t n, int32_t* map, int32_t* count);

/*
 * Writes "Male Node ID,Female Node ID" then "m%d,f%d" for every map[i] != 0,
 * exactly as write_mapping (src/graph-alignment-optimized.c:410-425).
 */
bm_status bm_write_mapping_csv(const char* path, int32_t n, const int32_t* map);

/*
 * Numeric matching format of refine-matching-hillclimb: header
 * "Male ID,Female ID" then "%d,%d" (src/refine-matching-hillclimb.c:454-503).
 */
bm_status bm_write_mapping_csv_numeric(const char* path, int32_t n, const int32_t* map);

/* Synthetic graph-pair generator (seeded, deterministic). */
typedef struct {
    int32_t n;             /* vertices                                           */
    int32_t wmax;          /* weight cap                                         */
    int64_t e;             /* G1 edges                                           */
    uint64_t seed;
    double  alpha;         /* out-degree power-law exponent (2.1)                */
    double  geom_p;        /* weight = 1 + Geometric(geom_p) failures (0.35)     */
    double  tail_prob;     /* probability of a heavy-tail weight (0 or 1e-3)     */
    double  tail_alpha;    /* heavy tail: floor(tail_scale * Pareto(tail_alpha)) */
    double  tail_scale;
    double  del_frac;      /* G2: fraction of relabelled G1 edges deleted (0.1)  */
    double  add_frac;      /* G2: random edges added, as a fraction of e (0.1)   */
    int32_t jitter;        /* G2: every weight += uniform{-jitter..jitter}, >= 1 */
    int32_t reserved;
} bm_gen_params;

/* Fills p with the defaults of the N=1,000 / 20,000-edge workload. */
void bm_gen_defaults(bm_gen_params* p);

/*
 * Generates G1 (exactly e edges, no self-loops, no duplicates, sorted by
 * (src,dst)), G2 = G1 relabelled by a random permutation with edges deleted,
 * added and jittered (sorted), and a uniform random initial matching.
 * Capacities: src1/dst1/w1 hold e entries, src2/dst2/w2 hold
 * e + ceil(add_frac*e) entries; pi and map0 hold n+1 entries (1-based; pi is
 * the hidden G1 -> G2 relabelling).  *e2 receives G2's edge count.
 */
bm_status bm_generate(const bm_gen_params* prm,
                      int32_t* src1, int32_t* dst1, int32_t* w1,
                      int64_t* e2, int32_t* src2, int32_t* dst2, int32_t* w2,
                      int32_t* pi, int32_t* map0);

#ifdef __cplusplus
}
#endif
#endif /* BM_H */
