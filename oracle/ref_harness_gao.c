/*
 * ref_harness_gao.c -- test infrastructure, not part of the engine.
 *
 * Compiles the reference's own src/graph-alignment-optimized.c in place (its
 * main() renamed) and exposes its score and swap-delta functions, plus an
 * OpenMP driver of calculate_swap_delta shaped like the race-free best-per-row
 * loop of src/alignment-omp.c:601-622 (parallel over partners m2 of each m1,
 * mapping held fixed).  Built into oracle/_ref/ by oracle/Makefile; only the
 * tests and bench.py's reference/CPU-baseline leg load it.
 */
#define main brain_match_reference_main
#include REF_SRC
#undef main
#include <omp.h>

/* Graph construction through the reference's own new_graph/add_edge. */
void* refgao_graph_new(void) { return new_graph(); }
void refgao_graph_add(void* g, int from, int to, int w) { add_edge((Graph*)g, from, to, w); }
void refgao_graph_add_many(void* g, long long m, const int* s, const int* d, const int* w) {
    for (long long i = 0; i < m; i++) add_edge((Graph*)g, s[i], d[i], w[i]);
}
void refgao_graph_free(void* g) { free_graph((Graph*)g); }
int refgao_num_nodes(void) { return NUM_NODES; }

/* mapping must hold NUM_NODES+1 entries (the reference indexes up to it). */
int refgao_score(void* gm, void* gf, int* mapping) {
    return calculate_alignment_score((Graph*)gm, (Graph*)gf, mapping);
}
int refgao_swap_delta(void* gm, void* gf, int* mapping, int m1, int m2) {
    return calculate_swap_delta((Graph*)gm, (Graph*)gf, mapping, m1, m2);
}
void refgao_pair_deltas(void* gm, void* gf, int* mapping, long long k, const int* m1, const int* m2,
                        int* out) {
    #pragma omp parallel for schedule(dynamic, 256)
    for (long long i = 0; i < k; i++)
        out[i] = calculate_swap_delta((Graph*)gm, (Graph*)gf, mapping, m1[i], m2[i]);
}

/*
 * For each listed row m1: delta(m1, m2) for every m2 in 1..n, m2 != m1, under
 * `#pragma omp parallel for schedule(dynamic)` with the mapping fixed (the
 * alignment-omp.c:601-622 shape without its serialising critical section).
 * Returns the number of deltas evaluated; *checksum receives their sum and
 * *threads the OpenMP thread count used.
 */
long long refgao_rows_omp(void* gm, void* gf, int* mapping, const int* rows, int nrows, int n,
                          long long* checksum, int* threads) {
    long long cnt = 0, sum = 0;
    int nt = 1;
    for (int r = 0; r < nrows; r++) {
        const int m1 = rows[r];
        #pragma omp parallel for schedule(dynamic, 64) reduction(+:cnt,sum)
        for (int m2 = 1; m2 <= n; m2++) {
            if (m2 == m1) continue;
            sum += calculate_swap_delta((Graph*)gm, (Graph*)gf, mapping, m1, m2);
            cnt++;
        }
    }
    #pragma omp parallel
    {
        #pragma omp single
        nt = omp_get_num_threads();
    }
    if (checksum) *checksum = sum;
    if (threads) *threads = nt;
    return cnt;
}

/*
 * The first-improvement loop of optimize_mapping (src/graph-alignment-
 * optimized.c:515-577) with the reference's own calculate_swap_delta,
 * validate_mapping_changes and post-commit calculate_alignment_score, over
 * m1, m2 in 1..n (ids above n have no edges and no positive delta), stopped
 * after a pass without a commit or after max_passes (the reference loops
 * forever and saves files; neither is timed here).  Returns the final score.
 */
int refgao_first_improvement(void* gm, void* gf, int* mapping, int n, int max_passes,
                             long long* commits, int* passes) {
    int* old_mapping = (int*)malloc(sizeof(int) * (NUM_NODES + 1));
    int score = calculate_alignment_score((Graph*)gm, (Graph*)gf, mapping);
    long long c = 0;
    int pass = 0;
    for (; pass < max_passes; pass++) {
        long long before = c;
        for (int m1 = 1; m1 <= n; m1++) {
            for (int m2 = 1; m2 <= n; m2++) {
                if (m1 == m2) continue;
                const int f1 = mapping[m1], f2 = mapping[m2];
                const int delta = calculate_swap_delta((Graph*)gm, (Graph*)gf, mapping, m1, m2);
                if (delta > 0) {
                    memcpy(old_mapping, mapping, sizeof(int) * (NUM_NODES + 1));
                    mapping[m1] = f2;
                    mapping[m2] = f1;
                    score += delta;
                    c++;
                    validate_mapping_changes(old_mapping, mapping, NUM_NODES, m1, m2);
                    const int verify = calculate_alignment_score((Graph*)gm, (Graph*)gf, mapping);
                    if (verify != score) score = verify;
                }
            }
        }
        if (c == before) { pass++; break; }
    }
    free(old_mapping);
    if (commits) *commits = c;
    if (passes) *passes = pass;
    return score;
}
