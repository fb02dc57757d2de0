/*
 * ref_harness_par.c -- test infrastructure, not part of the engine.
 *
 * Compiles the reference's own src/graph-alignment-optimized-parallel.c in
 * place (its main() renamed) and drives the body of its OpenMP loop
 * (:544-582) for a list of rows m1: partners m2 in parallel under
 * `#pragma omp parallel for schedule(dynamic)`, each improving delta
 * committed inside `omp critical` with the reference's validation and full
 * rescore.  Deltas read a mapping other threads are changing, so results are
 * not deterministic; bench.py times it only as the reference's racy upper
 * bound.  Built into oracle/_ref/ by oracle/Makefile.
 */
#define main brain_match_reference_main
#include REF_SRC
#undef main
#include <omp.h>

void* refpar_graph_new(void) { return new_graph(); }
void refpar_graph_add_many(void* g, long long m, const int* s, const int* d, const int* w) {
    for (long long i = 0; i < m; i++) add_edge((Graph*)g, s[i], d[i], w[i]);
}
void refpar_graph_free(void* g) { free_graph((Graph*)g); }
int refpar_num_nodes(void) { return NUM_NODES; }

/* Returns the deltas evaluated; *commits the swaps made, *threads the
 * OpenMP thread count. */
long long refpar_rows(void* gm, void* gf, int* mapping, const int* rows, int nrows, int n,
                      long long* commits, int* threads) {
    int* old_mapping = (int*)malloc(sizeof(int) * (NUM_NODES + 1));
    int current_score = calculate_alignment_score((Graph*)gm, (Graph*)gf, mapping);
    long long cnt = 0, improvements = 0;
    for (int r = 0; r < nrows; r++) {
        const int node_m1 = rows[r];
        #pragma omp parallel for reduction(+:improvements, cnt) schedule(dynamic)
        for (int node_m2 = 1; node_m2 <= n; node_m2++) {
            if (node_m1 == node_m2) continue;
            int node_f1 = mapping[node_m1];
            int node_f2 = mapping[node_m2];
            int delta = calculate_swap_delta((Graph*)gm, (Graph*)gf, mapping, node_m1, node_m2);
            cnt++;
            if (delta > 0) {
                #pragma omp critical
                {
                    memcpy(old_mapping, mapping, sizeof(int) * (NUM_NODES + 1));
                    mapping[node_m1] = node_f2;
                    mapping[node_m2] = node_f1;
                    current_score += delta;
                    improvements++;
                    validate_mapping_changes(old_mapping, mapping, NUM_NODES, node_m1, node_m2);
                    int verify_score = calculate_alignment_score((Graph*)gm, (Graph*)gf, mapping);
                    if (verify_score != current_score) current_score = verify_score;
                }
            }
        }
    }
    int nt = 1;
    #pragma omp parallel
    {
        #pragma omp single
        nt = omp_get_num_threads();
    }
    free(old_mapping);
    if (commits) *commits = improvements;
    if (threads) *threads = nt;
    return cnt;
}
