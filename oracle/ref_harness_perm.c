/*
 * ref_harness_perm.c -- test infrastructure, not part of the engine.
 *
 * Compiles the reference's own src/permutation.c in place (its main()
 * renamed) and exposes calculate_permutation_delta
 * (src/permutation.c:623-696): the local score of the unique G1 edges incident
 * to a vertex set under a mapping.  A 3-cycle's exact delta is that local
 * score after the move minus before it.  Built into oracle/_ref/ by
 * oracle/Makefile.
 */
#define main brain_match_reference_main
#include REF_SRC
#undef main

void* refperm_graph_new(void) { return new_graph(); }
void refperm_graph_add_many(void* g, long long m, const int* s, const int* d, const int* w) {
    for (long long i = 0; i < m; i++) add_edge((Graph*)g, s[i], d[i], w[i]);
}
void refperm_graph_free(void* g) { free_graph((Graph*)g); }
int refperm_local_score(void* gm, void* gf, int* mapping, int* set, int k) {
    return calculate_permutation_delta((Graph*)gm, (Graph*)gf, mapping, set, k);
}
int refperm_score(void* gm, void* gf, int* mapping) {
    return calculate_alignment_score((Graph*)gm, (Graph*)gf, mapping);
}
