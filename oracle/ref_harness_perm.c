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

/*
 * Both 3-cycle rotations of k triples (a[i], b[i], c[i]) by the reference's
 * local score: out[2i + rot] = calculate_permutation_delta after the rotation
 * minus before it, with rotation 0 giving (a, b, c) the images of (b, c, a)
 * and rotation 1 those of (c, a, b) (permutations 3 and 4 of
 * src/triple.cu:85-92).  OpenMP over triples, each thread on its own copy of
 * the mapping (NUM_NODES + 1 entries).  Returns the thread count.
 */
#include <omp.h>
int refperm_triples_omp(void* gm, void* gf, const int* mapping, long long k, const int* a, const int* b,
                        const int* c, int* out) {
    int nt = 1;
    #pragma omp parallel
    {
        int* m = (int*)malloc(sizeof(int) * (NUM_NODES + 1));
        memcpy(m, mapping, sizeof(int) * (NUM_NODES + 1));
        #pragma omp single
        nt = omp_get_num_threads();
        #pragma omp for schedule(dynamic, 4)
        for (long long i = 0; i < k; i++) {
            int set[3] = {a[i], b[i], c[i]};
            const int fa = m[a[i]], fb = m[b[i]], fc = m[c[i]];
            const int before = calculate_permutation_delta((Graph*)gm, (Graph*)gf, m, set, 3);
            m[a[i]] = fb; m[b[i]] = fc; m[c[i]] = fa;
            out[2 * i] = calculate_permutation_delta((Graph*)gm, (Graph*)gf, m, set, 3) - before;
            m[a[i]] = fc; m[b[i]] = fa; m[c[i]] = fb;
            out[2 * i + 1] = calculate_permutation_delta((Graph*)gm, (Graph*)gf, m, set, 3) - before;
            m[a[i]] = fa; m[b[i]] = fb; m[c[i]] = fc;
        }
        free(m);
    }
    return nt;
}
