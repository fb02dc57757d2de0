/*
 * greedy-feature-match -- drop-in for src/greedy-feature-match.c (main
 * :715-809): an initial matching of G1 onto G2 by vertex features and edge
 * overlap, written as "Node G1,Node G2" lines (write_matching, :690-712).
 * The features and the sequential matching run on the GPU
 * (bm_greedy_match).  Vertices are the ids 1..n, n the largest id in either
 * graph.
 */
#include "cli_common.h"

int main(int argc, char** argv) {
    if (argc != 4) {
        fprintf(stderr, "Usage: %s <g1.csv> <g2.csv> <output_matching.csv>\n", argv[0]);
        return EXIT_FAILURE;
    }
    printf("Starting graph matching process...\n");
    int64_t e1 = 0, e2 = 0;
    int32_t *s1 = NULL, *d1 = NULL, *w1 = NULL, *s2 = NULL, *d2 = NULL, *w2 = NULL;
    int32_t mx1 = 0, mx2 = 0;
    int rc = EXIT_FAILURE;
    int32_t* map = NULL;
    if (bm_read_graph_csv(argv[1], &e1, &s1, &d1, &w1, &mx1) != BM_OK) {
        fprintf(stderr, "Failed to load first graph from %s\n", argv[1]);
        goto done;
    }
    if (bm_read_graph_csv(argv[2], &e2, &s2, &d2, &w2, &mx2) != BM_OK) {
        fprintf(stderr, "Failed to load second graph from %s\n", argv[2]);
        goto done;
    }
    {
        const int n = mx1 > mx2 ? mx1 : mx2;
        printf("Loaded %d nodes, %lld + %lld edges\n", n, (long long)e1, (long long)e2);
        map = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
        bm_greedy_stats st;
        const double t0 = now_s();
        if (!map || bm_greedy_match(n, e1, s1, d1, w1, e2, s2, d2, w2, map, &st) != BM_OK) {
            fprintf(stderr, "Error during vertex matching: %s\n", bm_last_error(NULL));
            goto done;
        }
        printf("Matching completed: %d vertices (features %.1f ms, matching %.1f ms on the GPU, %.2f s total)\n", n,
               st.ms_features, st.ms_match, now_s() - t0);
        FILE* f = fopen(argv[3], "w");
        if (!f) {
            fprintf(stderr, "Error writing matching results to %s\n", argv[3]);
            goto done;
        }
        fprintf(f, "Node G1,Node G2\n");
        for (int v = 1; v <= n; v++) fprintf(f, "%d,%d\n", v, map[v]);
        fclose(f);
        printf("\nMatching completed successfully. Results written to %s\n", argv[3]);
        rc = EXIT_SUCCESS;
    }
done:
    bm_free(s1); bm_free(d1); bm_free(w1);
    bm_free(s2); bm_free(d2); bm_free(w2);
    free(map);
    return rc;
}
