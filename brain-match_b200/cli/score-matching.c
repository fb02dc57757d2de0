/*
 * score-matching -- drop-in for src/score-matching.c (main :599-704): prints
 * the graph sizes and then the alignment score of a matching on its own line.
 * The score is computed by the engine on the GPU (calculate_score_sparse,
 * :558-597, is the reference).
 */
#include "cli_common.h"

int main(int argc, char** argv) {
    if (argc != 4) {
        fprintf(stdout, "Usage: %s <g1.csv> <g2.csv> <matching.csv>\n", argv[0]);
        return EXIT_FAILURE;
    }
    cli_job j;
    if (cli_load(&j, argv[1], argv[2], argv[3])) { cli_free(&j); return EXIT_FAILURE; }
    fprintf(stdout, "Processing graphs with:\n");
    fprintf(stdout, "  Graph 1: %d vertices and %lld edges\n", j.n, (long long)j.e1);
    fprintf(stdout, "  Graph 2: %d vertices and %lld edges\n", j.n, (long long)j.e2);
    long long s = cli_score(&j);
    if (s < 0) { fprintf(stdout, "Error calculating score\n"); cli_free(&j); return EXIT_FAILURE; }
    printf("%lld\n", s);
    cli_free(&j);
    return EXIT_SUCCESS;
}
