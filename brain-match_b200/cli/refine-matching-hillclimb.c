/*
 * refine-matching-hillclimb -- drop-in for src/refine-matching-hillclimb.c
 * (main :509-574): same argv (exactly four files), numeric "id,id" matching in
 * and out with the "Male ID,Female ID" header (:454-503), and the same
 * messages.  The reference's 8-thread simulated annealing (:299-402) is
 * replaced by the engine's exact pairwise sweeps on the GPU until no
 * improving swap remains.
 */
#include "cli_common.h"

int main(int argc, char** argv) {
    if (argc != 5) {
        fprintf(stderr, "Usage: %s <g1.csv> <g2.csv> <initial_matching.csv> <output_matching.csv>\n", argv[0]);
        return EXIT_FAILURE;
    }
    cli_job j;
    printf("Loading graph 1...\nLoading graph 2...\nLoading initial matching...\n");
    if (cli_load(&j, argv[1], argv[2], argv[3])) { cli_free(&j); return EXIT_FAILURE; }
    long long s0 = cli_score(&j);
    printf("Initial matching score: %lld\n", s0);
    printf("Optimizing matching on the GPU...\n");
    if (cli_sweeps(&j, (int)env_long("BM_MAX_SWEEPS", 1000000), 0) < 0) { cli_free(&j); return EXIT_FAILURE; }
    long long s1 = cli_score(&j);
    printf("Final matching score: %lld\n", s1);
    if (s0 > 0) printf("Improvement: %.2f%%\n", 100.0 * (double)(s1 - s0) / (double)s0);
    printf("Writing results to %s...\n", argv[4]);
    if (cli_save(&j, argv[4], 1)) { cli_free(&j); return EXIT_FAILURE; }
    printf("Cleaning up...\n");
    cli_free(&j);
    printf("Done.\n");
    return EXIT_SUCCESS;
}
