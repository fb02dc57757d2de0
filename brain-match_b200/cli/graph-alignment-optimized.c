/*
 * graph-alignment-optimized -- drop-in for the reference tool of the same
 * name (src/graph-alignment-optimized.c:682-738): same argv, same matching
 * formats, same first-improvement order (for m1, for m2 != m1, commit every
 * improving swap immediately, :515-577).  The ordering files must exist, as
 * the reference reads them (:216-239), but do not steer the search (the
 * reference's use of them is commented out, :549-551).  Unlike the reference,
 * which loops forever, the search stops after a full pass without a commit
 * or after BM_MAX_PASSES passes.  Row evaluation runs on the GPU.
 */
#include "cli_common.h"

int main(int argc, char** argv) {
    if (argc < 7) {
        LOG_ERROR("Usage: %s <male graph> <female graph> <male ordering> <female ordering> <in mapping> <out mapping>", argv[0]);
        return 1;
    }
    LOG_INFO("Graph Alignment Tool (B200 engine)");
    for (int i = 3; i <= 4; i++) {
        FILE* f = fopen(argv[i], "r");
        if (!f) { LOG_ERROR("Error opening file: %s", argv[i]); return 1; }
        fclose(f);
    }
    cli_job j;
    if (cli_load(&j, argv[1], argv[2], argv[5])) { cli_free(&j); return 1; }
    long long s0 = cli_score(&j);
    LOG_INFO("Initial alignment score: %lld", s0);
    double t0 = now_s();
    int64_t commits = 0;
    int32_t passes = 0;
    bm_status st = bm_first_improvement(j.ctx, (int)env_long("BM_MAX_PASSES", 1000000), &commits, &passes);
    if (st != BM_OK) { LOG_ERROR("search: %s", bm_last_error(j.ctx)); cli_free(&j); return 1; }
    long long s1 = cli_score(&j);
    if (cli_save(&j, argv[6], 0)) { cli_free(&j); return 1; }
    LOG_INFO("Process completed:");
    LOG_INFO("  - Initial score: %lld", s0);
    LOG_INFO("  - Final score: %lld", s1);
    LOG_INFO("  - Improvements: %lld in %d passes", (long long)commits, passes);
    LOG_INFO("  - Total time: %.1f minutes", (now_s() - t0) / 60);
    cli_free(&j);
    return 0;
}
