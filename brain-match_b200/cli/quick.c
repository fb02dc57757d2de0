/*
 * quick -- drop-in for the reference GPU tool src/quick.cu (main :1435-1538):
 * same argv, reads "m<id>,f<id>" or numeric matchings, writes the best
 * matching to "<out minus .csv>-rank0.csv" in write_mapping format.  The
 * search is the engine's full pairwise sweep with best-per-row set commits
 * until no improving swap remains; BM_PERTURB > 0 adds that many seeded
 * random-swap restarts from the best matching (the reference perturbs with
 * time-seeded rand(), src/quick.cu:1151,842).
 */
#include "cli_common.h"

int main(int argc, char** argv) {
    if (argc < 5) {
        LOG_ERROR("Usage: %s <male graph> <female graph> <in mapping> <out mapping>", argv[0]);
        return 1;
    }
    char out[4096];
    rank0_name(out, sizeof out, argv[4]);
    LOG_INFO("output file name is %s", out);
    cli_job j;
    if (cli_load(&j, argv[1], argv[2], argv[3])) { cli_free(&j); return 1; }
    long long s0 = cli_score(&j), best = s0;
    LOG_INFO("Initial alignment score: %lld", s0);
    double t0 = now_s();
    int max_sweeps = (int)env_long("BM_MAX_SWEEPS", 1000000);
    if (cli_sweeps(&j, max_sweeps, 1) < 0) { cli_free(&j); return 1; }
    best = cli_score(&j);
    int32_t* bestmap = (int32_t*)malloc(sizeof(int32_t) * (j.n + 1));
    bm_get_mapping(j.ctx, bestmap);
    long rounds = env_long("BM_PERTURB", 0);
    unsigned long long rs = (unsigned long long)env_long("BM_SEED", 1);
    for (long r = 0; r < rounds; r++) {
        memcpy(j.map, bestmap, sizeof(int32_t) * (j.n + 1));
        int k = 3 + (int)(r % 2);
        for (int i = 0; i < k; i++) {   /* seeded random swaps (LCG) */
            rs = rs * 6364136223846793005ULL + 1442695040888963407ULL;
            int a = 1 + (int)((rs >> 33) % (unsigned)j.n);
            rs = rs * 6364136223846793005ULL + 1442695040888963407ULL;
            int b = 1 + (int)((rs >> 33) % (unsigned)j.n);
            int t = j.map[a]; j.map[a] = j.map[b]; j.map[b] = t;
        }
        if (bm_set_mapping(j.ctx, j.map) != BM_OK) break;
        if (cli_sweeps(&j, max_sweeps, 0) < 0) break;
        long long s = cli_score(&j);
        if (s > best) {
            best = s;
            bm_get_mapping(j.ctx, bestmap);
            LOG_INFO("Process 0 found new best score: %lld in iter %ld", best, r);
        }
    }
    bm_set_mapping(j.ctx, bestmap);
    if (cli_save(&j, out, 0)) { free(bestmap); cli_free(&j); return 1; }
    LOG_INFO("Process completed:");
    LOG_INFO("  - Initial score: %lld", s0);
    LOG_INFO("  - Final score: %lld", best);
    LOG_INFO("  - Total time: %.1f minutes", (now_s() - t0) / 60);
    free(bestmap);
    cli_free(&j);
    return 0;
}
