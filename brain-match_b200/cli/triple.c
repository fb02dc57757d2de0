/*
 * triple -- drop-in for the reference GPU tool src/triple.cu (main
 * :1308-1385): same argv, output "<out minus .csv>-rank0.csv".  The search
 * alternates full pairwise sweeps with 3-cycle rounds (both rotations of
 * 2-hop triples, src/triple.cu:85-92 permutations 3 and 4) until neither
 * improves or BM_TRIPLE_ROUNDS rounds ran.  BM_PARTNERS sets the 2-hop samples
 * per vertex (256), BM_SEED the sampler seed.
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
    long long s0 = cli_score(&j);
    LOG_INFO("Initial alignment score: %lld", s0);
    double t0 = now_s();
    long rounds = env_long("BM_TRIPLE_ROUNDS", 1000000);
    bm_triple_opts o;
    memset(&o, 0, sizeof o);
    o.partners = (int)env_long("BM_PARTNERS", 256);
    o.max_verify = -1;
    o.incremental = (int)env_long("BM_INCREMENTAL", 1);
    unsigned long long seed = (unsigned long long)env_long("BM_SEED", 20261205);
    for (long r = 0; r < rounds; r++) {
        long long c = cli_sweeps(&j, 1000000, 0);
        if (c < 0) { cli_free(&j); return 1; }
        o.seed = seed + (unsigned long long)r;
        bm_triple_stats ts;
        if (bm_triple_round(j.ctx, &o, &ts) != BM_OK) { LOG_ERROR("%s", bm_last_error(j.ctx)); cli_free(&j); return 1; }
        LOG_INFO("round %ld: %lld swaps, %d 3-cycles, score %lld", r + 1, c, ts.committed, (long long)ts.score_after);
        if (c == 0 && ts.committed == 0) break;
    }
    long long s1 = cli_score(&j);
    if (cli_save(&j, out, 0)) { cli_free(&j); return 1; }
    LOG_INFO("Process completed:");
    LOG_INFO("  - Initial score: %lld", s0);
    LOG_INFO("  - Final score: %lld", s1);
    LOG_INFO("  - Total time: %.1f minutes", (now_s() - t0) / 60);
    cli_free(&j);
    return 0;
}
