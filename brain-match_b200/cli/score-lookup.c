/*
 * score-lookup -- drop-in for src/best-swap/score-lookup.c (main :690-767):
 * best-swap descent on the swap-delta table, then the matching and the table
 * are written (save_mapping :420-434 lists every vertex as m<i>,f<j>;
 * save_lookup as create-score-lookup writes it).  The table is the engine's
 * exact profit matrix, rebuilt on the GPU from the graphs and kept exact
 * across every swap (bm_lookup_descent), so the input table is only checked
 * for existence: the reference reads it and then keeps it partly stale.
 * BM_ITERATIONS (default 200000, the reference's ITERATIONS) bounds the
 * swaps; the descent stops earlier when no swap improves.  The reference's
 * zero-delta and temperature swaps (:548-595) are not made.
 */
#define BM_LOOKUP_NO_MAIN
#include "create-score-lookup.c"

int main(int argc, char** argv) {
    if (argc < 7) {
        LOG_ERROR("Usage: %s <male graph> <female graph> <in mapping> <in lookup> <out mapping> <out lookup>",
                  argv[0]);
        return 1;
    }
    FILE* lk = fopen(argv[4], "r");
    if (!lk) { LOG_ERROR("Failed to open file: %s", argv[4]); LOG_ERROR("Failed to load lookup file"); return 1; }
    fclose(lk);
    cli_job j;
    if (cli_load(&j, argv[1], argv[2], argv[3])) { cli_free(&j); return 1; }
    const long long s0 = cli_score(&j);
    LOG_INFO("Initial alignment score: %lld", s0);
    const long iters = env_long("BM_ITERATIONS", 200000);
    bm_lookup_stats st;
    const double t0 = now_s();
    if (bm_lookup_descent(j.ctx, (int32_t)iters, &st) != BM_OK) {
        LOG_ERROR("descent: %s", bm_last_error(j.ctx));
        cli_free(&j);
        return 1;
    }
    LOG_INFO("%d swaps%s, score %lld -> %lld (%.1f ms on the GPU, %.2f s)", st.swaps,
             st.converged ? " (no improving swap left)" : "", (long long)st.score_before, (long long)st.score_after,
             st.ms_total, now_s() - t0);
    if (bm_get_mapping(j.ctx, j.map) != BM_OK) { LOG_ERROR("%s", bm_last_error(j.ctx)); cli_free(&j); return 1; }
    FILE* f = fopen(argv[5], "w");
    if (!f) { LOG_ERROR("Error creating file: %s", argv[5]); cli_free(&j); return 1; }
    fprintf(f, "Male Node ID,Female Node ID\n");
    for (int i = 1; i <= j.n; i++) fprintf(f, "m%d,f%d\n", i, j.map[i]);
    fclose(f);
    int rc = write_lookup(j.ctx, j.n, argv[6]);
    LOG_INFO("Process completed: initial score %lld, final score %lld", s0, cli_score(&j));
    cli_free(&j);
    return rc;
}
