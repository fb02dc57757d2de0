/*
 * create-score-lookup -- drop-in for src/best-swap/create-score-lookup.c
 * (main :451-503): writes the n x n table of swap deltas of a matching, row i
 * holding the deltas of vertex i+1 with every vertex (0 on the diagonal),
 * comma-separated, entries stored as 16-bit values like the reference's
 * short table (:289-296, save_lookup :303-318).  The table is computed on the
 * GPU from the exact profit matrix (bm_lookup_rows), streamed in row blocks.
 */
#include "cli_common.h"

int write_lookup(bm_ctx* ctx, int n, const char* path) {
    FILE* f = fopen(path, "w");
    if (!f) { LOG_ERROR("Error creating file: %s", path); return 1; }
    const int rows = 256;
    int32_t* buf = (int32_t*)malloc(sizeof(int32_t) * (size_t)rows * (size_t)n);
    if (!buf) { fclose(f); return 1; }
    for (int a0 = 1; a0 <= n; a0 += rows) {
        const int r = a0 + rows - 1 <= n ? rows : n - a0 + 1;
        if (bm_lookup_rows(ctx, a0, r, buf) != BM_OK) {
            LOG_ERROR("lookup: %s", bm_last_error(ctx));
            free(buf); fclose(f); return 1;
        }
        for (int i = 0; i < r; i++) {
            const int32_t* row = buf + (size_t)i * n;
            for (int j = 0; j < n; j++) fprintf(f, j + 1 < n ? "%d," : "%d\n", (int)(short)row[j]);
        }
    }
    free(buf);
    fclose(f);
    return 0;
}

#ifndef BM_LOOKUP_NO_MAIN
int main(int argc, char** argv) {
    if (argc < 5) {
        LOG_ERROR("Usage: %s <male graph> <female graph> <in mapping> <out lookup>", argv[0]);
        return 1;
    }
    cli_job j;
    if (cli_load(&j, argv[1], argv[2], argv[3])) { cli_free(&j); return 1; }
    LOG_INFO("Initial alignment score: %lld", cli_score(&j));
    const double t0 = now_s();
    int rc = write_lookup(j.ctx, j.n, argv[4]);
    if (!rc) LOG_INFO("Lookup of %d x %d deltas written to %s in %.1f s", j.n, j.n, argv[4], now_s() - t0);
    cli_free(&j);
    return rc;
}
#endif
