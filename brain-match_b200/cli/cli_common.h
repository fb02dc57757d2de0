/*
 * cli_common.h -- shared plumbing of the drop-in command-line tools.
 *
 * Each tool keeps the reference tool's argv and file formats; the search
 * itself runs on the GPU through the C ABI (include/bm.h).  Knobs that the
 * reference hard-codes are read from BM_* environment variables (BM_INCREMENTAL=0
 * rebuilds the profit matrix every sweep instead of updating it; the results
 * are the same).
 */
#ifndef BM_CLI_COMMON_H
#define BM_CLI_COMMON_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include "bm.h"

#define LOG_INFO(fmt, ...) printf("[INFO] " fmt "\n", ##__VA_ARGS__)
#define LOG_ERROR(fmt, ...) fprintf(stderr, "[ERROR] %s:%d: " fmt "\n", __func__, __LINE__, ##__VA_ARGS__)

typedef struct {
    int n;
    int64_t e1, e2;
    int32_t *s1, *d1, *w1, *s2, *d2, *w2;
    int32_t* map;       /* n+1 */
    bm_ctx* ctx;
} cli_job;

static inline long env_long(const char* name, long dflt) {
    const char* v = getenv(name);
    return (v && *v) ? strtol(v, NULL, 10) : dflt;
}

static inline double now_s(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* Loads both graphs and the matching, sizes n to cover every id, builds the
 * engine context and sets the matching.  Returns 0 on success. */
static inline int cli_load(cli_job* j, const char* g1, const char* g2, const char* mpath) {
    memset(j, 0, sizeof *j);
    int32_t mx1 = 0, mx2 = 0;
    LOG_INFO("Loading graph from %s", g1);
    if (bm_read_graph_csv(g1, &j->e1, &j->s1, &j->d1, &j->w1, &mx1) != BM_OK) { LOG_ERROR("Failed to load male graph"); return 1; }
    LOG_INFO("Loading graph from %s", g2);
    if (bm_read_graph_csv(g2, &j->e2, &j->s2, &j->d2, &j->w2, &mx2) != BM_OK) { LOG_ERROR("Failed to load female graph"); return 1; }
    int32_t* tmp = (int32_t*)calloc(65536, sizeof(int32_t));
    int32_t cnt = 0;
    if (!tmp || bm_read_mapping_csv(mpath, 65535, tmp, &cnt) != BM_OK) { LOG_ERROR("Failed to load benchmark mapping"); free(tmp); return 1; }
    int n = mx1 > mx2 ? mx1 : mx2;
    for (int i = 1; i <= 65535; i++)
        if (tmp[i]) { if (i > n) n = i; if (tmp[i] > n) n = tmp[i]; }
    if (n < 2) { LOG_ERROR("graphs have fewer than 2 vertices"); free(tmp); return 1; }
    j->n = n;
    j->map = (int32_t*)calloc((size_t)n + 1, sizeof(int32_t));
    memcpy(j->map, tmp, sizeof(int32_t) * ((size_t)n + 1));
    free(tmp);
    LOG_INFO("Loaded %d mappings; %d nodes, %lld + %lld edges", cnt, n, (long long)j->e1, (long long)j->e2);
    bm_status st = bm_create(&j->ctx, n, j->e1, j->s1, j->d1, j->w1, j->e2, j->s2, j->d2, j->w2, 0);
    if (st != BM_OK) { LOG_ERROR("engine: %s: %s", bm_status_string(st), bm_last_error(NULL)); return 1; }
    st = bm_set_mapping(j->ctx, j->map);
    if (st != BM_OK) { LOG_ERROR("mapping: %s: %s", bm_status_string(st), bm_last_error(j->ctx)); return 1; }
    return 0;
}

static inline long long cli_score(cli_job* j) {
    int64_t s = 0;
    if (bm_score(j->ctx, &s) != BM_OK) { LOG_ERROR("score: %s", bm_last_error(j->ctx)); return -1; }
    return (long long)s;
}

static inline int cli_save(cli_job* j, const char* path, int numeric) {
    if (bm_get_mapping(j->ctx, j->map) != BM_OK) { LOG_ERROR("%s", bm_last_error(j->ctx)); return 1; }
    bm_status st = numeric ? bm_write_mapping_csv_numeric(path, j->n, j->map) : bm_write_mapping_csv(path, j->n, j->map);
    if (st != BM_OK) { LOG_ERROR("Error creating file: %s", path); return 1; }
    return 0;
}

static inline void cli_free(cli_job* j) {
    if (j->ctx) bm_destroy(j->ctx);
    bm_free(j->s1); bm_free(j->d1); bm_free(j->w1);
    bm_free(j->s2); bm_free(j->d2); bm_free(j->w2);
    free(j->map);
}

/* "<out minus .csv>-rank0.csv", as quick.cu:1518 and triple.cu:1365 name it */
static inline void rank0_name(char* dst, size_t cap, const char* out) {
    int L = (int)strlen(out);
    snprintf(dst, cap, "%.*s-rank0.csv", L >= 4 ? L - 4 : L, out);
}

/* pairwise sweeps until none improves (or BM_MAX_SWEEPS) */
static inline long long cli_sweeps(cli_job* j, int max_sweeps, int verbose) {
    bm_sweep_opts o;
    memset(&o, 0, sizeof o);
    o.max_candidates = (int)env_long("BM_MAX_CANDIDATES", 0);
    o.max_verify = (int)env_long("BM_MAX_VERIFY", -1);
    o.incremental = (int)env_long("BM_INCREMENTAL", 1);
    long long commits = 0;
    for (int s = 0; s < max_sweeps; s++) {
        bm_sweep_stats st;
        if (bm_sweep(j->ctx, &o, &st) != BM_OK) { LOG_ERROR("sweep: %s", bm_last_error(j->ctx)); return -1; }
        commits += st.committed;
        if (verbose)
            LOG_INFO("sweep %d: score %lld -> %lld, %d swaps, %.2f ms", s + 1, (long long)st.score_before,
                     (long long)st.score_after, st.committed, st.ms_total);
        if (st.committed == 0) break;
    }
    return commits;
}
#endif
