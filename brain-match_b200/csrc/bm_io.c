/*
 * bm_io.c -- graph and matching CSV formats of brain-match (host C).
 *
 * Formats follow the reference loaders and writers:
 *   graph CSV    load_graph_from_csv     src/graph-alignment-optimized.c:635-679
 *   matching in  load_benchmark_mapping  src/graph-alignment-optimized.c:428-475
 *   matching out write_mapping           src/graph-alignment-optimized.c:410-425
 *   numeric out  write_matching          src/refine-matching-hillclimb.c:488-503
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include "bm.h"

#define BM_LINE 1024

const char* bm_status_string(bm_status s) {
    switch (s) {
    case BM_OK: return "ok";
    case BM_E_INPUT: return "invalid input";
    case BM_E_CUDA: return "CUDA error";
    case BM_E_OVERFLOW: return "int32 overflow risk";
    case BM_E_TIMEOUT: return "device wait timed out";
    case BM_E_NOMEM: return "out of memory";
    case BM_E_STATE: return "invalid call order";
    case BM_E_IO: return "file I/O error";
    default: return "unknown status";
    }
}

void bm_free(void* p) { free(p); }

/* Parses "from,to,weight"; returns 1 on success (sscanf semantics of the
 * reference: leading integers separated by commas, trailing text ignored). */
static int parse_edge(const char* line, int32_t* a, int32_t* b, int32_t* w) {
    int x, y, z;
    if (sscanf(line, "%d,%d,%d", &x, &y, &z) != 3) return 0;
    *a = x; *b = y; *w = z;
    return 1;
}

bm_status bm_read_graph_csv(const char* path, int64_t* e, int32_t** src, int32_t** dst,
                            int32_t** w, int32_t* max_id) {
    if (!path || !e || !src || !dst || !w || !max_id) return BM_E_INPUT;
    FILE* f = fopen(path, "r");
    if (!f) {
        fprintf(stderr, "[ERROR] bm_read_graph_csv: failed to open file: %s\n", path);
        return BM_E_IO;
    }
    char line[BM_LINE];
    int64_t cap = 1 << 16, cnt = 0;
    int32_t* s = (int32_t*)malloc(sizeof(int32_t) * cap);
    int32_t* d = (int32_t*)malloc(sizeof(int32_t) * cap);
    int32_t* ww = (int32_t*)malloc(sizeof(int32_t) * cap);
    if (!s || !d || !ww) { free(s); free(d); free(ww); fclose(f); return BM_E_NOMEM; }
    int32_t mx = 0;
    /* header line is skipped, as the reference does */
    if (!fgets(line, sizeof line, f)) { fclose(f); free(s); free(d); free(ww); *e = 0; *src = *dst = *w = NULL; *max_id = 0; return BM_OK; }
    while (fgets(line, sizeof line, f)) {
        int32_t a, b, c;
        if (!parse_edge(line, &a, &b, &c)) {
            size_t L = strlen(line);
            if (L && line[L - 1] == '\n') line[L - 1] = 0;
            if (line[0]) fprintf(stderr, "[ERROR] bm_read_graph_csv: malformed line in CSV: %s\n", line);
            continue;
        }
        if (cnt == cap) {
            cap *= 2;
            int32_t* s2 = (int32_t*)realloc(s, sizeof(int32_t) * cap);
            int32_t* d2 = (int32_t*)realloc(d, sizeof(int32_t) * cap);
            int32_t* w2 = (int32_t*)realloc(ww, sizeof(int32_t) * cap);
            if (!s2 || !d2 || !w2) {
                free(s2 ? s2 : s); free(d2 ? d2 : d); free(w2 ? w2 : ww); fclose(f);
                return BM_E_NOMEM;
            }
            s = s2; d = d2; ww = w2;
        }
        s[cnt] = a; d[cnt] = b; ww[cnt] = c; cnt++;
        if (a > mx) mx = a;
        if (b > mx) mx = b;
    }
    fclose(f);
    *e = cnt; *src = s; *dst = d; *w = ww; *max_id = mx;
    return BM_OK;
}

/* One matching line: "<id>,<id>" or "m<id>,f<id>" (prefixes optional on either
 * side), as load_benchmark_mapping accepts (src/graph-alignment-optimized.c:456-467). */
static int parse_match(const char* line, int32_t* m, int32_t* fv) {
    int x, y;
    if (sscanf(line, "%d,%d", &x, &y) == 2) { *m = x; *fv = y; return 1; }
    char ms[20], fs[20];
    if (sscanf(line, "%19[^,],%19s", ms, fs) == 2) {
        *m = atoi(ms + (ms[0] == 'm' ? 1 : 0));
        *fv = atoi(fs + (fs[0] == 'f' ? 1 : 0));
        return 1;
    }
    return 0;
}

bm_status bm_read_mapping_csv(const char* path, int32_t n, int32_t* map, int32_t* count) {
    if (!path || !map || n <= 0) return BM_E_INPUT;
    FILE* f = fopen(path, "r");
    if (!f) {
        fprintf(stderr, "[ERROR] bm_read_mapping_csv: failed to open file: %s\n", path);
        return BM_E_IO;
    }
    memset(map, 0, sizeof(int32_t) * ((size_t)n + 1));
    char line[BM_LINE];
    int32_t cnt = 0;
    bm_status st = BM_OK;
    if (fgets(line, sizeof line, f)) {
        while (fgets(line, sizeof line, f)) {
            int32_t m, fv;
            if (!parse_match(line, &m, &fv)) continue;
            if (m < 1 || m > n || fv < 0 || fv > n) {
                fprintf(stderr, "[ERROR] bm_read_mapping_csv: id out of range 1..%d: %d,%d\n", n, m, fv);
                st = BM_E_INPUT;
                break;
            }
            map[m] = fv;
            cnt++;
        }
    }
    fclose(f);
    if (count) *count = cnt;
    return st;
}

bm_status bm_write_mapping_csv(const char* path, int32_t n, const int32_t* map) {
    if (!path || !map || n < 0) return BM_E_INPUT;
    FILE* f = fopen(path, "w");
    if (!f) {
        fprintf(stderr, "[ERROR] bm_write_mapping_csv: error creating file: %s\n", path);
        return BM_E_IO;
    }
    fprintf(f, "Male Node ID,Female Node ID\n");
    for (int32_t i = 1; i <= n; i++)
        if (map[i] != 0) fprintf(f, "m%d,f%d\n", i, map[i]);
    int bad = ferror(f);
    if (fclose(f) != 0 || bad) return BM_E_IO;
    return BM_OK;
}

bm_status bm_write_mapping_csv_numeric(const char* path, int32_t n, const int32_t* map) {
    if (!path || !map || n < 0) return BM_E_INPUT;
    FILE* f = fopen(path, "w");
    if (!f) return BM_E_IO;
    fprintf(f, "Male ID,Female ID\n");
    for (int32_t i = 1; i <= n; i++)
        if (map[i] != 0) fprintf(f, "%d,%d\n", i, map[i]);
    int bad = ferror(f);
    if (fclose(f) != 0 || bad) return BM_E_IO;
    return BM_OK;
}
