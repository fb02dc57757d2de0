/*
 * bm_oracle.c -- CPU oracle for the swap-delta engine.  TEST INFRASTRUCTURE:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
 * it, and only to check or time against; the engine never calls it.
 *
 * A plain C restatement of the reference arithmetic plus the engine's
 * deterministic move-selection rules, 1-based like the reference:
 *   orc_score          calculate_alignment_score  src/graph-alignment-optimized.c:292-307
 *   orc_swap_delta     calculate_swap_delta       src/graph-alignment-optimized.c:321-408
 *   orc_first_improvement  the m1/m2 loop of optimize_mapping
 *                          src/graph-alignment-optimized.c:515-577, stopped
 *                          after a pass without a commit
 *   orc_triple_local   calculate_permutation_delta src/permutation.c:623-696
 *                      (local score of the edges incident to a vertex set)
 *   orc_quad_delta     4-set permutations: calculate_permutation_delta
 *                      differences (src/permutation.c:623-744) for k = 4
 *   orc_best_swap_descent  the extract_max / swap / update loop of the
 *                      best-swap tool (src/best-swap/score-lookup.c:597-640)
 *                      on an exact delta table, largest delta first
 *   orc_greedy_features / orc_greedy_distance / orc_greedy_match  the
 *                      greedy feature matcher (src/greedy-feature-match.c:
 *                      527-712): compute_vertex_features,
 *                      compute_feature_distance and match_vertices with
 *                      compute_edge_alignment's evident intent
 *   orc_sweep / orc_triple_round / orc_quad_round  the best-per-row set commit that the engine
 *                      runs (candidates sorted by delta desc then ids, each
 *                      re-verified on the updated mapping).
 *   orc_sweep_given / orc_triple_round_given  the same selection and commit
 *                      from deltas the caller supplies (for sizes where the
 *                      CPU cannot evaluate every pair or triple in a test;
 *                      the caller checks those deltas by sampling)
 *   orc_pair_deltas / orc_triple_deltas  many deltas at once, OpenMP
 * Graph semantics match the reference loaders: every G1 edge entry counts,
 * the last G2 weight for a (src,dst) pair wins, zero weights contribute 0.
 * Deviation, on purpose: a G1 self-loop (a,a,s) is scored exactly
 * (min(s, w2(map a, map a)) before, min(s, w2(map b, map b)) after a swap),
 * where the reference delta counts it through both of a's lists; on inputs
 * without G1 self-loops or repeated edges between the two swapped vertices
 * the delta is the reference's.  The tests pin this file against the
 * compiled reference (oracle/_ref/librefgao.so, librefperm.so).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define MIN(a, b) ((a) < (b) ? (a) : (b))

typedef struct {
    int n;
    int *o_off, *o_id, *o_w;   /* G1 out-lists (self-loops excluded), rows sorted by id (stable) */
    int *i_off, *i_id, *i_w;   /* G1 in-lists */
    int *s_off, *s_w;          /* G1 self-loops */
    int *g_off, *g_id, *g_w;   /* G2 out-rows, unique ids sorted, last weight wins */
    int* dense;                /* (n+1)^2 copy of G2 for small n (NULL otherwise) */
} orc;

static int* csr_offsets(int n, long long m, const int* key) {
    int* off = (int*)calloc((size_t)n + 2, sizeof(int));
    for (long long i = 0; i < m; i++) off[key[i] + 1]++;
    for (int v = 0; v <= n; v++) off[v + 1] += off[v];
    return off;
}

/* stable counting sort of entries by key, then stable insertion by id within rows */
static void build_rows(int n, long long m, const int* key, const int* id, const int* w,
                       int** off_out, int** id_out, int** w_out) {
    int* off = csr_offsets(n, m, key);
    int* pos = (int*)malloc(sizeof(int) * ((size_t)n + 2));
    memcpy(pos, off, sizeof(int) * ((size_t)n + 2));
    int* I = (int*)malloc(sizeof(int) * (size_t)(m ? m : 1));
    int* W = (int*)malloc(sizeof(int) * (size_t)(m ? m : 1));
    for (long long i = 0; i < m; i++) { int q = pos[key[i]]++; I[q] = id[i]; W[q] = w[i]; }
    for (int v = 0; v <= n; v++) {
        for (int i = off[v] + 1; i < off[v + 1]; i++) {
            int x = I[i], y = W[i], j = i - 1;
            while (j >= off[v] && I[j] > x) { I[j + 1] = I[j]; W[j + 1] = W[j]; j--; }
            I[j + 1] = x; W[j + 1] = y;
        }
    }
    free(pos);
    *off_out = off; *id_out = I; *w_out = W;
}

void* orc_create(int n, long long e1, const int* s1, const int* d1, const int* w1,
                 long long e2, const int* s2, const int* d2, const int* w2) {
    orc* g = (orc*)calloc(1, sizeof(orc));
    g->n = n;
    /* G1: drop zero weights, self-loops apart */
    int *os = malloc(sizeof(int) * (e1 + 1)), *od = malloc(sizeof(int) * (e1 + 1)), *ow = malloc(sizeof(int) * (e1 + 1));
    int *ss = malloc(sizeof(int) * (e1 + 1)), *sw = malloc(sizeof(int) * (e1 + 1)), *zz = calloc(e1 + 1, sizeof(int));
    long long m = 0, ms = 0;
    for (long long i = 0; i < e1; i++) {
        if (w1[i] == 0) continue;
        if (s1[i] == d1[i]) { ss[ms] = s1[i]; sw[ms] = w1[i]; ms++; continue; }
        os[m] = s1[i]; od[m] = d1[i]; ow[m] = w1[i]; m++;
    }
    build_rows(n, m, os, od, ow, &g->o_off, &g->o_id, &g->o_w);
    build_rows(n, m, od, os, ow, &g->i_off, &g->i_id, &g->i_w);
    int* dummy;
    build_rows(n, ms, ss, zz, sw, &g->s_off, &dummy, &g->s_w);
    free(dummy);
    free(os); free(od); free(ow); free(ss); free(sw); free(zz);
    /* G2: last weight per (src,dst) wins, as the reference's dense matrix does */
    int* gi; int* gw; int* goff;
    build_rows(n, e2, s2, d2, w2, &goff, &gi, &gw);
    int* off2 = (int*)calloc((size_t)n + 2, sizeof(int));
    long long q = 0;
    for (int v = 0; v <= n; v++) {
        off2[v] = (int)q;
        for (int i = goff[v]; i < goff[v + 1]; i++) {
            if (i + 1 < goff[v + 1] && gi[i + 1] == gi[i]) continue;  /* a later copy wins */
            /* stable sort keeps input order within equal ids, so the last copy is last */
            if (gw[i] == 0) continue;
            gi[q] = gi[i]; gw[q] = gw[i]; q++;
        }
    }
    off2[n + 1] = (int)q;
    free(goff);
    g->g_off = off2; g->g_id = gi; g->g_w = gw;
    g->dense = NULL;
    if (n <= 8192) {
        g->dense = (int*)calloc((size_t)(n + 1) * (n + 1), sizeof(int));
        for (int v = 1; v <= n; v++)
            for (int i = off2[v]; i < off2[v + 1]; i++) g->dense[(size_t)v * (n + 1) + gi[i]] = gw[i];
    }
    return g;
}

void orc_free(void* p) {
    orc* g = (orc*)p;
    if (!g) return;
    free(g->o_off); free(g->o_id); free(g->o_w);
    free(g->i_off); free(g->i_id); free(g->i_w);
    free(g->s_off); free(g->s_w);
    free(g->g_off); free(g->g_id); free(g->g_w);
    free(g->dense);
    free(g);
}

/* dense-lookup equivalent: w2(f,g), 0 when either id is 0 (unmatched) */
static int W2(const orc* g, int f, int t) {
    if (f <= 0 || t <= 0) return 0;
    if (g->dense) return g->dense[(size_t)f * (g->n + 1) + t];
    int lo = g->g_off[f], hi = g->g_off[f + 1];
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (g->g_id[mid] < t) lo = mid + 1; else hi = mid;
    }
    return (lo < g->g_off[f + 1] && g->g_id[lo] == t) ? g->g_w[lo] : 0;
}

long long orc_score(void* p, const int* map) {
    const orc* g = (const orc*)p;
    long long s = 0;
    for (int a = 1; a <= g->n; a++) {
        for (int i = g->o_off[a]; i < g->o_off[a + 1]; i++)
            s += MIN(g->o_w[i], W2(g, map[a], map[g->o_id[i]]));
        for (int i = g->s_off[a]; i < g->s_off[a + 1]; i++)
            s += MIN(g->s_w[i], W2(g, map[a], map[a]));
    }
    return s;
}

/* calculate_swap_delta restated (src/graph-alignment-optimized.c:321-408) */
int orc_swap_delta(void* p, const int* map, int m1, int m2) {
    const orc* g = (const orc*)p;
    const int f1 = map[m1], f2 = map[m2];
    int delta = 0;
    for (int i = g->o_off[m1]; i < g->o_off[m1 + 1]; i++) {          /* out of m1 */
        int v = g->o_id[i], w = g->o_w[i];
        if (v == m2) continue;
        delta += MIN(w, W2(g, f2, map[v])) - MIN(w, W2(g, f1, map[v]));
    }
    for (int i = g->i_off[m1]; i < g->i_off[m1 + 1]; i++) {          /* into m1 */
        int u = g->i_id[i], w = g->i_w[i];
        if (u == m2) continue;
        delta += MIN(w, W2(g, map[u], f2)) - MIN(w, W2(g, map[u], f1));
    }
    for (int i = g->o_off[m2]; i < g->o_off[m2 + 1]; i++) {          /* out of m2 */
        int v = g->o_id[i], w = g->o_w[i];
        if (v == m1) continue;
        delta += MIN(w, W2(g, f1, map[v])) - MIN(w, W2(g, f2, map[v]));
    }
    for (int i = g->i_off[m2]; i < g->i_off[m2 + 1]; i++) {          /* into m2 */
        int u = g->i_id[i], w = g->i_w[i];
        if (u == m1) continue;
        delta += MIN(w, W2(g, map[u], f1)) - MIN(w, W2(g, map[u], f2));
    }
    for (int i = g->o_off[m1]; i < g->o_off[m1 + 1]; i++)            /* m1 -> m2 */
        if (g->o_id[i] == m2)
            delta += MIN(g->o_w[i], W2(g, f2, f1)) - MIN(g->o_w[i], W2(g, f1, f2));
    for (int i = g->o_off[m2]; i < g->o_off[m2 + 1]; i++)            /* m2 -> m1 */
        if (g->o_id[i] == m1)
            delta += MIN(g->o_w[i], W2(g, f1, f2)) - MIN(g->o_w[i], W2(g, f2, f1));
    for (int i = g->s_off[m1]; i < g->s_off[m1 + 1]; i++)            /* self-loops, exact */
        delta += MIN(g->s_w[i], W2(g, f2, f2)) - MIN(g->s_w[i], W2(g, f1, f1));
    for (int i = g->s_off[m2]; i < g->s_off[m2 + 1]; i++)
        delta += MIN(g->s_w[i], W2(g, f1, f1)) - MIN(g->s_w[i], W2(g, f2, f2));
    return delta;
}

/* all n(n-1)/2 deltas in the reference's linear pair order (m1<m2, row-major) */
void orc_all_deltas(void* p, const int* map, int* out) {
    const orc* g = (const orc*)p;
    const int n = g->n;
    #pragma omp parallel for schedule(dynamic, 8)
    for (int a = 1; a <= n; a++) {
        long long base = (long long)(a - 1) * (2LL * n - a) / 2;
        for (int b = a + 1; b <= n; b++) out[base + (b - a - 1)] = orc_swap_delta(p, map, a, b);
    }
}

/* deltas of k given pairs (m1[i], m2[i]) on one matching, OpenMP over pairs */
void orc_pair_deltas(void* p, const int* map, long long k, const int* m1, const int* m2, int* out) {
    #pragma omp parallel for schedule(dynamic, 256)
    for (long long i = 0; i < k; i++) out[i] = orc_swap_delta(p, map, m1[i], m2[i]);
}

static void taint_nbrs(const orc* g, int x, unsigned char* taint) {
    for (int i = g->o_off[x]; i < g->o_off[x + 1]; i++) taint[g->o_id[i]] = 1;
    for (int i = g->i_off[x]; i < g->i_off[x + 1]; i++) taint[g->i_id[i]] = 1;
}

static int cmp_u64(const void* a, const void* b) {
    uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
    return (x > y) - (x < y);
}

/*
 * One pairwise sweep.  stats[0..6] = total delta, candidates, scanned,
 * verified, committed, best delta, deltas evaluated.  moves (optional, 3 ints
 * per commit: m1, m2, delta).
 */
/* The sweep's selection and commit given every pair's delta on the current
 * matching (`all`, the linear pair order of orc_all_deltas).  orc_sweep
 * computes `all` itself; orc_sweep_given takes it from the caller, so a test
 * can run this rule on deltas it has checked row by row against the compiled
 * reference where a full CPU evaluation would take minutes. */
int orc_sweep_given(void* p, int* map, const int* all, int max_candidates, int max_verify,
                    long long* stats, int* moves) {
    const orc* g = (const orc*)p;
    const int n = g->n;
    int* bestd = (int*)malloc(sizeof(int) * (n + 1));
    int* bestb = (int*)malloc(sizeof(int) * (n + 1));
    /* every unordered pair once; row a's best partner: largest delta, then smallest b */
    for (int a = 0; a <= n; a++) { bestd[a] = 0; bestb[a] = 0; }
    for (int a = 1; a <= n; a++) {
        long long base = (long long)(a - 1) * (2LL * n - a) / 2;
        for (int b = a + 1; b <= n; b++) {
            int d = all[base + (b - a - 1)];
            if (bestb[a] == 0 || d > bestd[a]) { bestd[a] = d; bestb[a] = b; }
            if (bestb[b] == 0 || d > bestd[b] || (d == bestd[b] && a < bestb[b])) { bestd[b] = d; bestb[b] = a; }
        }
    }
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
    int nk = 0, best = 0;
    for (int a = 1; a <= n; a++) {
        int d = bestd[a], b = bestb[a];
        if (d <= 0) continue;
        if (d > best) best = d;
        if (bestb[b] == a && b < a) continue;  /* mutual pair: emitted once, by the smaller row */
        int lo = a < b ? a : b, hi = a < b ? b : a;
        keys[nk++] = ((uint64_t)(0x7fffffffu - (unsigned)d) << 32) | ((uint64_t)(lo - 1) << 16) | (uint64_t)(hi - 1);
    }
    qsort(keys, nk, sizeof(uint64_t), cmp_u64);
    unsigned char* used = calloc(n + 1, 1);
    unsigned char* taint = calloc(n + 1, 1);
    long long total = 0;
    int scanned = 0, verified = 0, committed = 0;
    int lim = (max_candidates > 0 && max_candidates < nk) ? max_candidates : nk;
    for (int k = 0; k < lim; k++) {
        int lo = (int)((keys[k] >> 16) & 0xffff) + 1, hi = (int)(keys[k] & 0xffff) + 1;
        int d0 = (int)(0x7fffffffu - (unsigned)(keys[k] >> 32));
        scanned++;
        if (used[lo] || used[hi]) continue;
        int d = d0;
        if (taint[lo] || taint[hi]) {
            if (max_verify >= 0 && verified >= max_verify) continue;
            verified++;
            d = orc_swap_delta(p, map, lo, hi);
        }
        if (d <= 0) continue;
        int t = map[lo]; map[lo] = map[hi]; map[hi] = t;
        used[lo] = used[hi] = 1;
        if (moves) { moves[3 * committed] = lo; moves[3 * committed + 1] = hi; moves[3 * committed + 2] = d; }
        total += d;
        committed++;
        taint_nbrs(g, lo, taint);
        taint_nbrs(g, hi, taint);
    }
    if (stats) {
        stats[0] = total; stats[1] = nk; stats[2] = scanned; stats[3] = verified;
        stats[4] = committed; stats[5] = best; stats[6] = (long long)n * (n - 1) / 2;
    }
    free(bestd); free(bestb); free(keys); free(used); free(taint);
    return committed;
}

int orc_sweep(void* p, int* map, int max_candidates, int max_verify, long long* stats, int* moves) {
    const orc* g = (const orc*)p;
    const int n = g->n;
    long long np = (long long)n * (n - 1) / 2;
    int* all = (int*)malloc(sizeof(int) * (size_t)(np ? np : 1));
    orc_all_deltas(p, map, all);
    int c = orc_sweep_given(p, map, all, max_candidates, max_verify, stats, moves);
    free(all);
    return c;
}

/* The reference's first-improvement order; returns commits, *passes = passes run. */
long long orc_first_improvement(void* p, int* map, int max_passes, int* passes, long long* delta_sum) {
    const orc* g = (const orc*)p;
    long long commits = 0, dsum = 0;
    int pass = 0;
    for (; pass < max_passes; pass++) {
        long long in_pass = 0;
        for (int m1 = 1; m1 <= g->n; m1++)
            for (int m2 = 1; m2 <= g->n; m2++) {
                if (m1 == m2) continue;
                int d = orc_swap_delta(p, map, m1, m2);
                if (d > 0) {
                    int t = map[m1]; map[m1] = map[m2]; map[m2] = t;
                    in_pass++;
                    dsum += d;
                }
            }
        commits += in_pass;
        if (in_pass == 0) { pass++; break; }
    }
    if (passes) *passes = pass;
    if (delta_sum) *delta_sum = dsum;
    return commits;
}

/* ---- 3-cycles ---- */

/* Local score of the G1 edges incident to `set` (each edge entry once), the
 * quantity calculate_permutation_delta returns (src/permutation.c:623-696). */
long long orc_local_score(void* p, const int* map, const int* set, int k) {
    const orc* g = (const orc*)p;
    long long s = 0;
    for (int i = 0; i < k; i++) {
        int x = set[i];
        for (int q = g->o_off[x]; q < g->o_off[x + 1]; q++)
            s += MIN(g->o_w[q], W2(g, map[x], map[g->o_id[q]]));
        for (int q = g->i_off[x]; q < g->i_off[x + 1]; q++) {
            int u = g->i_id[q], in_set = 0;
            for (int j = 0; j < k; j++) if (set[j] == u) in_set = 1;
            if (in_set) continue;  /* counted from u's out-list */
            s += MIN(g->i_w[q], W2(g, map[u], map[x]));
        }
        for (int q = g->s_off[x]; q < g->s_off[x + 1]; q++)
            s += MIN(g->s_w[q], W2(g, map[x], map[x]));
    }
    return s;
}

/* rotation 0: (f1,f2,f3) <- (f2,f3,f1); rotation 1: <- (f3,f1,f2)
 * (permutations 3 and 4 of src/triple.cu:85-92, apply_permutation :903-934) */
static void rotate(int* map, int a, int b, int c, int rot) {
    int fa = map[a], fb = map[b], fc = map[c];
    if (rot == 0) { map[a] = fb; map[b] = fc; map[c] = fa; }
    else          { map[a] = fc; map[b] = fa; map[c] = fb; }
}

int orc_triple_delta(void* p, const int* map, int a, int b, int c, int rot) {
    const orc* g = (const orc*)p;
    int set[3] = {a, b, c};
    int* m2 = (int*)malloc(sizeof(int) * (g->n + 1));
    memcpy(m2, map, sizeof(int) * (g->n + 1));
    long long before = orc_local_score(p, map, set, 3);
    rotate(m2, a, b, c, rot);
    long long after = orc_local_score(p, m2, set, 3);
    free(m2);
    return (int)(after - before);
}

/* both rotations of k given triples, out[2i + rot], OpenMP over triples */
void orc_triple_deltas(void* p, const int* map, long long k, const int* a, const int* b, const int* c,
                       int* out) {
    #pragma omp parallel for schedule(dynamic, 64)
    for (long long i = 0; i < k; i++)
        for (int rot = 0; rot < 2; rot++) out[2 * i + rot] = orc_triple_delta(p, map, a[i], b[i], c[i], rot);
}

static uint64_t mix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ULL;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static int ndeg(const orc* g, int x) {
    return (g->o_off[x + 1] - g->o_off[x]) + (g->i_off[x + 1] - g->i_off[x]);
}
static int nbr_at(const orc* g, int x, int k) {
    int lo = g->o_off[x + 1] - g->o_off[x];
    return k < lo ? g->o_id[g->o_off[x] + k] : g->i_id[g->i_off[x] + (k - lo)];
}
/* 2-hop sample of slot j of vertex a (1-based ids; the hash uses a-1). */
int orc_sample_triple(void* p, uint64_t seed, int a, int j, int* b, int* c) {
    const orc* g = (const orc*)p;
    int da = ndeg(g, a);
    if (da == 0) return 0;
    uint64_t h1 = mix64(seed ^ (((uint64_t)(a - 1) << 32) | (unsigned)j));
    *b = nbr_at(g, a, (int)(h1 % (uint64_t)da));
    int db = ndeg(g, *b);
    if (db == 0) return 0;
    uint64_t h2 = mix64(h1);
    *c = nbr_at(g, *b, (int)(h2 % (uint64_t)db));
    return *c != a && *c != *b;
}

/* One 3-cycle round.  stats[0..6] = total delta, candidates, scanned, verified,
 * committed, best delta, valid triples. */
/* Every sampled triple of a round: b[(a-1)*partners + j], c[...] for slot j of
 * vertex a, 0 where the slot has no valid triple.  Returns the valid count. */
long long orc_triple_samples(void* p, uint64_t seed, int partners, int* bs, int* cs) {
    const orc* g = (const orc*)p;
    long long valid = 0;
    for (int a = 1; a <= g->n; a++)
        for (int j = 0; j < partners; j++) {
            int b = 0, c = 0;
            const size_t q = (size_t)(a - 1) * partners + j;
            if (orc_sample_triple(p, seed, a, j, &b, &c)) { bs[q] = b; cs[q] = c; valid++; }
            else { bs[q] = 0; cs[q] = 0; }
        }
    return valid;
}

/* One 3-cycle round; `given` (NULL: computed here) holds both rotations' deltas
 * of every slot, given[2*((a-1)*partners + j) + rot], ignored for slots
 * without a valid triple -- a test passes deltas it has checked by sampling
 * against this file's triple delta, where evaluating all of them on the CPU
 * would take minutes. */
int orc_triple_round_given(void* p, int* map, int partners, uint64_t seed, const int* given,
                           int max_candidates, int max_verify, long long* stats) {
    const orc* g = (const orc*)p;
    const int n = g->n;
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
    long long valid = 0;
    #pragma omp parallel for schedule(dynamic, 4) reduction(+:valid)
    for (int a = 1; a <= n; a++) {
        uint64_t k = ~0ULL;
        for (int j = 0; j < partners; j++) {
            int b, c;
            if (!orc_sample_triple(p, seed, a, j, &b, &c)) continue;
            valid++;
            for (int rot = 0; rot < 2; rot++) {
                int d = given ? given[2 * ((size_t)(a - 1) * partners + j) + rot]
                              : orc_triple_delta(p, map, a, b, c, rot);
                if (d > 0) {
                    uint64_t kk = ((uint64_t)(0x7fffffffu - (unsigned)d) << 32) |
                                  ((uint64_t)(a - 1) << 16) | ((unsigned)j << 1) | (unsigned)rot;
                    if (kk < k) k = kk;
                }
            }
        }
        keys[a - 1] = k;
    }
    qsort(keys, n, sizeof(uint64_t), cmp_u64);
    int nk = 0;
    while (nk < n && keys[nk] != ~0ULL) nk++;
    unsigned char* used = calloc(n + 1, 1);
    unsigned char* taint = calloc(n + 1, 1);
    long long total = 0;
    int scanned = 0, verified = 0, committed = 0;
    int lim = (max_candidates > 0 && max_candidates < nk) ? max_candidates : nk;
    for (int k = 0; k < lim; k++) {
        int a = (int)((keys[k] >> 16) & 0xffff) + 1, j = (int)((keys[k] >> 1) & 0x7fff), rot = (int)(keys[k] & 1);
        int d0 = (int)(0x7fffffffu - (unsigned)(keys[k] >> 32));
        int b = 0, c = 0;
        orc_sample_triple(p, seed, a, j, &b, &c);
        scanned++;
        if (used[a] || used[b] || used[c]) continue;
        int d = d0;
        if (taint[a] || taint[b] || taint[c]) {
            if (max_verify >= 0 && verified >= max_verify) continue;
            verified++;
            d = orc_triple_delta(p, map, a, b, c, rot);
        }
        if (d <= 0) continue;
        rotate(map, a, b, c, rot);
        used[a] = used[b] = used[c] = 1;
        total += d;
        committed++;
        taint_nbrs(g, a, taint); taint_nbrs(g, b, taint); taint_nbrs(g, c, taint);
    }
    if (stats) {
        stats[0] = total; stats[1] = nk; stats[2] = scanned; stats[3] = verified;
        stats[4] = committed; stats[5] = nk ? (long long)(0x7fffffffu - (unsigned)(keys[0] >> 32)) : 0;
        stats[6] = valid;
    }
    free(keys); free(used); free(taint);
    return committed;
}

int orc_triple_round(void* p, int* map, int partners, uint64_t seed, int max_candidates,
                     int max_verify, long long* stats) {
    return orc_triple_round_given(p, map, partners, seed, NULL, max_candidates, max_verify, stats);
}

/* ---- 4-set permutations ----
 * The k = 4 case of src/permutation.c:700-744 (generate_permutations over
 * the images of a 4-vertex set, scored with calculate_permutation_delta
 * :623-696), on sampled connected 4-sets and with the same best-per-vertex
 * set commit as the 3-cycle round.  Permutation index q in 1..23 is the q-th
 * permutation of (0,1,2,3) in lexicographic order (0 = identity): vertex i of
 * the set takes the image of vertex perm[q][i]. */
static const int kQuadPerm[24][4] = {
    {0,1,2,3},{0,1,3,2},{0,2,1,3},{0,2,3,1},{0,3,1,2},{0,3,2,1},
    {1,0,2,3},{1,0,3,2},{1,2,0,3},{1,2,3,0},{1,3,0,2},{1,3,2,0},
    {2,0,1,3},{2,0,3,1},{2,1,0,3},{2,1,3,0},{2,3,0,1},{2,3,1,0},
    {3,0,1,2},{3,0,2,1},{3,1,0,2},{3,1,2,0},{3,2,0,1},{3,2,1,0}};

static void permute4(int* map, const int* set, int q) {
    int f[4];
    for (int i = 0; i < 4; i++) f[i] = map[set[i]];
    for (int i = 0; i < 4; i++) map[set[i]] = f[kQuadPerm[q][i]];
}

int orc_quad_delta(void* p, const int* map, int a, int b, int c, int d, int q) {
    const orc* g = (const orc*)p;
    int set[4] = {a, b, c, d};
    int* m2 = (int*)malloc(sizeof(int) * (g->n + 1));
    memcpy(m2, map, sizeof(int) * (g->n + 1));
    long long before = orc_local_score(p, map, set, 4);
    permute4(m2, set, q);
    long long after = orc_local_score(p, m2, set, 4);
    free(m2);
    return (int)(after - before);
}

/* 3-step walk of slot j of vertex a along undirected G1 edges: a -> b -> c
 * -> d with h1 = mix64(seed ^ (a-1 << 32 | j)), h2 = mix64(h1), h3 =
 * mix64(h2); valid when the four vertices are distinct. */
int orc_sample_quad(void* p, uint64_t seed, int a, int j, int* b, int* c, int* d) {
    const orc* g = (const orc*)p;
    int da = ndeg(g, a);
    if (da == 0) return 0;
    uint64_t h1 = mix64(seed ^ (((uint64_t)(a - 1) << 32) | (unsigned)j));
    *b = nbr_at(g, a, (int)(h1 % (uint64_t)da));
    int db = ndeg(g, *b);
    if (db == 0) return 0;
    uint64_t h2 = mix64(h1);
    *c = nbr_at(g, *b, (int)(h2 % (uint64_t)db));
    int dc = ndeg(g, *c);
    if (dc == 0) return 0;
    uint64_t h3 = mix64(h2);
    *d = nbr_at(g, *c, (int)(h3 % (uint64_t)dc));
    return *b != a && *c != a && *c != *b && *d != a && *d != *b && *d != *c;
}

/* One 4-set round.  Keys (0x7fffffff - delta) << 32 | (a-1) << 16 | j << 5 | q;
 * stats[0..6] = total delta, candidates, scanned, verified, committed, best
 * delta, valid 4-sets. */
int orc_quad_round(void* p, int* map, int partners, uint64_t seed, int max_candidates,
                   int max_verify, long long* stats) {
    const orc* g = (const orc*)p;
    const int n = g->n;
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1));
    long long valid = 0;
    #pragma omp parallel for schedule(dynamic, 4) reduction(+:valid)
    for (int a = 1; a <= n; a++) {
        uint64_t k = ~0ULL;
        for (int j = 0; j < partners; j++) {
            int b, c, d;
            if (!orc_sample_quad(p, seed, a, j, &b, &c, &d)) continue;
            valid++;
            for (int q = 1; q < 24; q++) {
                int dd = orc_quad_delta(p, map, a, b, c, d, q);
                if (dd > 0) {
                    uint64_t kk = ((uint64_t)(0x7fffffffu - (unsigned)dd) << 32) |
                                  ((uint64_t)(a - 1) << 16) | ((unsigned)j << 5) | (unsigned)q;
                    if (kk < k) k = kk;
                }
            }
        }
        keys[a - 1] = k;
    }
    qsort(keys, n, sizeof(uint64_t), cmp_u64);
    int nk = 0;
    while (nk < n && keys[nk] != ~0ULL) nk++;
    unsigned char* used = calloc(n + 1, 1);
    unsigned char* taint = calloc(n + 1, 1);
    long long total = 0;
    int scanned = 0, verified = 0, committed = 0;
    int lim = (max_candidates > 0 && max_candidates < nk) ? max_candidates : nk;
    for (int k = 0; k < lim; k++) {
        int a = (int)((keys[k] >> 16) & 0xffff) + 1, j = (int)((keys[k] >> 5) & 0x7ff), q = (int)(keys[k] & 31);
        int d0 = (int)(0x7fffffffu - (unsigned)(keys[k] >> 32));
        int b = 0, c = 0, d = 0;
        orc_sample_quad(p, seed, a, j, &b, &c, &d);
        scanned++;
        if (used[a] || used[b] || used[c] || used[d]) continue;
        int dd = d0;
        if (taint[a] || taint[b] || taint[c] || taint[d]) {
            if (max_verify >= 0 && verified >= max_verify) continue;
            verified++;
            dd = orc_quad_delta(p, map, a, b, c, d, q);
        }
        if (dd <= 0) continue;
        int set[4] = {a, b, c, d};
        permute4(map, set, q);
        used[a] = used[b] = used[c] = used[d] = 1;
        total += dd;
        committed++;
        taint_nbrs(g, a, taint); taint_nbrs(g, b, taint); taint_nbrs(g, c, taint); taint_nbrs(g, d, taint);
    }
    if (stats) {
        stats[0] = total; stats[1] = nk; stats[2] = scanned; stats[3] = verified;
        stats[4] = committed; stats[5] = nk ? (long long)(0x7fffffffu - (unsigned)(keys[0] >> 32)) : 0;
        stats[6] = valid;
    }
    free(keys); free(used); free(taint);
    return committed;
}

/* Best-swap descent on an exact table (src/best-swap/score-lookup.c:597-640
 * with every delta current): each step swaps the pair of largest delta over
 * all pairs, the first in (m1, m2) order among equals, while that delta is
 * > 0.  swaps[2i], swaps[2i+1] and deltas[i] record step i (either may be
 * NULL).  Returns the number of swaps. */
int orc_best_swap_descent(void* p, int* map, int max_swaps, int* swaps, int* deltas) {
    const orc* g = (const orc*)p;
    const int n = g->n;
    int done = 0;
    while (done < max_swaps) {
        int bd = 0, ba = 0, bb = 0;
        for (int a = 1; a <= n; a++)
            for (int b = a + 1; b <= n; b++) {
                const int d = orc_swap_delta(p, map, a, b);
                if (d > bd) { bd = d; ba = a; bb = b; }
            }
        if (bd <= 0) break;
        const int t = map[ba]; map[ba] = map[bb]; map[bb] = t;
        if (swaps) { swaps[2 * done] = ba; swaps[2 * done + 1] = bb; }
        if (deltas) deltas[done] = bd;
        done++;
    }
    return done;
}

/* ---- greedy feature matcher (src/greedy-feature-match.c:527-712) ---- */

typedef struct { int *off, *id, *w; } glists;

/* rows keyed by key[] (0-based), every entry, input order within a row */
static void g_csr(int n, long long m, const int* key, const int* other, const int* w, glists* L) {
    L->off = (int*)calloc((size_t)n + 1, sizeof(int));
    L->id = (int*)malloc(sizeof(int) * (size_t)(m ? m : 1));
    L->w = (int*)malloc(sizeof(int) * (size_t)(m ? m : 1));
    for (long long i = 0; i < m; i++) L->off[key[i] + 1]++;
    for (int v = 0; v < n; v++) L->off[v + 1] += L->off[v];
    int* pos = (int*)malloc(sizeof(int) * (size_t)(n ? n : 1));
    memcpy(pos, L->off, sizeof(int) * (size_t)n);
    for (long long i = 0; i < m; i++) {
        const int p = pos[key[i]]++;
        L->id[p] = other[i];
        L->w[p] = w ? w[i] : 0;
    }
    free(pos);
}

static void g_free(glists* L) { free(L->off); free(L->id); free(L->w); }

/* distinct w with u -> v -> w along L */
static int g_two_hop(const glists* L, int n, int u, unsigned char* seen) {
    int c = 0;
    memset(seen, 0, (size_t)n);
    for (int j = L->off[u]; j < L->off[u + 1]; j++) {
        const int v = L->id[j];
        for (int k = L->off[v]; k < L->off[v + 1]; k++)
            if (!seen[L->id[k]]) { seen[L->id[k]] = 1; c++; }
    }
    return c;
}

/* compute_vertex_features (:527-566) over 1-based edges: feat[4(v-1)+k] =
 * in-degree, out-degree, 2-hop reachable, 2-hop can-reach (every edge entry
 * counts, self-loops and repeats included). */
void orc_greedy_features(int n, long long e, const int* src, const int* dst, int* feat) {
    int* s0 = (int*)malloc(sizeof(int) * (size_t)(e ? e : 1));
    int* d0 = (int*)malloc(sizeof(int) * (size_t)(e ? e : 1));
    for (long long i = 0; i < e; i++) { s0[i] = src[i] - 1; d0[i] = dst[i] - 1; }
    glists lo, li;
    g_csr(n, e, s0, d0, NULL, &lo);
    g_csr(n, e, d0, s0, NULL, &li);
    #pragma omp parallel
    {
        unsigned char* seen = (unsigned char*)malloc((size_t)n + 1);
        #pragma omp for schedule(dynamic, 16)
        for (int v = 0; v < n; v++) {
            feat[4 * v + 0] = li.off[v + 1] - li.off[v];
            feat[4 * v + 1] = lo.off[v + 1] - lo.off[v];
            feat[4 * v + 2] = g_two_hop(&lo, n, v, seen);
            feat[4 * v + 3] = g_two_hop(&li, n, v, seen);
        }
        free(seen);
    }
    g_free(&lo); g_free(&li); free(s0); free(d0);
}

static void g_ratios(const int* f, double* r) {
    const int total = f[0] + f[1] + f[2] + f[3];
    for (int k = 0; k < 4; k++) r[k] = total > 0 ? (double)f[k] / (double)total : 0.0;
}

static int g_distance(const double* r1, const double* r2) {
    const double d1 = fabs(r1[0] - r2[0]), d2 = fabs(r1[1] - r2[1]);
    const double d3 = fabs(r1[2] - r2[2]), d4 = fabs(r1[3] - r2[3]);
    return (int)((d1 + d2 + d3 + d4) * 1000);
}

/* compute_feature_distance (:575-586) of two feature rows (in, out, r2, c2);
 * a row whose total is 0 has ratios 0. */
int orc_greedy_distance(const int* f1, const int* f2) {
    double r1[4], r2[4];
    g_ratios(f1, r1);
    g_ratios(f2, r2);
    return g_distance(r1, r2);
}

typedef struct { unsigned total; int v; } g_key;
static int g_cmp(const void* a, const void* b) {
    const g_key* x = (const g_key*)a;
    const g_key* y = (const g_key*)b;
    if (x->total != y->total) return x->total > y->total ? -1 : 1;
    return x->v < y->v ? -1 : (x->v > y->v);
}

/* match_vertices (:588-676): map[v] (1-based, n+1 entries) = the G2 vertex
 * chosen for G1 vertex v. */
void orc_greedy_match(int n, long long e1, const int* s1, const int* d1, const int* w1,
                      long long e2, const int* s2, const int* d2, const int* w2, int* map) {
    int* f1 = (int*)malloc(sizeof(int) * 4 * (size_t)n);
    int* f2 = (int*)malloc(sizeof(int) * 4 * (size_t)n);
    orc_greedy_features(n, e1, s1, d1, f1);
    orc_greedy_features(n, e2, s2, d2, f2);
    double* r1 = (double*)malloc(sizeof(double) * 4 * (size_t)n);
    double* r2 = (double*)malloc(sizeof(double) * 4 * (size_t)n);
    g_key* k1 = (g_key*)malloc(sizeof(g_key) * (size_t)n);
    g_key* k2 = (g_key*)malloc(sizeof(g_key) * (size_t)n);
    for (int v = 0; v < n; v++) {
        g_ratios(f1 + 4 * v, r1 + 4 * v);
        g_ratios(f2 + 4 * v, r2 + 4 * v);
        k1[v].total = (unsigned)(f1[4 * v] + f1[4 * v + 1] + f1[4 * v + 2] + f1[4 * v + 3]); k1[v].v = v;
        k2[v].total = (unsigned)(f2[4 * v] + f2[4 * v + 1] + f2[4 * v + 2] + f2[4 * v + 3]); k2[v].v = v;
    }
    qsort(k1, (size_t)n, sizeof(g_key), g_cmp);
    qsort(k2, (size_t)n, sizeof(g_key), g_cmp);
    /* G1 lists with every entry; G2 with the last weight of each pair */
    int *a1 = (int*)malloc(sizeof(int) * (size_t)(e1 ? e1 : 1)), *b1 = (int*)malloc(sizeof(int) * (size_t)(e1 ? e1 : 1));
    for (long long i = 0; i < e1; i++) { a1[i] = s1[i] - 1; b1[i] = d1[i] - 1; }
    glists g1o, g1i;
    g_csr(n, e1, a1, b1, w1, &g1o);
    g_csr(n, e1, b1, a1, w1, &g1i);
    int *a2 = (int*)malloc(sizeof(int) * (size_t)(e2 ? e2 : 1)), *b2 = (int*)malloc(sizeof(int) * (size_t)(e2 ? e2 : 1));
    int* c2 = (int*)malloc(sizeof(int) * (size_t)(e2 ? e2 : 1));
    long long m2 = 0;
    {
        glists t;
        int* s20 = (int*)malloc(sizeof(int) * (size_t)(e2 ? e2 : 1));
        int* d20 = (int*)malloc(sizeof(int) * (size_t)(e2 ? e2 : 1));
        for (long long i = 0; i < e2; i++) { s20[i] = s2[i] - 1; d20[i] = d2[i] - 1; }
        g_csr(n, e2, s20, d20, w2, &t);
        int* last = (int*)malloc(sizeof(int) * (size_t)n);
        for (int v = 0; v < n; v++) last[v] = -1;
        for (int u = 0; u < n; u++)
            for (int k = t.off[u + 1] - 1; k >= t.off[u]; k--) {
                const int v = t.id[k];
                if (last[v] == u) continue;
                last[v] = u;
                a2[m2] = u; b2[m2] = v; c2[m2] = t.w[k]; m2++;
            }
        free(last); free(s20); free(d20); g_free(&t);
    }
    glists g2o, g2i;
    g_csr(n, m2, a2, b2, c2, &g2o);
    g_csr(n, m2, b2, a2, c2, &g2i);
    int* m0 = (int*)malloc(sizeof(int) * (size_t)n);        /* G1 -> G2, -1 unmatched */
    unsigned char* taken = (unsigned char*)calloc((size_t)n, 1);
    long long* acc = (long long*)calloc((size_t)n, sizeof(long long));
    for (int v = 0; v < n; v++) m0[v] = -1;
    for (int i = 0; i < n; i++) {
        const int v1 = k1[i].v;
        for (int j = g1o.off[v1]; j < g1o.off[v1 + 1]; j++) {       /* v1 -> t */
            const int f = m0[g1o.id[j]], w = g1o.w[j];
            if (f < 0) continue;
            for (int k = g2i.off[f]; k < g2i.off[f + 1]; k++) acc[g2i.id[k]] += MIN(w, g2i.w[k]);
        }
        for (int j = g1i.off[v1]; j < g1i.off[v1 + 1]; j++) {       /* s -> v1 */
            const int f = m0[g1i.id[j]], w = g1i.w[j];
            if (f < 0) continue;
            for (int k = g2o.off[f]; k < g2o.off[f + 1]; k++) acc[g2o.id[k]] += MIN(w, g2o.w[k]);
        }
        double best = -INFINITY;
        int bg = -1;
        for (int j = 0; j < n; j++) {
            const int v2 = k2[j].v;
            if (taken[v2]) continue;
            const double st = -g_distance(r1 + 4 * v1, r2 + 4 * v2);
            const double al = (double)acc[v2];
            const double tot = 0.3 * st + 0.7 * al;
            if (tot > best) { best = tot; bg = v2; }
        }
        memset(acc, 0, sizeof(long long) * (size_t)n);
        m0[v1] = bg;
        if (bg >= 0) taken[bg] = 1;
    }
    map[0] = 0;
    for (int v = 0; v < n; v++) map[v + 1] = m0[v] + 1;
    free(m0); free(taken); free(acc);
    g_free(&g1o); g_free(&g1i); g_free(&g2o); g_free(&g2i);
    free(a1); free(b1); free(a2); free(b2); free(c2);
    free(f1); free(f2); free(r1); free(r2); free(k1); free(k2);
}
