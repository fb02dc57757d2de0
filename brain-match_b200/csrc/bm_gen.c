/*
 * bm_gen.c -- seeded synthetic graph-pair generator (host C).
 *
 * The reference's own inputs (the VNC male/female connectomes) are not
 * available, so workloads are synthetic graphs with the reference's shapes:
 *   G1: n vertices, exactly e directed edges, no self-loops or duplicates,
 *       out-degrees from a power law (exponent alpha) scaled to sum to e,
 *       targets uniform; weights 1 + Geometric(geom_p) failures, with an
 *       optional heavy tail floor(tail_scale * Pareto(tail_alpha)), capped
 *       at wmax.
 *   G2: G1 relabelled by a random permutation pi, del_frac of its edges
 *       deleted, add_frac*e random new edges added (no self-loops or
 *       duplicates), every weight jittered by uniform{-jitter..jitter},
 *       floored at 1 and capped at wmax.
 *   map0: a uniform random matching.
 * Everything is drawn from one xoshiro256** stream seeded by splitmix64, in a
 * fixed order, so a (params, seed) pair always gives the same graphs.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include "bm.h"

typedef struct { uint64_t s[4]; } rng_t;

static uint64_t splitmix64(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static void rng_seed(rng_t* r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&x);
}
static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
static uint64_t rng_next(rng_t* r) {
    uint64_t* s = r->s;
    uint64_t res = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return res;
}
/* uniform in (0,1] */
static double rng_unit(rng_t* r) { return ((rng_next(r) >> 11) + 1) * (1.0 / 9007199254740992.0); }
/* uniform integer in [0,m) */
static uint64_t rng_below(rng_t* r, uint64_t m) {
    return (uint64_t)(((unsigned __int128)rng_next(r) * m) >> 64);
}

void bm_gen_defaults(bm_gen_params* p) {
    memset(p, 0, sizeof *p);
    p->n = 1000; p->e = 20000; p->seed = 20261203ULL;
    p->alpha = 2.1; p->geom_p = 0.35; p->wmax = 5000;
    p->tail_prob = 0.0; p->tail_alpha = 1.1; p->tail_scale = 8.0;
    p->del_frac = 0.1; p->add_frac = 0.1; p->jitter = 1;
}

static int32_t draw_weight(rng_t* r, const bm_gen_params* p) {
    double w;
    if (p->tail_prob > 0 && rng_unit(r) <= p->tail_prob) {
        w = floor(p->tail_scale * pow(rng_unit(r), -1.0 / p->tail_alpha));
    } else {
        w = 1.0 + floor(log(rng_unit(r)) / log(1.0 - p->geom_p));
    }
    if (w < 1) w = 1;
    if (w > p->wmax) w = p->wmax;
    return (int32_t)w;
}

static int cmp_i32(const void* a, const void* b) {
    int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
    return (x > y) - (x < y);
}

/* open-addressing set of 64-bit keys (key+1 stored, 0 = empty) */
typedef struct { uint64_t* t; uint64_t mask; } hset_t;
static int hs_init(hset_t* h, int64_t cap) {
    uint64_t sz = 1;
    while (sz < (uint64_t)cap * 2 + 16) sz <<= 1;
    h->t = (uint64_t*)calloc(sz, sizeof(uint64_t));
    h->mask = sz - 1;
    return h->t != NULL;
}
static inline uint64_t hs_hash(uint64_t k) { k ^= k >> 33; k *= 0xff51afd7ed558ccdULL; k ^= k >> 33; return k; }
/* returns 1 if inserted, 0 if present */
static int hs_insert(hset_t* h, uint64_t key) {
    uint64_t i = hs_hash(key) & h->mask;
    while (h->t[i]) {
        if (h->t[i] == key + 1) return 0;
        i = (i + 1) & h->mask;
    }
    h->t[i] = key + 1;
    return 1;
}

static int cmp64(const void* a, const void* b) {
    int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x > y) - (x < y);
}

/* sorts (src,dst,w) triplets by (src,dst) with a counting sort on src */
static int sort_edges(int32_t n, int64_t m, int32_t* s, int32_t* d, int32_t* w) {
    int64_t* off = (int64_t*)calloc((size_t)n + 2, sizeof(int64_t));
    int32_t* d2 = (int32_t*)malloc(sizeof(int32_t) * (size_t)(m ? m : 1));
    int64_t* key = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
    if (!off || !d2 || !key) { free(off); free(d2); free(key); return 0; }
    for (int64_t i = 0; i < m; i++) off[s[i] + 1]++;
    for (int32_t v = 0; v < n; v++) off[v + 1] += off[v];
    int64_t* pos = (int64_t*)malloc(sizeof(int64_t) * ((size_t)n + 1));
    if (!pos) { free(off); free(d2); free(key); return 0; }
    memcpy(pos, off, sizeof(int64_t) * ((size_t)n + 1));
    for (int64_t i = 0; i < m; i++) {
        int64_t q = pos[s[i]]++;
        key[q] = ((int64_t)d[i] << 32) | (uint32_t)w[i];
    }
    for (int32_t v = 0; v < n; v++) {
        int64_t a = off[v], b = off[v + 1];
        /* sort by dst (upper 32 bits); dst values are unique within a row */
        if (b - a <= 64) {
            for (int64_t i = a + 1; i < b; i++) {
                int64_t x = key[i], j = i - 1;
                while (j >= a && key[j] > x) { key[j + 1] = key[j]; j--; }
                key[j + 1] = x;
            }
        } else {
            qsort(key + a, (size_t)(b - a), sizeof(int64_t), cmp64);
        }
        for (int64_t i = a; i < b; i++) {
            s[i] = v;
            d2[i] = (int32_t)(key[i] >> 32);
            w[i] = (int32_t)(uint32_t)(key[i] & 0xffffffffu);
        }
    }
    memcpy(d, d2, sizeof(int32_t) * (size_t)m);
    free(off); free(d2); free(key); free(pos);
    return 1;
}

bm_status bm_generate(const bm_gen_params* prm,
                      int32_t* src1, int32_t* dst1, int32_t* w1,
                      int64_t* e2out, int32_t* src2, int32_t* dst2, int32_t* w2,
                      int32_t* pi, int32_t* map0) {
    if (!prm || !src1 || !dst1 || !w1 || !e2out || !src2 || !dst2 || !w2 || !pi || !map0)
        return BM_E_INPUT;
    const int32_t n = prm->n;
    const int64_t e = prm->e;
    if (n < 2 || e < 0 || e > (int64_t)n * (n - 1) || prm->alpha <= 1.0 ||
        prm->geom_p <= 0 || prm->geom_p >= 1 || prm->wmax < 1 ||
        prm->del_frac < 0 || prm->del_frac > 1 || prm->add_frac < 0 || prm->jitter < 0)
        return BM_E_INPUT;
    rng_t r;
    rng_seed(&r, prm->seed);

    /* ---- out-degrees: truncated power law on [1, n-1], scaled to sum e ---- */
    int64_t* deg = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
    int32_t* stamp = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    int32_t* buf = (int32_t*)malloc(sizeof(int32_t) * (size_t)n);
    if (!deg || !stamp || !buf) { free(deg); free(stamp); free(buf); return BM_E_NOMEM; }
    const double D = (double)(n - 1), a1 = prm->alpha - 1.0;
    const double tail = 1.0 - pow(D, -a1);
    double raw_sum = 0;
    for (int32_t i = 0; i < n; i++) {
        double x = pow(1.0 - rng_unit(&r) * tail, -1.0 / a1);
        double v = floor(x);
        if (v < 1) v = 1;
        if (v > D) v = D;
        deg[i] = (int64_t)v;
        raw_sum += v;
    }
    const int64_t lo = (e >= n) ? 1 : 0;
    int64_t sum = 0;
    for (int32_t i = 0; i < n; i++) {
        int64_t v = llround((double)deg[i] * ((double)e / raw_sum));
        if (v < lo) v = lo;
        if (v > n - 1) v = n - 1;
        deg[i] = v;
        sum += v;
    }
    while (sum < e) { int32_t i = (int32_t)rng_below(&r, n); if (deg[i] < n - 1) { deg[i]++; sum++; } }
    while (sum > e) { int32_t i = (int32_t)rng_below(&r, n); if (deg[i] > lo) { deg[i]--; sum--; } }

    /* ---- targets: distinct, != source, uniform; rows emitted sorted ---- */
    for (int32_t i = 0; i < n; i++) stamp[i] = -1;
    int64_t q = 0;
    for (int32_t s = 0; s < n; s++) {
        int64_t d = deg[s];
        if (d <= (n - 1) / 2) {
            int64_t c = 0;
            while (c < d) {
                int32_t t = (int32_t)rng_below(&r, n);
                if (t == s || stamp[t] == s) continue;
                stamp[t] = s;
                buf[c++] = t;
            }
            qsort(buf, (size_t)d, sizeof(int32_t), cmp_i32);
            for (int64_t k = 0; k < d; k++) { src1[q] = s; dst1[q] = buf[k]; q++; }
        } else {
            /* pick the (n-1-d) excluded targets, keep the rest in order */
            int64_t x = (n - 1) - d, c = 0;
            while (c < x) {
                int32_t t = (int32_t)rng_below(&r, n);
                if (t == s || stamp[t] == s) continue;
                stamp[t] = s;
                c++;
            }
            for (int32_t t = 0; t < n; t++)
                if (t != s && stamp[t] != s) { src1[q] = s; dst1[q] = t; q++; }
        }
    }
    for (int64_t k = 0; k < e; k++) w1[k] = draw_weight(&r, prm);

    /* ---- G2 = pi(G1) minus deletions plus additions, jittered ---- */
    int32_t* perm = buf;
    for (int32_t i = 0; i < n; i++) perm[i] = i;
    for (int32_t i = n - 1; i > 0; i--) {
        int32_t j = (int32_t)rng_below(&r, (uint64_t)i + 1);
        int32_t t = perm[i]; perm[i] = perm[j]; perm[j] = t;
    }
    const int64_t ndel = llround(prm->del_frac * (double)e);
    const int64_t nadd = llround(prm->add_frac * (double)e);
    /* deletion: partial Fisher-Yates over edge indices */
    int64_t* idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(e ? e : 1));
    unsigned char* dead = (unsigned char*)calloc((size_t)(e ? e : 1), 1);
    hset_t hs;
    if (!idx || !dead || !hs_init(&hs, e + nadd)) {
        free(idx); free(dead); free(deg); free(stamp); free(buf); return BM_E_NOMEM;
    }
    for (int64_t k = 0; k < e; k++) idx[k] = k;
    for (int64_t k = 0; k < ndel; k++) {
        int64_t j = k + (int64_t)rng_below(&r, (uint64_t)(e - k));
        int64_t t = idx[k]; idx[k] = idx[j]; idx[j] = t;
        dead[idx[k]] = 1;
    }
    int64_t m = 0;
    for (int64_t k = 0; k < e; k++) {
        if (dead[k]) continue;
        int32_t s = perm[src1[k]], d = perm[dst1[k]];
        src2[m] = s; dst2[m] = d; w2[m] = w1[k];
        hs_insert(&hs, (uint64_t)s * (uint64_t)n + (uint64_t)d);
        m++;
    }
    int64_t added = 0, tries = 0, max_tries = 64 * nadd + 4096;
    while (added < nadd && tries < max_tries) {
        tries++;
        int32_t s = (int32_t)rng_below(&r, n), d = (int32_t)rng_below(&r, n);
        if (s == d) continue;
        if (!hs_insert(&hs, (uint64_t)s * (uint64_t)n + (uint64_t)d)) continue;
        src2[m] = s; dst2[m] = d; w2[m] = draw_weight(&r, prm);
        m++; added++;
    }
    free(idx); free(dead); free(hs.t);
    if (added < nadd) { free(deg); free(stamp); free(buf); return BM_E_INPUT; }
    for (int64_t k = 0; k < m; k++) {
        int32_t j = (int32_t)rng_below(&r, 2 * (uint64_t)prm->jitter + 1) - prm->jitter;
        int64_t v = (int64_t)w2[k] + j;
        if (v < 1) v = 1;
        if (v > prm->wmax) v = prm->wmax;
        w2[k] = (int32_t)v;
    }
    if (!sort_edges(n, m, src2, dst2, w2)) { free(deg); free(stamp); free(buf); return BM_E_NOMEM; }

    /* ---- initial matching: uniform random permutation ---- */
    pi[0] = 0;
    for (int32_t i = 0; i < n; i++) pi[i + 1] = perm[i] + 1;
    for (int32_t i = 0; i < n; i++) buf[i] = i;
    for (int32_t i = n - 1; i > 0; i--) {
        int32_t j = (int32_t)rng_below(&r, (uint64_t)i + 1);
        int32_t t = buf[i]; buf[i] = buf[j]; buf[j] = t;
    }
    map0[0] = 0;
    for (int32_t i = 0; i < n; i++) map0[i + 1] = buf[i] + 1;

    /* 1-based ids at the boundary */
    for (int64_t k = 0; k < e; k++) { src1[k]++; dst1[k]++; }
    for (int64_t k = 0; k < m; k++) { src2[k]++; dst2[k]++; }
    *e2out = m;
    free(deg); free(stamp); free(buf);
    return BM_OK;
}
