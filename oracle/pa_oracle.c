/*
 * pa_oracle.c -- sequential CPU oracle for the copy-model PA generator.
 *
 * TEST INFRASTRUCTURE ONLY (see pa_oracle.h).  Plain C, single thread, no
 * attempt at speed beyond a tight loop: it is the checker and the timed CPU
 * restatement, never the product.
 */
#include "pa_oracle.h"

#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon et al., SC'11).  Multipliers and Weyl key increments
 * are the published constants of the Philox-4x32 family.                    */
/* ------------------------------------------------------------------------ */
#define PHILOX_M0 0xD2511F53u
#define PHILOX_M1 0xCD9E8D57u
#define PHILOX_W0 0x9E3779B9u
#define PHILOX_W1 0xBB67AE85u

static inline void philox_round(uint32_t x[4], uint32_t k0, uint32_t k1)
{
    uint64_t p0 = (uint64_t)PHILOX_M0 * x[0];
    uint64_t p1 = (uint64_t)PHILOX_M1 * x[2];
    uint32_t y0 = (uint32_t)(p1 >> 32) ^ x[1] ^ k0;
    uint32_t y1 = (uint32_t)p1;
    uint32_t y2 = (uint32_t)(p0 >> 32) ^ x[3] ^ k1;
    uint32_t y3 = (uint32_t)p0;
    x[0] = y0; x[1] = y1; x[2] = y2; x[3] = y3;
}

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t x[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        philox_round(x, k0, k1);
        k0 += PHILOX_W0;
        k1 += PHILOX_W1;
    }
    out[0] = x[0]; out[1] = x[1]; out[2] = x[2]; out[3] = x[3];
}

/* ------------------------------------------------------------------------ */
/* MT19937-64 (Matsumoto & Nishimura), the generator behind the reference's  */
/* Random::Uniform() (src/Common/Random64.hpp:64-102).                        */
/* ------------------------------------------------------------------------ */
#define MT_N 312
#define MT_M 156
#define MT_A 0xB5026F5AA96619E9ULL
#define MT_UPPER 0xFFFFFFFF80000000ULL
#define MT_LOWER 0x000000007FFFFFFFULL

typedef struct {
    uint64_t s[MT_N];
    int idx;
} mt64;

static void mt64_seed(mt64 *m, uint64_t seed)
{
    m->s[0] = seed;
    for (int i = 1; i < MT_N; ++i)
        m->s[i] = 6364136223846793005ULL * (m->s[i - 1] ^ (m->s[i - 1] >> 62)) + (uint64_t)i;
    m->idx = MT_N;
}

static void mt64_twist(mt64 *m)
{
    for (int i = 0; i < MT_N; ++i) {
        uint64_t y = (m->s[i] & MT_UPPER) | (m->s[(i + 1) % MT_N] & MT_LOWER);
        uint64_t v = m->s[(i + MT_M) % MT_N] ^ (y >> 1);
        if (y & 1ULL) v ^= MT_A;
        m->s[i] = v;
    }
    m->idx = 0;
}

static inline uint64_t mt64_next(mt64 *m)
{
    if (m->idx >= MT_N) mt64_twist(m);
    uint64_t x = m->s[m->idx++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= (x >> 43);
    return x;
}

void orc_mt19937_64(uint64_t seed, uint64_t count, uint64_t *out)
{
    mt64 m;
    mt64_seed(&m, seed);
    for (uint64_t i = 0; i < count; ++i) out[i] = mt64_next(&m);
}

/* ------------------------------------------------------------------------ */
/* Parameters and seed graph                                                 */
/* ------------------------------------------------------------------------ */
uint64_t orc_p_threshold(double p)
{
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 1ULL << 32;
    double t = p * 4294967296.0; /* exact: scaling by a power of two */
    uint64_t th = (uint64_t)t;   /* floor for non-negative values */
    if (th > (1ULL << 32)) th = 1ULL << 32;
    return th;
}

uint64_t orc_seed_edge_count(uint32_t d, int seed_mode)
{
    if (seed_mode == ORC_SEED_CLIQUE) return (uint64_t)d * (d + 1) / 2;
    return d; /* star node d linked to 0..d-1 */
}

uint64_t orc_edge_count(uint64_t n, uint32_t d, int seed_mode)
{
    if (n < (uint64_t)d + 1) return 0;
    return orc_seed_edge_count(d, seed_mode) + (n - d - 1) * (uint64_t)d;
}

/* Value of slot k of seed node v (v <= d). */
static inline int64_t seed_slot(uint64_t v, uint32_t k, uint32_t d, int seed_mode)
{
    if (seed_mode == ORC_SEED_CLIQUE) return (int64_t)(k < v ? k : k + 1);
    return (int64_t)(v < d ? v : k);
}

static inline uint64_t mulhi64(uint64_t a, uint64_t b)
{
    return (uint64_t)(((unsigned __int128)a * b) >> 64);
}

/* Generation loops for int64 and int32 slot storage (pa_oracle_gen.inc). */
#define SLOT_T int64_t
#define GEN_FN(name) name##_i64
#include "pa_oracle_gen.inc"
#undef SLOT_T
#undef GEN_FN
#define SLOT_T int32_t
#define GEN_FN(name) name##_i32
#include "pa_oracle_gen.inc"
#undef SLOT_T
#undef GEN_FN

int orc_generate(uint64_t n, uint32_t d, double p, uint64_t seed, int seed_mode, int rng,
                 int64_t *G, uint64_t *retries_out)
{
    return generate_i64(n, d, p, seed, seed_mode, rng, G, retries_out);
}

int orc_generate_ba(uint64_t n, uint32_t d, uint64_t seed, int rng, int64_t *G,
                    uint64_t *retries_out)
{
    return generate_ba_i64(n, d, seed, rng, G, retries_out);
}

/* ------------------------------------------------------------------------ */
/* Output forms                                                              */
/* ------------------------------------------------------------------------ */
static void sort_small(int64_t *a, uint32_t len)
{
    for (uint32_t i = 1; i < len; ++i) {
        int64_t x = a[i];
        uint32_t j = i;
        while (j > 0 && a[j - 1] > x) { a[j] = a[j - 1]; --j; }
        a[j] = x;
    }
}

/* Seed rows' canonical edges (v, w) with w < v, rows ascending. */
static uint64_t emit_seed(uint32_t d, int seed_mode, const int64_t *G, int64_t *pairs)
{
    uint64_t e = 0;
    for (uint64_t v = 0; v <= d; ++v)
        for (uint32_t k = 0; k < d; ++k) {
            int64_t w = G[v * d + k];
            if (w < (int64_t)v) {
                pairs[2 * e] = (int64_t)v;
                pairs[2 * e + 1] = w;
                ++e;
            }
        }
    (void)seed_mode;
    return e;
}

void orc_pairs_slot_order(uint64_t n, uint32_t d, int seed_mode, const int64_t *G,
                          int64_t *pairs)
{
    uint64_t e = emit_seed(d, seed_mode, G, pairs);
    for (uint64_t u = (uint64_t)d + 1; u < n; ++u)
        for (uint32_t i = 0; i < d; ++i, ++e) {
            pairs[2 * e] = (int64_t)u;
            pairs[2 * e + 1] = G[u * d + i];
        }
}

void orc_pairs_canonical(uint64_t n, uint32_t d, int seed_mode, const int64_t *G,
                         int64_t *pairs)
{
    uint64_t e = emit_seed(d, seed_mode, G, pairs);
    int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * d);
    for (uint64_t u = (uint64_t)d + 1; u < n; ++u) {
        memcpy(tmp, G + u * d, sizeof(int64_t) * d);
        sort_small(tmp, d);
        for (uint32_t i = 0; i < d; ++i, ++e) {
            pairs[2 * e] = (int64_t)u;
            pairs[2 * e + 1] = tmp[i];
        }
    }
    free(tmp);
}

void orc_degrees(uint64_t n, uint32_t d, int seed_mode, const int64_t *G, int64_t *deg)
{
    memset(deg, 0, sizeof(int64_t) * n);
    for (uint64_t v = 0; v <= d && v < n; ++v)
        for (uint32_t k = 0; k < d; ++k) {
            int64_t w = G[v * d + k];
            if (w < (int64_t)v) { deg[v]++; deg[w]++; }
        }
    (void)seed_mode;
    for (uint64_t u = (uint64_t)d + 1; u < n; ++u) {
        deg[u] += d;
        for (uint32_t i = 0; i < d; ++i) deg[G[u * d + i]]++;
    }
}

void orc_csr(uint64_t n, uint32_t d, int seed_mode, const int64_t *G, int64_t *rowptr,
             int64_t *col)
{
    uint64_t E = orc_edge_count(n, d, seed_mode);
    int64_t *pairs = (int64_t *)malloc(sizeof(int64_t) * 2 * (E ? E : 1));
    int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (n ? n : 1));
    orc_pairs_canonical(n, d, seed_mode, G, pairs);
    orc_degrees(n, d, seed_mode, G, cur);
    rowptr[0] = 0;
    for (uint64_t x = 0; x < n; ++x) rowptr[x + 1] = rowptr[x] + cur[x];
    for (uint64_t x = 0; x < n; ++x) cur[x] = rowptr[x];
    /* Canonical order appends, to row x, first its own targets v < x (row x
     * is visited before any u > x) and then every u > x in increasing u: the
     * rows come out sorted without a sort. */
    for (uint64_t e = 0; e < E; ++e) {
        int64_t u = pairs[2 * e], v = pairs[2 * e + 1];
        col[cur[u]++] = v;
        col[cur[v]++] = u;
    }
    free(cur);
    free(pairs);
}

/* ------------------------------------------------------------------------ */
/* Whole-graph digests                                                       */
/* ------------------------------------------------------------------------ */
/* MurmurHash3's 64-bit finalizer (Appleby, public domain): a bijective mix. */
static inline uint64_t fmix64(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xFF51AFD7ED558CCDULL;
    k ^= k >> 33;
    k *= 0xC4CEB9FE1A85EC53ULL;
    k ^= k >> 33;
    return k;
}

/* Term of element x at position pos: the position is mixed in first, so the
 * digest changes when two elements trade places. */
static inline uint64_t digest_term(uint64_t pos, uint64_t x)
{
    return fmix64(fmix64(pos * 0x9E3779B97F4A7C15ULL + 0x632BE59BD9B4E019ULL) ^ x);
}

static inline void digest_add(uint64_t acc[2], uint64_t pos, int64_t x)
{
    const uint64_t h = digest_term(pos, (uint64_t)x);
    acc[0] += h;
    acc[1] ^= h;
}

void orc_digest_ids(const int64_t *x, uint64_t count, uint64_t index_base, uint64_t acc[2])
{
    for (uint64_t i = 0; i < count; ++i) digest_add(acc, index_base + i, x[i]);
}

/* Canonical seed edges of row v <= d, targets ascending, into tmp; returns how many. */
static uint32_t seed_row_targets(uint64_t v, uint32_t d, const int32_t *G, int64_t *tmp)
{
    uint32_t c = 0;
    for (uint32_t k = 0; k < d; ++k)
        if ((int64_t)G[v * d + k] < (int64_t)v) tmp[c++] = G[v * d + k];
    sort_small(tmp, c);
    return c;
}

int orc_graph_digests(uint64_t n, uint32_t d, double p, uint64_t seed, int seed_mode, int model,
                      int with_csr, uint64_t out[7])
{
    if (d == 0 || n < (uint64_t)d + 1 || n > (1ULL << 31) || out == NULL) return -1;
    if (model != ORC_MODEL_COPY && model != ORC_MODEL_BA) return -1;
    int32_t *G = (int32_t *)malloc(sizeof(int32_t) * n * d);
    int64_t *tmp = (int64_t *)malloc(sizeof(int64_t) * d);
    if (!G || !tmp) { free(G); free(tmp); return -2; }
    uint64_t retries = 0;
    const int rc = model == ORC_MODEL_BA
                       ? generate_ba_i32(n, d, seed, ORC_RNG_PHILOX, G, &retries)
                       : generate_i32(n, d, p, seed, seed_mode, ORC_RNG_PHILOX, G, &retries);
    if (rc != 0) { free(G); free(tmp); return rc; }
    for (int i = 0; i < 7; ++i) out[i] = 0;
    out[6] = retries;

    /* PAIRS slot order as one flat id array: src of edge e at 2e, dst at 2e+1. */
    uint64_t e = 0;
    for (uint64_t v = 0; v <= d; ++v)
        for (uint32_t k = 0; k < d; ++k) {
            const int64_t w = G[v * d + k];
            if (w < (int64_t)v) {
                digest_add(out, 2 * e, (int64_t)v);
                digest_add(out, 2 * e + 1, w);
                ++e;
            }
        }
    for (uint64_t u = (uint64_t)d + 1; u < n; ++u)
        for (uint32_t i = 0; i < d; ++i, ++e) {
            digest_add(out, 2 * e, (int64_t)u);
            digest_add(out, 2 * e + 1, G[u * d + i]);
        }

    if (with_csr) {
        /* rp[x] = row start (degrees, then an exclusive scan). */
        uint64_t *rp = (uint64_t *)calloc(n + 1, sizeof(uint64_t));
        if (!rp) { free(G); free(tmp); return -2; }
        for (uint64_t v = 0; v <= d; ++v)
            for (uint32_t k = 0; k < d; ++k) {
                const int64_t w = G[v * d + k];
                if (w < (int64_t)v) { rp[v + 1]++; rp[w + 1]++; }
            }
        for (uint64_t u = (uint64_t)d + 1; u < n; ++u) {
            rp[u + 1] += d;
            for (uint32_t i = 0; i < d; ++i) rp[(uint64_t)G[u * d + i] + 1]++;
        }
        for (uint64_t x = 0; x < n; ++x) rp[x + 1] += rp[x];
        for (uint64_t x = 0; x <= n; ++x) digest_add(out + 2, x, (int64_t)rp[x]);
        /* Out parts: row x's own targets (< x) ascending at the row's start; the
         * row start then becomes the cursor of its in part. */
        for (uint64_t x = 0; x < n; ++x) {
            uint32_t c;
            if (x <= d) {
                c = seed_row_targets(x, d, G, tmp);
            } else {
                for (uint32_t i = 0; i < d; ++i) tmp[i] = G[x * d + i];
                sort_small(tmp, d);
                c = d;
            }
            for (uint32_t j = 0; j < c; ++j) digest_add(out + 4, rp[x] + j, tmp[j]);
            rp[x] += c;
        }
        /* In parts: every u > v in increasing u, appended to row v. */
        for (uint64_t u = 1; u < n; ++u) {
            if (u <= d) {
                const uint32_t c = seed_row_targets(u, d, G, tmp);
                for (uint32_t j = 0; j < c; ++j) digest_add(out + 4, rp[tmp[j]]++, (int64_t)u);
            } else {
                for (uint32_t i = 0; i < d; ++i)
                    digest_add(out + 4, rp[(uint64_t)G[u * d + i]]++, (int64_t)u);
            }
        }
        free(rp);
    }
    free(tmp);
    free(G);
    return 0;
}

uint64_t orc_fnv1a64(const void *data, uint64_t bytes)
{
    const unsigned char *b = (const unsigned char *)data;
    uint64_t h = 0xcbf29ce484222325ULL;
    for (uint64_t i = 0; i < bytes; ++i) {
        h ^= b[i];
        h *= 0x100000001b3ULL;
    }
    return h;
}
