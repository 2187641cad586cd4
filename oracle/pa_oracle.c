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

int orc_generate(uint64_t n, uint32_t d, double p, uint64_t seed, int seed_mode, int rng,
                 int64_t *G, uint64_t *retries_out)
{
    if (d == 0 || n < (uint64_t)d + 1 || G == NULL) return -1;
    if (seed_mode != ORC_SEED_STAR_REF && seed_mode != ORC_SEED_CLIQUE) return -1;
    if (rng != ORC_RNG_PHILOX && rng != ORC_RNG_MT_REF) return -1;

    for (uint64_t v = 0; v <= d; ++v)
        for (uint32_t k = 0; k < d; ++k) G[v * d + k] = seed_slot(v, k, d, seed_mode);

    uint64_t retries = 0;
    if (rng == ORC_RNG_PHILOX) {
        const uint64_t pth = orc_p_threshold(p);
        const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
        for (uint64_t u = (uint64_t)d + 1; u < n; ++u) {
            int64_t *row = G + u * d;
            for (uint32_t i = 0; i < d; ++i) {
                for (uint32_t r = 0;; ++r) {
                    const uint32_t ctr[4] = {(uint32_t)u, (uint32_t)(u >> 32), i, r};
                    uint32_t w[4];
                    orc_philox4x32_10(ctr, key, w);
                    uint64_t v = mulhi64(((uint64_t)w[1] << 32) | w[0], u);
                    int64_t cand;
                    if ((uint64_t)w[2] < pth) {
                        cand = (int64_t)v;
                    } else {
                        uint32_t k = (uint32_t)(((uint64_t)w[3] * d) >> 32);
                        cand = G[v * d + k];
                    }
                    int dup = 0;
                    for (uint32_t j = 0; j < i; ++j)
                        if (row[j] == cand) { dup = 1; break; }
                    if (!dup) { row[i] = cand; break; }
                    ++retries;
                }
            }
        }
    } else {
        /* The reference's own draw sequence: one global MT19937-64 stream with
         * its default seed, R = U % Z then coin = U53 * 2^-53, for every try. */
        mt64 m;
        mt64_seed(&m, seed);
        for (uint64_t u = (uint64_t)d + 1; u < n; ++u) {
            int64_t *row = G + u * d;
            const uint64_t Z = (uint64_t)d * u;
            for (uint32_t i = 0; i < d; ++i) {
                for (;;) {
                    uint64_t R = mt64_next(&m) % Z;
                    double coin = (double)(mt64_next(&m) >> 11) * (1.0 / 9007199254740992.0);
                    int64_t cand = coin < p ? (int64_t)(R / d) : G[R];
                    int dup = 0;
                    for (uint32_t j = 0; j < i; ++j)
                        if (row[j] == cand) { dup = 1; break; }
                    if (!dup) { row[i] = cand; break; }
                    ++retries;
                }
            }
        }
    }
    if (retries_out) *retries_out = retries;
    return 0;
}

/*
 * Repeated-nodes Barabasi-Albert (the reference's -A sba,
 * src/PA/SPA/SerialBA.cpp:68-186): node u picks d distinct targets uniformly
 * from the endpoint list of all earlier edges -- the seed block (node i < d
 * repeated 2d times) followed, per node w = d, d+1, ..., by [target_0, w,
 * target_1, w, ...] -- so a draw is R uniform in [0, Z_u), Z_u = 2d^2 +
 * 2d(u - d), decoded as: R < 2d^2 -> node R / 2d; else r = R - 2d^2, w = d +
 * r / 2d, q = r % 2d -> q odd: w itself, q even: the target in slot q/2 of w.
 * Node d's targets are 0..d-1 (the reference's initial set), which is the
 * STAR_REF seed row.  PHILOX: R = mulhi64(w1:w0, Z_u) of
 * Philox(ctr = (u_lo, u_hi, i, r)); MT_REF: R = U % Z_u from the reference's
 * MT19937-64 stream, one draw per try, nodes in order.
 */
static int64_t ba_endpoint(uint64_t R, uint32_t d, const int64_t *G)
{
    const uint64_t seed_block = 2ull * d * d;
    if (R < seed_block) return (int64_t)(R / (2ull * d));
    const uint64_t r = R - seed_block;
    const uint64_t w = d + r / (2ull * d);
    const uint64_t q = r % (2ull * d);
    return (q & 1) ? (int64_t)w : G[w * d + q / 2];
}

int orc_generate_ba(uint64_t n, uint32_t d, uint64_t seed, int rng, int64_t *G,
                    uint64_t *retries_out)
{
    if (d == 0 || n < (uint64_t)d + 1 || G == NULL) return -1;
    if (rng != ORC_RNG_PHILOX && rng != ORC_RNG_MT_REF) return -1;
    for (uint64_t v = 0; v <= d; ++v)
        for (uint32_t k = 0; k < d; ++k) G[v * d + k] = seed_slot(v, k, d, ORC_SEED_STAR_REF);
    uint64_t retries = 0;
    const uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    mt64 m;
    mt64_seed(&m, seed);
    for (uint64_t u = (uint64_t)d + 1; u < n; ++u) {
        int64_t *row = G + u * d;
        const uint64_t Z = 2ull * d * d + 2ull * d * (u - d);
        for (uint32_t i = 0; i < d; ++i) {
            for (uint32_t r = 0;; ++r) {
                uint64_t R;
                if (rng == ORC_RNG_PHILOX) {
                    const uint32_t ctr[4] = {(uint32_t)u, (uint32_t)(u >> 32), i, r};
                    uint32_t w[4];
                    orc_philox4x32_10(ctr, key, w);
                    R = mulhi64(((uint64_t)w[1] << 32) | w[0], Z);
                } else {
                    R = mt64_next(&m) % Z;
                }
                const int64_t cand = ba_endpoint(R, d, G);
                int dup = 0;
                for (uint32_t j = 0; j < i; ++j)
                    if (row[j] == cand) { dup = 1; break; }
                if (!dup) { row[i] = cand; break; }
                ++retries;
            }
        }
    }
    if (retries_out) *retries_out = retries;
    return 0;
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
