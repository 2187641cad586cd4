/*
 * pa_oracle.h -- CPU oracle for the copy-model preferential-attachment generator.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is loaded by the
 * tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, and by
 * nothing else.  The product library (libcuppa_pa.so) never links or calls it.
 *
 * What it restates (reference paths are relative to the cuPPA-Public tree):
 *   - the sequential copy model of src/PA/SPA/SerialCopyModel3.cpp:38-78
 *     (per-node order u = M+1..N-1, slot order j = 0..M-1, redraw until the
 *     candidate is not already among the node's earlier slots -- the unique
 *     insert of src/Graph/Vertex/CPU/BSTVertex.h:189-238);
 *   - the reference seed graph ("M disjoint self-slots + star node M") of
 *     SerialCopyModel3.cpp:38-49 == src/PA/cuPPA/cuPPA_RRP.cu:57-73, and the
 *     (d+1)-clique seed that the benchmark configurations ask for;
 *   - two random-number front ends:
 *       PHILOX   Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 *                numbers: as easy as 1, 2, 3", SC'11) keyed (seed) with counter
 *                (u_lo, u_hi, slot, retry) -- the bit-exact contract of the GPU
 *                generator;
 *       MT_REF   MT19937-64 (Matsumoto & Nishimura, published algorithm) with the
 *                reference's default seed 5489 and its draw order
 *                R = U64 % (M*u), coin = (U64 >> 11) * 2^-53
 *                (src/Common/Random64.hpp:64-114, SerialCopyModel3.cpp:62-74).
 *                This mode reproduces the reference `-A scm` run exactly and so
 *                pins the copy-model semantics shared with PHILOX mode.
 *   - the degree distribution of src/PA/SPA/PAHelper.hpp:15-67 and
 *     src/PA/cuPPA/cuPPA.cu:103-165, the edge text of PAHelper.hpp:163-177, and
 *     an undirected CSR with sorted rows.
 */
#ifndef PA_ORACLE_H_
#define PA_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_SEED_STAR_REF = 0, ORC_SEED_CLIQUE = 1 };
enum { ORC_RNG_PHILOX = 0, ORC_RNG_MT_REF = 1 };

/* Philox4x32-10 block function: out = philox(ctr, key). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* MT19937-64: seed then draw `count` outputs into out. */
void orc_mt19937_64(uint64_t seed, uint64_t count, uint64_t *out);

/* p -> 33-bit threshold: a slot is direct iff (uint64)w2 < thresh. */
uint64_t orc_p_threshold(double p);

/* Number of canonical edges contributed by the seed rows 0..d. */
uint64_t orc_seed_edge_count(uint32_t d, int seed_mode);

/* Total canonical edges: seed edges + (n-d-1)*d. */
uint64_t orc_edge_count(uint64_t n, uint32_t d, int seed_mode);

/*
 * Generate the slot array G[n][d] (row-major, generation order).
 * Returns 0 on success, -1 on invalid arguments.  retries_out (may be NULL)
 * receives the number of rejected draws.
 */
int orc_generate(uint64_t n, uint32_t d, double p, uint64_t seed, int seed_mode,
                 int rng, int64_t *G, uint64_t *retries_out);

/*
 * The repeated-nodes Barabasi-Albert model (the reference's -A sba,
 * src/PA/SPA/SerialBA.cpp:68-186) in the same slot array: STAR_REF seed rows,
 * then node u's d distinct targets drawn uniformly from the endpoints of all
 * earlier edges.  rng as for orc_generate (MT_REF: the reference's own stream).
 */
int orc_generate_ba(uint64_t n, uint32_t d, uint64_t seed, int rng, int64_t *G,
                    uint64_t *retries_out);

/*
 * Edge list in the GPU generator's PAIRS layout: the canonical seed edges
 * (u > v, sorted), then rows d+1..n-1 in slot (generation) order.
 * pairs has 2*orc_edge_count() entries (src, dst interleaved).
 */
void orc_pairs_slot_order(uint64_t n, uint32_t d, int seed_mode, const int64_t *G,
                          int64_t *pairs);

/* Canonical edge list: every (u, v) with v < u, sorted by (u, v). */
void orc_pairs_canonical(uint64_t n, uint32_t d, int seed_mode, const int64_t *G,
                         int64_t *pairs);

/* Undirected degree of every node over the canonical edges. */
void orc_degrees(uint64_t n, uint32_t d, int seed_mode, const int64_t *G, int64_t *deg);

/*
 * Undirected CSR with each edge in both rows and every row sorted ascending.
 * rowptr has n+1 entries, col has 2*orc_edge_count() entries.
 */
void orc_csr(uint64_t n, uint32_t d, int seed_mode, const int64_t *G, int64_t *rowptr,
             int64_t *col);

/*
 * Position-keyed digest of an id array: acc[0] += h, acc[1] ^= h over
 * h = fmix64(fmix64(pos * 0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019) ^ x) for every
 * element x at pos = index_base + i (fmix64: MurmurHash3's finalizer).  The
 * digest of a concatenation is the sum / xor of the digests of its parts with
 * their index bases, so it can be taken chunk by chunk; swapping two elements
 * changes it.  acc is accumulated into, not cleared.
 */
void orc_digest_ids(const int64_t *x, uint64_t count, uint64_t index_base, uint64_t acc[2]);

enum { ORC_MODEL_COPY = 0, ORC_MODEL_BA = 1 };

/*
 * Whole-graph digests of a Philox-mode graph of n <= 2^31 nodes, generated with
 * int32 slot storage (n*d*4 bytes of host memory, plus 8*(n+1) with CSR):
 *   out[0..1]  the PAIRS slot-order edge list as one flat id array
 *              (src of edge e at 2e, dst at 2e+1);
 *   out[2..3]  the undirected CSR's rowptr[0..n];
 *   out[4..5]  the CSR's col[0..2E) (out[2..5] stay zero unless with_csr);
 *   out[6]     the number of rejected draws.
 * model: ORC_MODEL_COPY (seed_mode as given) or ORC_MODEL_BA (STAR_REF seed).
 * Returns 0, -1 on invalid arguments, -2 when host memory runs out.
 */
int orc_graph_digests(uint64_t n, uint32_t d, double p, uint64_t seed, int seed_mode, int model,
                      int with_csr, uint64_t out[7]);

/* 64-bit FNV-1a over a byte buffer (fixture digests). */
uint64_t orc_fnv1a64(const void *data, uint64_t bytes);

#ifdef __cplusplus
}
#endif

#endif /* PA_ORACLE_H_ */
