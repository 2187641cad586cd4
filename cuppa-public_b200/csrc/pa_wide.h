// pa_wide.h -- generation and row ranking for nodes with more than 32 edges
// (pa_wide.cu).
#pragma once

#include "pa_gen_core.cuh"

namespace pa {
namespace gen {

// Largest d: the reference's EdgeIndexType is an int16 (src/Common/DataTypes.h:11-28).
constexpr uint32_t kWideMaxD = 32767;
// Largest d whose rows the canonicalisation and the CSR out part rank (one
// row of ids per warp in shared memory).
constexpr uint32_t kWideRankMaxD = 4096;
// Shared memory of one block's hash sets / row copies, and the most one warp's
// set may take while it can still be at most half full.
constexpr size_t kWideBlockSetBytes = 64 * 1024;
constexpr uint32_t kWideSetMaxBytes = 128 * 1024;

// Generate nodes [a.u_first, a.start_end) of a graph with d > 32 into caller
// memory whose slots of those nodes hold all-ones; *ticket must be zero.  Also
// writes the seed edges (PAIRS).  `blocks` 0 = one wave.
int launch_wide(uint32_t id_bytes, bool slots, const GenArgs &a, unsigned long long *ticket,
                uint32_t blocks, cudaStream_t s);
// Canonical rows (out may equal E) and CSR out parts of a PAIRS graph with
// 32 < d <= kWideRankMaxD (PA_ERR_NOT_SUPPORTED above).
int canon_wide(uint32_t id_bytes, const void *E, void *out, uint64_t n, uint32_t d,
               uint64_t seed_edges, cudaStream_t s);
int csr_out_wide(uint32_t id_bytes, const void *E, const int64_t *rowptr, void *col, uint64_t n,
                 uint32_t d, uint64_t seed_edges, uint64_t col_len, cudaStream_t s);

}  // namespace gen
}  // namespace pa
