// pa_internal.h -- declarations shared by the library's translation units.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "cuppa_pa.h"

namespace pa {

// Control block at the head of the generation scratch.  Cleared before every
// launch.  The tile ticket (the hottest atomic) has a 128-byte line of its own;
// the watermark, the device status and the counters share the next one.
struct GenCtl {
    unsigned long long ticket;   // next chunk of tiles to claim
    unsigned long long pad0[15];
    unsigned long long water;    // superblocks [0, water) are complete and visible
    unsigned long long retries;  // rejected draws
    unsigned long long waits;    // resolve iterations that made no progress
    unsigned long long tiles;    // tiles completed
    unsigned long long pending_reads;  // copy reads whose source tile was not yet known complete
    unsigned long long pending_polls;  // flag polls that found the source tile unfinished
    uint32_t error;              // pa_status raised on the device
    uint32_t trace_count;        // progress samples written
    unsigned long long t_start;  // globaltimer at the watermark warp's start
};
static_assert(sizeof(GenCtl) == 192, "GenCtl layout");

// Read-mostly copies of the watermark and the device status, one 128-byte line
// each; a warp reads copy (warp id mod kReps), so waiting warps spread their
// polls over kReps L2 lines instead of one.
struct GenRep {
    unsigned long long water;
    uint32_t error;
    uint32_t pad[29];
};
static_assert(sizeof(GenRep) == 128, "GenRep layout");
constexpr uint32_t kReps = 16;
constexpr uint64_t kRepOffset = 256;                        // replicas after GenCtl
constexpr uint64_t kCtlBytes = kRepOffset + kReps * 128;    // flags start here
constexpr uint32_t kSbTiles = 64;    // tiles per superblock (watermark granularity)
constexpr uint32_t kClaimTilesAuto = 4;  // default tiles claimed by one ticket
constexpr uint32_t kTraceMax = 2048; // progress samples kept per generation
// the start kernel's claim counters: 8, a 128-byte line each
constexpr uint64_t kStartAreaBytes = 1024;

// Warp passes per start tile, the start kernel's unit of work.
constexpr int kStartPasses = 4;

// Resolved launch geometry of one generation.
struct GenPlan {
    uint32_t id_bytes;      // 4 or 8
    uint32_t groups;        // nodes per warp pass (32 / d)
    uint32_t passes;        // passes per tile
    uint32_t tile_nodes;    // groups * passes
    uint64_t u_first;       // d + 1
    uint64_t n_tiles;
    uint64_t n_sb;          // superblocks of kSbTiles tiles
    uint64_t sb_offset;     // byte offset of the superblock counters in the scratch
    uint64_t trace_offset;  // byte offset of the progress trace in the scratch
    uint64_t start_offset;  // byte offset of the start kernel's counters
    uint64_t start_tiles;   // start tiles of the start region
    uint64_t u_split;       // nodes [u_first, u_split) are the start kernel's
    uint32_t claim_tiles;   // tiles (or start tiles) per claim-counter atomic
    uint64_t seed_edges;
    uint64_t n_edges;
    uint64_t pth;           // direct threshold
    uint32_t model;         // PA_MODEL_*
    bool slots;             // PA_LAYOUT_SLOTS: targets only, seed rows implied
    bool wide;              // d > 32: the wide kernel (pa_wide.cu) generates every node
    uint64_t edges_bytes;
    uint64_t scratch_bytes;
    uint64_t spin_limit_ns;
};

// Thread-local record of the last CUDA error behind a PA_ERR_CUDA / PA_ERR_OOM.
int set_cuda_error(cudaError_t e);

int make_plan(const pa_params *prm, GenPlan *plan);

// Start region of a graph: nodes [u_first, u_split) with u_split - u_first the
// smallest whole number of superblocks covering `want` nodes, capped at n.
uint64_t start_split(uint64_t n, uint64_t u_first, uint64_t sb_nodes, uint64_t want);

// Default start region: every node up to the start kernel's limit of 2^31 (the
// start kernel, with the memset of its region, outran the persistent kernel at
// every size measured on B200; the persistent kernel takes nodes beyond).
constexpr uint64_t kStartNodesAuto = 1ull << 31;

// Launch the generator kernel on `stream` into caller memory; scratch must hold
// plan.scratch_bytes and is cleared here.
// Queue the CSR build of a generated graph on s without waiting; the device
// error word is at d_scratch + *err_offset once the stream has run it.
int csr_enqueue(const pa_params *prm, const void *d_edges, int64_t *d_rowptr, void *d_col,
                void *d_scratch, uint64_t scratch_bytes, cudaStream_t s, uint64_t *err_offset);

// The all-ones region of a generation (byte offset and length in the edge
// buffer), and a fill of it on a small grid (pa_fill).
void fill_region(const pa_params &prm, const GenPlan &plan, uint64_t *off, uint64_t *len);
int fill_prefill(const pa_params *prm, const GenPlan &plan, void *d_edges, cudaStream_t s);

int launch_generate(const pa_params *prm, const GenPlan &plan, void *d_edges, void *d_scratch,
                    cudaStream_t stream, uint32_t blocks_override,
                    const cudaEvent_t *events = nullptr);

}  // namespace pa
