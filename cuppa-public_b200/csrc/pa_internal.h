// pa_internal.h -- declarations shared by the library's translation units.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "cuppa_pa.h"

namespace pa {

// Control block at the head of the generation scratch.  Cleared before every
// launch; the kernel's tile ticket, completion watermark, counters and device
// status live here.
struct GenCtl {
    unsigned long long ticket;   // next tile to claim
    unsigned long long water;    // tiles [0, water) are complete and visible
    unsigned long long retries;  // rejected draws
    unsigned long long waits;    // resolve iterations that made no progress
    unsigned long long tiles;    // tiles completed
    uint32_t error;              // pa_status raised on the device
    uint32_t pad;
    unsigned long long reserved[2];
};
static_assert(sizeof(GenCtl) == 64, "GenCtl layout");

constexpr uint64_t kCtlBytes = 256;  // flags start 256 B into the scratch

// Resolved launch geometry of one generation.
struct GenPlan {
    uint32_t id_bytes;      // 4 or 8
    uint32_t groups;        // nodes per warp pass (32 / d)
    uint32_t passes;        // passes per tile
    uint32_t tile_nodes;    // groups * passes
    uint64_t u_first;       // d + 1
    uint64_t n_tiles;
    uint64_t seed_edges;
    uint64_t n_edges;
    uint64_t pth;           // direct threshold
    uint64_t edges_bytes;
    uint64_t scratch_bytes;
    uint64_t spin_limit_ns;
};

// Thread-local record of the last CUDA error behind a PA_ERR_CUDA / PA_ERR_OOM.
int set_cuda_error(cudaError_t e);

int make_plan(const pa_params *prm, GenPlan *plan);

// Launch the generator kernel on `stream` into caller memory; scratch must hold
// plan.scratch_bytes and is cleared here.
int launch_generate(const pa_params *prm, const GenPlan &plan, void *d_edges, void *d_scratch,
                    cudaStream_t stream, uint32_t blocks_override);

}  // namespace pa
