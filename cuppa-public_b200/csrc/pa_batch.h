// pa_batch.h -- host side of a batch launch, shared by pa_batch_generate and
// the request server: plan the scratch layout, write the device image of the
// instance and level tables into host memory, and enqueue the launches.
#pragma once

#include <vector>

#include "pa_gen_core.cuh"

namespace pa {

// Level tables of one launch over a set of instances (host copies and their
// offsets in the scratch).
struct BatchLevels {
    uint32_t levels = 0;
    std::vector<unsigned long long> lvl, ibase, lstart;
    uint64_t lvl_off = 0, ibase_off = 0, lstart_off = 0;
};

struct BatchJob {
    uint32_t count = 0, passes = 0, id_bytes = 0, claim_tiles = 0;
    std::vector<GenPlan> plans;
    std::vector<uint64_t> flags_off, sb_off;
    BatchLevels start, tail;
    uint64_t image_off = 0, image_bytes = 0;   // scratch bytes copied from the host image
    uint64_t table_off = 0, ticket_off = 0, scratch_bytes = 0;
    uint64_t max_start_pairs = 0;       // the largest start region (fill launch size)
    gen::GenArgs first{};                      // instance 0 (the start kernel's count == 1 path)
};

// Validate prms and lay out the scratch (J.scratch_bytes, J.image_bytes).
int batch_prepare(const pa_params *prms, uint32_t count, BatchJob &J);
// Write the image (J.image_bytes) for these edge buffers and this scratch.
int batch_bind(BatchJob &J, const pa_params *prms, void *const *d_edges, const uint64_t *edges_bytes,
               void *d_scratch, unsigned char *image);
// Queue the launches on s.  `image` must stay readable until the copy from it
// has run (pinned memory stays valid; pageable memory needs a synchronize).
int batch_enqueue(const BatchJob &J, void *d_scratch, const void *image, cudaStream_t s);

}  // namespace pa
