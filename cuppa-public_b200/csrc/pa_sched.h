// pa_sched.h -- lane-aware admission used by the request server (the C ABI's
// pa_sched_submit / pa_sched_admit are the single-lane case: every request in
// lane 0, every lane admitting).
#pragma once

#include <cstdint>

#include "cuppa_pa.h"

namespace pa {

// Queue a request in `lane` (0..31).
int sched_submit_lane(pa_sched *q, uint64_t ticket, uint64_t bytes, uint64_t now_ns, uint32_t lane);
// Admit up to cap requests of the lanes in lane_mask, in arrival order; other
// lanes' requests are skipped, and an aged request that does not fit stops the
// admission of its own lane only.
uint32_t sched_admit_lanes(pa_sched *q, uint64_t now_ns, uint64_t *out, uint32_t cap,
                           uint32_t lane_mask);

}  // namespace pa
