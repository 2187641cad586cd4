// pa_generate.cu -- the copy-model generator kernel (one persistent launch).
//
// Replaces the reference's staged driver and its per-stage kernels
// (src/PA/cuPPA/cuPPA_1.cu:112-226 launching generate_graph_rrp_by_batch,
// src/PA/cuPPA/cuPPA_RRP_1.cu:29-209, with the per-thread curand state of
// src/Common/cuRandom.cu:47-52 and the global-memory BST of
// src/Graph/Vertex/CUDA/cuBSTVertex.cuh:153-319).
//
// Semantics (identical to the sequential model of
// src/PA/SPA/SerialCopyModel3.cpp:52-78 with Philox draws): for node
// u = d+1..n-1 and slot i = 0..d-1, try r = 0, 1, ... with
//   (v, k, direct) = draw(seed; u, i, r),  cand = direct ? v : G[v][k],
// and keep the first candidate that is not among G[u][0..i-1].
//
// Why any schedule gives the same bits: slot (u,i) depends only on its own
// draws, on the final values of u's slots 0..i-1, and on final values G[v][k]
// with v < u.  The kernel therefore computes each slot from final inputs only:
//
//  * Work unit: a warp claims a tile of `tile_nodes` consecutive nodes from a
//    global ticket (tiles are claimed in increasing order).  A warp pass covers
//    G = 32/d nodes: lane L owns slot L%d of node L/d.
//  * Phase A draws retry 0 for every slot of the tile and issues the copy-target
//    loads whose source tile is already complete, so one tile keeps up to
//    32*passes loads in flight per warp.
//  * Phase B resolves pass by pass.  The duplicate set of a node is its d lanes:
//    __match_any_sync finds equal candidates, and a lane is final once every
//    lane at or below it in its group is known and unique.  A lane whose
//    candidate equals a final lane's value is rejected for certain and redraws
//    (r+1) at once.  Copy targets inside the tile come from a shared-memory copy
//    of the tile's finished passes (or by shuffle from the same pass); targets in
//    other tiles come from global memory once that tile's completion flag is set.
//  * Publication: after its stores the warp fences, sets its tile flag with a
//    release store and advances the completion watermark; readers acquire the
//    flag (or the watermark) before loading a slot.
//  * Deadlock freedom: a node waits only on smaller nodes; tiles are claimed in
//    order by running warps, so the smallest unfinished tile never waits on an
//    unfinished one.  Every wait is bounded by spin_limit_ns (globaltimer); on
//    expiry the warp records PA_ERR_SPIN_TIMEOUT and returns, and every other
//    warp returns when it sees the error word.
//  * Output: (u, target) pairs.  int64 ids: one 128-bit store per lane; int32
//    ids: two adjacent lanes' pairs in one 128-bit store.
#include <cstdio>
#include <mutex>

#include "pa_device.cuh"
#include "pa_internal.h"

namespace pa {

namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kThreads = 256;

enum : uint32_t { ST_KNOWN = 0, ST_PEND_GLOBAL = 1, ST_PEND_TILE = 2 };

struct GenArgs {
    void *edges;
    GenCtl *ctl;
    uint32_t *flags;
    uint64_t n;
    uint64_t u_first;
    uint64_t n_tiles;
    uint64_t seed_edges;
    uint64_t pth;
    uint64_t spin_limit_ns;
    uint32_t key0, key1;
    uint32_t d;
    uint32_t groups;
    uint32_t tile_nodes;
    uint32_t seed_mode;
    uint32_t withhold_first;   // test-only: never publish tile 0
};

// e-th canonical seed edge.
__device__ __forceinline__ void seed_edge(uint64_t e, uint32_t d, uint32_t mode, uint64_t &src,
                                          uint64_t &dst)
{
    if (mode == 1) {  // clique: rows v = 1..d hold (v, 0..v-1)
        uint64_t v = 1, base = 0;
        while (base + v <= e) { base += v; ++v; }
        src = v;
        dst = e - base;
    } else {          // star node d -> 0..d-1
        src = d;
        dst = e;
    }
}

template <typename Id>
__device__ __forceinline__ const Id *slot_addr(const Id *E, const GenArgs &a, uint64_t v, uint32_t k)
{
    return E + 2 * (a.seed_edges + (v - a.u_first) * a.d + k) + 1;
}

// Per-slot resolution state held in registers.
struct Slot {
    uint64_t val;   // candidate value, or the pending source node v
    uint32_t st;    // ST_*
    uint32_t kr;    // retry << 8 | k
};

// Where the candidate of a fresh draw comes from.
template <typename Id>
__device__ __forceinline__ void classify(Slot &s, const Draw &dr, uint32_t r, const GenArgs &a,
                                         const Id *E, uint64_t tb, uint64_t water_node)
{
    s.kr = (r << 8) | dr.k;
    if (dr.direct) {
        s.val = dr.v;
        s.st = ST_KNOWN;
    } else if (dr.v <= a.d) {
        s.val = seed_slot(dr.v, dr.k, a.d, a.seed_mode);
        s.st = ST_KNOWN;
    } else if (dr.v < tb) {
        if (dr.v < water_node) {
            s.val = ld_slot(slot_addr(E, a, dr.v, dr.k));
            s.st = ST_KNOWN;
        } else {
            s.val = dr.v;
            s.st = ST_PEND_GLOBAL;
        }
    } else {
        s.val = dr.v;
        s.st = ST_PEND_TILE;
    }
}

// Resolve the slots of one warp pass until every active lane is final.
// Returns false when the warp must stop (wait limit, or another warp failed).
template <typename Id>
__device__ __forceinline__ bool resolve_pass(Slot &s, const GenArgs &a, const Id *E,
                                             const Id *tilebuf, uint64_t tb, uint64_t pbase,
                                             uint32_t pass_off, uint64_t u, bool active,
                                             uint32_t slot, uint32_t lane, uint32_t gmask,
                                             uint32_t lt, uint32_t le, uint64_t &water_node,
                                             unsigned long long &n_retry,
                                             unsigned long long &n_wait)
{
    const uint32_t d = a.d;
    uint64_t spin_t0 = 0;
    for (;;) {
        bool changed = false;
        const uint32_t k = s.kr & 0xffu;
        if (active && s.st == ST_PEND_GLOBAL) {
            const uint64_t v = s.val;
            bool ready = v < water_node;
            if (!ready) ready = ld_acquire_u32(a.flags + (v - a.u_first) / a.tile_nodes) != 0u;
            if (ready) {
                s.val = ld_slot(slot_addr(E, a, v, k));
                s.st = ST_KNOWN;
                changed = true;
            }
        } else if (active && s.st == ST_PEND_TILE) {
            const uint64_t off = s.val - tb;
            if (off < (uint64_t)pass_off) {   // a finished earlier pass of this tile
                s.val = (uint64_t)tilebuf[off * d + k];
                s.st = ST_KNOWN;
                changed = true;
            }
        }

        const bool known = active && s.st == ST_KNOWN;
        const unsigned long long key =
            known ? (unsigned long long)s.val : (0x8000000000000000ull | lane);
        const uint32_t eq = __match_any_sync(kFull, key);
        const bool bad = active && (!known || (eq & lt & gmask) != 0u);
        const uint32_t badm = __ballot_sync(kFull, bad);
        const bool fin = active && (badm & gmask & le) == 0u;
        const uint32_t finm = __ballot_sync(kFull, fin || !active);
        if (finm == kFull) return true;

        // Copy targets in this same pass: take the source lane's value once
        // that lane is final.
        const bool same = active && s.st == ST_PEND_TILE && s.val >= pbase;
        const uint32_t src = same ? (uint32_t)((s.val - pbase) * d + k) : lane;
        const uint64_t sv = __shfl_sync(kFull, s.val, src);
        if (same && ((finm >> src) & 1u)) {
            s.val = sv;
            s.st = ST_KNOWN;
            changed = true;
        }

        // A candidate equal to a final lower slot is rejected for certain.
        if (known && !fin && (eq & lt & gmask & finm) != 0u) {
            const uint32_t r = (s.kr >> 8) + 1u;
            classify(s, draw_slot(u, slot, r, a.key0, a.key1, a.pth, d), r, a, E, tb, water_node);
            changed = true;
            ++n_retry;
        }

        if (!__any_sync(kFull, changed)) {
            // Nothing moved: every open slot waits on another tile.
            unsigned long long now = 0, err = 0, w2 = 0;
            if (lane == 0) {
                now = globaltimer_ns();
                err = ld_relaxed_u32(&a.ctl->error);
                w2 = ld_acquire_u64(&a.ctl->water);
                ++n_wait;
            }
            now = __shfl_sync(kFull, now, 0);
            err = __shfl_sync(kFull, err, 0);
            w2 = __shfl_sync(kFull, w2, 0);
            __syncwarp();
            water_node = a.u_first + w2 * a.tile_nodes;
            if (spin_t0 == 0) spin_t0 = now;
            if (err != 0) return false;
            if (now - spin_t0 > a.spin_limit_ns) {
                if (lane == 0) atomicCAS(&a.ctl->error, 0u, (uint32_t)PA_ERR_SPIN_TIMEOUT);
                return false;
            }
            __nanosleep(100);
        } else {
            spin_t0 = 0;
        }
    }
}

template <typename Id, int P>
__global__ void __launch_bounds__(kThreads) gen_kernel(const GenArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t warp = threadIdx.x >> 5;
    Id *tilebuf = reinterpret_cast<Id *>(smem_raw) + warp * (32u * P);
    Id *E = reinterpret_cast<Id *>(a.edges);

    const uint32_t d = a.d;
    const uint32_t G = a.groups;
    const uint32_t g = lane / d;
    const uint32_t slot = lane - g * d;
    const bool lane_used = lane < G * d;
    const uint32_t gmask =
        lane_used ? (d == 32 ? kFull : (((1u << d) - 1u) << (g * d))) : 0u;
    const uint32_t lt = lanemask_lt();
    const uint32_t le = lt | (1u << lane);

    if (blockIdx.x == 0 && warp == 0) {
        for (uint64_t e = lane; e < a.seed_edges; e += 32) {
            uint64_t s, t;
            seed_edge(e, d, a.seed_mode, s, t);
            st_pair(E + 2 * e, s, t);
        }
    }

    unsigned long long n_retry = 0, n_wait = 0, n_done = 0;
    bool ok = true;

    while (ok) {
        unsigned long long t = 0, wt = 0;
        if (lane == 0) {
            t = atomicAdd(&a.ctl->ticket, 1ull);
            wt = ld_acquire_u64(&a.ctl->water);
        }
        t = __shfl_sync(kFull, t, 0);
        if (t >= a.n_tiles) break;
        wt = __shfl_sync(kFull, wt, 0);
        __syncwarp();  // orders lane 0's acquire before every lane's slot loads
        uint64_t water_node = a.u_first + wt * a.tile_nodes;

        const uint64_t tb = a.u_first + t * a.tile_nodes;
        const uint64_t te = min(a.n, tb + a.tile_nodes);

        // ---- Phase A: retry-0 draws and early copy loads for the whole tile.
        Slot s[P];
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const uint64_t u = tb + (uint64_t)j * G + g;
            s[j].val = 0;
            s[j].st = ST_KNOWN;
            s[j].kr = 0;
            if (lane_used && u < te)
                classify(s[j], draw_slot(u, slot, 0, a.key0, a.key1, a.pth, d), 0u, a, E, tb,
                         water_node);
        }

        // ---- Phase B: resolve and store pass by pass.
#pragma unroll
        for (int j = 0; j < P; ++j) {
            const uint64_t pbase = tb + (uint64_t)j * G;   // first node of the pass
            const uint64_t u = pbase + g;
            const bool active = lane_used && u < te;
            if (ok)
                ok = resolve_pass(s[j], a, E, tilebuf, tb, pbase, (uint32_t)j * G, u, active, slot,
                                  lane, gmask, lt, le, water_node, n_retry, n_wait);
            if (ok) {
                // Finished pass: keep it for in-tile copy reads, then emit the edges.
                if (active) tilebuf[(uint32_t)j * G * d + lane] = (Id)s[j].val;
                __syncwarp();
                const uint64_t e0 = a.seed_edges + (pbase - a.u_first) * d;
                if constexpr (sizeof(Id) == 8) {
                    if (active) st_pair(E + 2 * (e0 + lane), u, s[j].val);
                } else {
                    const uint32_t nu = __shfl_down_sync(kFull, (uint32_t)u, 1);
                    const uint32_t nv = __shfl_down_sync(kFull, (uint32_t)s[j].val, 1);
                    const uint32_t na = __shfl_down_sync(kFull, (uint32_t)active, 1);
                    const bool leader = ((lane + (uint32_t)(e0 & 1u)) & 1u) == 0u;
                    if (active) {
                        Id *p = E + 2 * (e0 + lane);
                        if (leader) {
                            if (lane < 31u && na) st_pair2(p, u, s[j].val, nu, nv);
                            else st_pair(p, u, s[j].val);
                        } else if (lane == 0) {
                            st_pair(p, u, s[j].val);
                        }
                    }
                }
            }
        }
        if (!ok) break;

        // ---- Publish the tile.
        __threadfence();
        __syncwarp();
        if (lane == 0 && !(a.withhold_first && t == 0)) {
            st_release_u32(a.flags + t, 1u);
            unsigned long long w = ld_acquire_u64(&a.ctl->water);
            const unsigned long long w0 = w;
            while (w < a.n_tiles && ld_acquire_u32(a.flags + w) != 0u) ++w;
            if (w > w0) red_max_release_u64(&a.ctl->water, w);
        }
        ++n_done;
    }

    // Warp totals, one atomic each.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) n_retry += __shfl_down_sync(kFull, n_retry, o);
    if (lane == 0) {
        if (n_retry) atomicAdd(&a.ctl->retries, n_retry);
        if (n_wait) atomicAdd(&a.ctl->waits, n_wait);
        if (n_done) atomicAdd(&a.ctl->tiles, n_done);
    }
}

template <typename Id, int P>
int launch_one(const GenArgs &args, uint32_t blocks, cudaStream_t stream)
{
    auto kern = gen_kernel<Id, P>;
    const size_t smem = (size_t)(kThreads / 32) * 32 * P * sizeof(Id);
    if (blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)kThreads, smem);
        if (e != cudaSuccess) return set_cuda_error(e);
        blocks = (uint32_t)(sms * (per_sm > 0 ? per_sm : 1));
    }
    kern<<<blocks, kThreads, smem, stream>>>(args);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

}  // namespace

int launch_generate(const pa_params *prm, const GenPlan &plan, void *d_edges, void *d_scratch,
                    cudaStream_t stream, uint32_t blocks_override)
{
    cudaError_t e = cudaMemsetAsync(d_scratch, 0, plan.scratch_bytes, stream);
    if (e != cudaSuccess) return set_cuda_error(e);

    GenArgs a;
    a.edges = d_edges;
    a.ctl = reinterpret_cast<GenCtl *>(d_scratch);
    a.flags = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(d_scratch) + kCtlBytes);
    a.n = prm->n;
    a.u_first = plan.u_first;
    a.n_tiles = plan.n_tiles;
    a.seed_edges = plan.seed_edges;
    a.pth = plan.pth;
    a.spin_limit_ns = plan.spin_limit_ns;
    a.key0 = (uint32_t)prm->seed;
    a.key1 = (uint32_t)(prm->seed >> 32);
    a.d = prm->d;
    a.groups = plan.groups;
    a.tile_nodes = plan.tile_nodes;
    a.seed_mode = prm->seed_mode;
    a.withhold_first = (prm->flags & PA_FLAG_TEST_WITHHOLD_FIRST_TILE) ? 1u : 0u;

    const uint32_t blocks = blocks_override ? blocks_override : prm->blocks;
    if (plan.id_bytes == 8) {
        switch (plan.passes) {
        case 1: return launch_one<int64_t, 1>(a, blocks, stream);
        case 2: return launch_one<int64_t, 2>(a, blocks, stream);
        case 4: return launch_one<int64_t, 4>(a, blocks, stream);
        case 8: return launch_one<int64_t, 8>(a, blocks, stream);
        }
    } else {
        switch (plan.passes) {
        case 1: return launch_one<int32_t, 1>(a, blocks, stream);
        case 2: return launch_one<int32_t, 2>(a, blocks, stream);
        case 4: return launch_one<int32_t, 4>(a, blocks, stream);
        case 8: return launch_one<int32_t, 8>(a, blocks, stream);
        }
    }
    return PA_ERR_INVALID;
}

}  // namespace pa
