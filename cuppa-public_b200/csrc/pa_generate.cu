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
// with v < u.  The kernel computes each slot from final inputs only:
//
//  * Work unit: a warp claims a tile of `tile_nodes` consecutive nodes from a
//    global ticket (tiles are claimed in increasing order).  A warp pass covers
//    G = 32/d nodes: lane L owns slot L%d of node L/d.
//  * Two-stage software pipeline per warp.  Stage 1 of the next tile draws
//    retry 0 for every slot and issues the copy-target loads whose source tile
//    is already known complete; stage 2 of the current tile then consumes its
//    loads (issued one stage earlier), resolves, stores and publishes.  The
//    ticket for the tile after next is requested at the start of each stage,
//    so the claim round trip, the copy loads and the publication fence of
//    consecutive tiles overlap.  Holding claimed tiles cannot deadlock: each is
//    larger than the tile in hand, whose dependencies are all smaller still.
//  * Resolution: the duplicate set of a node is its d lanes.  __match_any_sync
//    finds equal candidates; a lane is final once every lane at or below it in
//    its group is known and unique.  A lane whose candidate equals a final
//    lane's value is rejected for certain and redraws (r+1) at once.  Copy
//    targets inside the tile come from a shared-memory copy of the tile's
//    finished passes (or by shuffle from the same pass); targets in other tiles
//    come from global memory once that tile is complete.
//  * Publication: after its stores the warp passes a warp barrier, lane 0
//    issues a release fence, sets the tile's flag and adds the tile to its
//    superblock's count (64 tiles per superblock; a fire-and-forget reduction).
//    One dedicated warp (block 0, warp 0) is the only writer of the completion
//    watermark: it reads 32 superblock counts per round trip and advances over
//    the complete prefix.  Readers of a slot acquire the watermark (or, above
//    it, the source tile's flag) before loading the slot.
//  * Deadlock freedom: a node waits only on smaller nodes; tiles are claimed in
//    order by running warps, so the smallest unfinished tile never waits on an
//    unfinished one.  Every wait is bounded by spin_limit_ns (globaltimer); on
//    expiry the warp records PA_ERR_SPIN_TIMEOUT and returns, and every other
//    warp returns when it sees the error word.
//  * Node arithmetic is 32-bit when n <= 2^32 (the multiply-shift of the draw
//    and the duplicate match then take one word); stored ids keep the width
//    the caller asked for.
//  * Output: (u, target) pairs.  int64 ids: one 128-bit store per lane; int32
//    ids: two adjacent lanes' pairs in one 128-bit store.
#include <cstring>

#include "pa_gen_core.cuh"
#include "pa_wide.h"

namespace pa {

namespace {

using namespace gen;

// The single writer of the completion watermark.  Each round trip reads the
// tile counts of 128 consecutive superblocks (one 16-byte load per lane),
// advances over the complete prefix and publishes it with a release store.  It
// stops when every superblock is complete, when a worker has raised an error,
// or after spin_limit_ns without progress (the workers' own waits are bounded by
// the same limit, so a stall that long means they have stopped).
__device__ __forceinline__ void advance_watermark(const GenArgs &a, uint32_t lane)
{
    // Tiles before tile_begin were generated by the start kernel, which ran
    // before this launch: publish that prefix first.
    uint64_t w = a.water_init;
    if (lane <= kReps) st_relaxed_u64(lane < kReps ? &a.reps[lane].water : &a.ctl->water, w);
    uint64_t t0 = globaltimer_ns();
    const uint64_t t_start = t0;
    uint64_t next_sample = 0;
    uint32_t n_samples = 0;
    if (lane == 0) a.ctl->t_start = t_start;
    auto need = [&](uint64_t b) {
        return (uint32_t)min((uint64_t)kSbTiles, a.n_tiles - b * kSbTiles);
    };
    while (w < a.n_sb) {
        // The counter array is padded to a multiple of 64 entries, so the
        // 4-entry load at b0 < n_sb stays inside it.
        const uint64_t base = w & ~3ull;
        const uint64_t b0 = base + 4ull * lane;
        uint4 c = make_uint4(0, 0, 0, 0);
        if (b0 < a.n_sb) c = ld_relaxed_v4_u32(a.sbcnt + b0);
        const uint32_t cv[4] = {c.x, c.y, c.z, c.w};
        uint32_t first = 128;   // first open position (4*lane + j) at or after w
#pragma unroll
        for (int j = 3; j >= 0; --j) {
            const uint64_t b = b0 + j;
            const bool open = b >= w && (b >= a.n_sb || cv[j] != need(b));
            if (open) first = 4 * lane + j;
        }
        const uint32_t p = __reduce_min_sync(kFull, first);
        const uint64_t nw = min(base + p, a.n_sb);
        if (nw > w) {
            w = nw;
            __syncwarp();   // every lane's load before the publishing lanes' fence
            if (lane <= kReps) {
                fence_acq_rel_gpu();
                st_relaxed_u64(lane < kReps ? &a.reps[lane].water : &a.ctl->water, w);
            }
            __syncwarp();
            t0 = globaltimer_ns();
            if (w >= next_sample && n_samples < kTraceMax) {
                if (lane == 0) {
                    const uint64_t done = min(a.n, a.u_first + w * a.sb_nodes);
                    a.trace[2 * n_samples] = t0 - t_start;
                    a.trace[2 * n_samples + 1] = done;
                    a.ctl->trace_count = n_samples + 1;
                }
                ++n_samples;
                next_sample = w + a.trace_step;
            }
            continue;
        }
        uint32_t err = 0;
        if (lane == 0) err = ld_relaxed_u32(&a.ctl->error);
        err = __shfl_sync(kFull, err, 0);
        if (err != 0 || globaltimer_ns() - t0 > a.spin_limit_ns) return;
        __nanosleep(64);
    }
}

// Tiles are claimed claim_tiles at a time: one ticket names a chunk of
// consecutive tiles that the warp then takes in order.  The ticket of the next
// chunk is requested as soon as a chunk is opened, so its round trip is hidden
// behind the chunk's work.  Chunks are claimed in increasing order by running
// warps, so the ordered-claim argument for deadlock freedom still holds.
struct Claimer {
    uint64_t base;             // first tile of the open chunk
    uint32_t idx;              // next tile within it
    unsigned long long pre;    // lane 0: the chunk claimed ahead
};

__device__ __forceinline__ uint64_t claim_next(Claimer &c, const GenArgs &a, const Lane &L)
{
    if (c.idx == a.claim_tiles) {
        const uint64_t chunk = __shfl_sync(kFull, c.pre, 0);
        if (L.lane == 0) c.pre = atomicAdd(&a.ctl->ticket, 1ull);
        c.base = a.tile_begin + chunk * a.claim_tiles;
        c.idx = 0;
    }
    return c.base + c.idx++;
}

// Start gate.  Early in the graph the nodes in flight are a large share of all
// earlier nodes, so most copy reads would wait on unfinished tiles and the wait
// chains grow with the number of warps.  A tile whose first node is tb is
// therefore started only once every node below tb - max(min_window,
// tb >> window_shift) is complete: the share of copy reads that can hit an
// unfinished tile stays below 2^-window_shift, and once tb is large the gate
// never binds.  The gate cannot deadlock: the warp holding the smallest
// unstarted tile waits only for tiles below it, and those are complete or in
// stage 2, which never waits on a gate.
template <typename NodeT>
__device__ __forceinline__ bool gate_open(NodeT tb, NodeT water_node, const GenArgs &a)
{
    const uint64_t win = max(a.min_window, (uint64_t)tb >> a.window_shift);
    return (uint64_t)water_node + win >= (uint64_t)tb;
}

template <typename NodeT>
__device__ __forceinline__ bool wait_gate(NodeT tb, NodeT &water_node, const GenArgs &a,
                                          const Lane &L, uint32_t &n_wait)
{
    uint64_t t0 = 0;
    uint32_t sleep_ns = 256;
    while (!gate_open(tb, water_node, a)) {
        unsigned long long w = 0, now = 0;
        uint32_t err = 0;
        if (L.lane == 0) {
            const GenRep *rp = my_rep(a);
            w = ld_acquire_u64(&rp->water);
            now = globaltimer_ns();
            err = ld_relaxed_u32(&rp->error);
            ++n_wait;
        }
        w = __shfl_sync(kFull, w, 0);
        now = __shfl_sync(kFull, now, 0);
        err = __shfl_sync(kFull, err, 0);
        __syncwarp();
        water_node = (NodeT)(a.u_first + w * a.sb_nodes);
        if (err != 0) return false;
        if (t0 == 0) t0 = now;
        if (now - t0 > a.spin_limit_ns) {
            if (L.lane == 0) raise_error(a, (uint32_t)PA_ERR_SPIN_TIMEOUT);
            return false;
        }
        if (!gate_open(tb, water_node, a)) {
            __nanosleep(sleep_ns);
            sleep_ns = min(sleep_ns * 2u, 8192u);
        }
    }
    return true;
}

// One pipeline step: start tile t_next in `nxt`, finish tile t_cur in `cur`,
// and take the tile after next.  Returns whether `nxt` holds a tile.  When the
// start gate of `nxt` is closed the step runs in order instead: finish `cur`,
// wait at the gate, then start `nxt`.
template <typename Id, typename NodeT, int P>
__device__ __forceinline__ bool pipeline_step(Slot<NodeT> (&cur)[P], Slot<NodeT> (&nxt)[P],
                                              uint64_t t_cur, uint64_t &t_nxt_out,
                                              uint64_t &t_next, Claimer &cl, const GenArgs &a,
                                              Id *E, Id *tilebuf, const Lane &L,
                                              NodeT &water_node, uint32_t &n_retry,
                                              uint32_t &n_wait, uint32_t &n_pend,
                                              uint32_t &n_poll, uint32_t &n_done, bool &ok)
{
    unsigned long long w = 0;
    if (L.lane == 0) w = ld_acquire_u64(&my_rep(a)->water);
    const uint64_t t_nxt = t_next;
    const bool has_next = t_nxt < a.n_tiles;
    const NodeT tb_nxt = (NodeT)(a.u_first + (has_next ? t_nxt : 0) * a.tile_nodes);
    const bool early = has_next && gate_open(tb_nxt, water_node, a);
    if (early) stage1<Id, NodeT, P>(nxt, t_nxt, a, E, L, water_node, n_pend);
    if (!stage2<Id, NodeT, P>(cur, t_cur, a, E, tilebuf, L, water_node, n_retry, n_wait, n_pend,
                              n_poll)) {
        ok = false;
        return false;
    }
    ++n_done;
    t_next = claim_next(cl, a, L);
    w = __shfl_sync(kFull, w, 0);
    __syncwarp();
    const NodeT wn = (NodeT)(a.u_first + w * a.sb_nodes);
    if (wn > water_node) water_node = wn;
    if (has_next && !early) {
        if (!wait_gate(tb_nxt, water_node, a, L, n_wait)) {
            ok = false;
            return false;
        }
        stage1<Id, NodeT, P>(nxt, t_nxt, a, E, L, water_node, n_pend);
    }
    t_nxt_out = t_nxt;
    return has_next;
}

template <typename Id, typename NodeT, int P>
__global__ void __launch_bounds__(kThreads, kMinBlocks) gen_kernel(const GenArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const uint32_t warp = threadIdx.x >> 5;
    Id *tilebuf = reinterpret_cast<Id *>(smem_raw) + warp * (32u * P);
    Id *E = reinterpret_cast<Id *>(a.edges);

    Lane L;
    L.lane = threadIdx.x & 31u;
    L.g = L.lane / a.d;
    L.slot = L.lane - L.g * a.d;
    L.used = L.lane < a.groups * a.d;
    L.gmask = L.used ? (a.d == 32 ? kFull : (((1u << a.d) - 1u) << (L.g * a.d))) : 0u;
    L.lt = lanemask_lt();
    L.le = L.lt | (1u << L.lane);

    if (blockIdx.x == 0 && warp == 0) {
        for (uint64_t e = L.lane; e < a.seed_edges; e += 32) {
            uint64_t s, t;
            seed_edge(e, a.d, a.seed_mode, s, t);
            st_pair(E + 2 * e, s, t);
        }
        if (gridDim.x * (blockDim.x >> 5) > 1) {
            advance_watermark(a, L.lane);
            return;
        }
    }

    uint32_t n_retry = 0, n_wait = 0, n_done = 0, n_pend = 0, n_poll = 0;   // per-lane counts

    // Prologue: the first two tiles and the current watermark.
    Claimer cl;
    cl.base = 0;
    cl.idx = a.claim_tiles;
    cl.pre = 0;
    unsigned long long wt = 0;
    if (L.lane == 0) {
        cl.pre = atomicAdd(&a.ctl->ticket, 1ull);
        wt = ld_acquire_u64(&my_rep(a)->water);
    }
    uint64_t tA = claim_next(cl, a, L);
    uint64_t t_next = claim_next(cl, a, L);
    wt = __shfl_sync(kFull, wt, 0);
    __syncwarp();   // orders lane 0's acquire before every lane's slot loads
    if (wt < a.water_init) wt = a.water_init;   // the start kernel's nodes
    NodeT water_node = (NodeT)(a.u_first + wt * a.sb_nodes);

    Slot<NodeT> A[P], B[P];
    bool ok = true;
    bool more = tA < a.n_tiles;
    if (more) {
        ok = wait_gate((NodeT)(a.u_first + tA * a.tile_nodes), water_node, a, L, n_wait);
        more = ok;
    }
    if (more) stage1<Id, NodeT, P>(A, tA, a, E, L, water_node, n_pend);

    uint64_t tB = 0;
    while (more) {
        more = pipeline_step<Id, NodeT, P>(A, B, tA, tB, t_next, cl, a, E, tilebuf, L, water_node,
                                           n_retry, n_wait, n_pend, n_poll, n_done, ok);
        if (!more) break;
        more = pipeline_step<Id, NodeT, P>(B, A, tB, tA, t_next, cl, a, E, tilebuf, L, water_node,
                                           n_retry, n_wait, n_pend, n_poll, n_done, ok);
    }

    // Warp totals, one atomic each.
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_retry += __shfl_down_sync(kFull, n_retry, o);
        n_pend += __shfl_down_sync(kFull, n_pend, o);
        n_poll += __shfl_down_sync(kFull, n_poll, o);
    }
    if (L.lane == 0) {
        if (n_pend) atomicAdd(&a.ctl->pending_reads, (unsigned long long)n_pend);
        if (n_poll) atomicAdd(&a.ctl->pending_polls, (unsigned long long)n_poll);
        if (n_retry) atomicAdd(&a.ctl->retries, (unsigned long long)n_retry);
        if (n_wait) atomicAdd(&a.ctl->waits, (unsigned long long)n_wait);
        if (n_done) atomicAdd(&a.ctl->tiles, (unsigned long long)n_done);
    }
}

template <typename Id, typename NodeT, int P>
int launch_one(const GenArgs &args, uint32_t blocks, cudaStream_t stream)
{
    auto kern = gen_kernel<Id, NodeT, P>;
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

template <typename Id, typename NodeT>
int launch_passes(const GenArgs &a, uint32_t passes, uint32_t blocks, cudaStream_t stream)
{
    switch (passes) {
    case 1: return launch_one<Id, NodeT, 1>(a, blocks, stream);
    case 2: return launch_one<Id, NodeT, 2>(a, blocks, stream);
    case 4: return launch_one<Id, NodeT, 4>(a, blocks, stream);
    case 8: return launch_one<Id, NodeT, 8>(a, blocks, stream);
    }
    return PA_ERR_INVALID;
}

}  // namespace

// Bytes [*off, *off + *len) of the edge buffer that a generation fills with
// all-ones before its kernels run: the slots of the start kernel's nodes (every
// node, for d > 32), after the seed edges.
void fill_region(const pa_params &prm, const GenPlan &plan, uint64_t *off, uint64_t *len)
{
    const uint64_t slot_bytes = (plan.slots ? 1ull : 2ull) * plan.id_bytes;
    const uint64_t seed = plan.slots ? 0 : plan.seed_edges;
    const uint64_t end = plan.wide ? prm.n : plan.u_split;
    *off = seed * slot_bytes;
    *len = end > plan.u_first ? (end - plan.u_first) * prm.d * slot_bytes : 0;
}

namespace {

// All-ones over bytes [lo, hi) of p: 16-byte stores over the aligned body, the
// ragged ends byte by byte from the first thread.  One small block per SM, so
// that a generation on another stream keeps its own blocks resident beside it.
__global__ void __launch_bounds__(128) fill_ones_kernel(unsigned char *p, uint64_t lo, uint64_t hi)
{
    const uint64_t a = (lo + 15) & ~15ull, b = hi & ~15ull;
    if (a >= b) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            for (uint64_t i = lo; i < hi; ++i) p[i] = 0xff;
        return;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (uint64_t i = lo; i < a; ++i) p[i] = 0xff;
        for (uint64_t i = b; i < hi; ++i) p[i] = 0xff;
    }
    uint4 *q = reinterpret_cast<uint4 *>(p + a);
    const uint64_t n16 = (b - a) >> 4;
    const uint4 ones = make_uint4(~0u, ~0u, ~0u, ~0u);
    // eight stores per thread per step keep enough writes in flight for a grid
    // this small
    constexpr uint32_t U = 8;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (; x + (U - 1) * stride < n16; x += U * stride) {
#pragma unroll
        for (uint32_t j = 0; j < U; ++j) q[x + j * stride] = ones;
    }
    for (; x < n16; x += stride) q[x] = ones;
}

}  // namespace

int fill_prefill(const pa_params *prm, const GenPlan &plan, void *d_edges, cudaStream_t s)
{
    uint64_t off = 0, len = 0;
    fill_region(*prm, plan, &off, &len);
    if (len == 0) return PA_OK;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    fill_ones_kernel<<<sms, 128, 0, s>>>(reinterpret_cast<unsigned char *>(d_edges), off, off + len);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

int launch_generate(const pa_params *prm, const GenPlan &plan, void *d_edges, void *d_scratch,
                    cudaStream_t stream, uint32_t blocks_override, const cudaEvent_t *events)
{
    // optional phase marks: [0] before the first launch, [1] before the start
    // kernel (after the clear and the fill), [2] before the persistent launch,
    // [3] after the last launch
    auto mark = [&](int i) -> int {
        if (!events || !events[i]) return PA_OK;
        const cudaError_t er = cudaEventRecord(events[i], stream);
        return er == cudaSuccess ? PA_OK : set_cuda_error(er);
    };
    int mrc = mark(0);
    if (mrc != PA_OK) return mrc;
    cudaError_t e = cudaMemsetAsync(d_scratch, 0, plan.scratch_bytes, stream);
    if (e != cudaSuccess) return set_cuda_error(e);

    GenArgs a;
    a.edges = d_edges;
    a.ctl = reinterpret_cast<GenCtl *>(d_scratch);
    a.reps = reinterpret_cast<GenRep *>(reinterpret_cast<unsigned char *>(d_scratch) + kRepOffset);
    a.flags = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(d_scratch) + kCtlBytes);
    a.sbcnt = reinterpret_cast<uint32_t *>(reinterpret_cast<unsigned char *>(d_scratch) + plan.sb_offset);
    a.n_sb = plan.n_sb;
    a.sb_nodes = (uint64_t)kSbTiles * plan.tile_nodes;
    a.n = prm->n;
    a.u_first = plan.u_first;
    a.n_tiles = plan.n_tiles;
    // SLOTS stores no seed rows: its ids start with node u_first's
    a.seed_edges = plan.slots ? 0 : plan.seed_edges;
    a.slot_off = (int64_t)a.seed_edges - (int64_t)(plan.u_first * prm->d);
    a.pth = plan.pth;
    a.spin_limit_ns = plan.spin_limit_ns;
    a.key0 = (uint32_t)prm->seed;
    a.key1 = (uint32_t)(prm->seed >> 32);
    a.d = prm->d;
    a.groups = plan.groups;
    a.tile_nodes = plan.tile_nodes;
    a.seed_mode = prm->seed_mode;
    a.withhold_first = (prm->flags & PA_FLAG_TEST_WITHHOLD_FIRST_TILE) ? 1u : 0u;
    a.trace = reinterpret_cast<uint64_t *>(reinterpret_cast<unsigned char *>(d_scratch) + plan.trace_offset);
    a.trace_step = (plan.n_sb + kTraceMax - 1) / kTraceMax;
    if (a.trace_step == 0) a.trace_step = 1;
    a.max_sleep_ns = 1024;
    a.window_shift = 3;
    a.min_window = 16384;
    a.tile_begin = 0;
    a.water_init = 0;

    a.start_end = plan.u_split;
    a.claim_tiles = plan.claim_tiles;
    a.model = plan.model;


    const uint32_t blocks = blocks_override ? blocks_override : prm->blocks;
    const bool prefilled = (prm->flags & PA_FLAG_PREFILLED) != 0;
    if (plan.wide) {
        // every node by the wide kernel, its slots starting as all-ones
        uint64_t off = 0, len = 0;
        fill_region(*prm, plan, &off, &len);
        if (!prefilled) {
            e = cudaMemsetAsync(reinterpret_cast<unsigned char *>(d_edges) + off, 0xff, len, stream);
            if (e != cudaSuccess) return set_cuda_error(e);
        }
        a.start_end = prm->n;
        if ((mrc = mark(1)) != PA_OK) return mrc;
        const int rc = launch_wide(plan.id_bytes, plan.slots, a,
                                   reinterpret_cast<unsigned long long *>(
                                       reinterpret_cast<unsigned char *>(d_scratch) + plan.start_offset),
                                   blocks, stream);
        if (rc != PA_OK) return rc;
        if ((mrc = mark(2)) != PA_OK) return mrc;
        return mark(3);
    }
    // 32-bit node arithmetic needs every node id, and tile base + tile_nodes,
    // below 2^32 - 32 (the top 32 values are the unknown-lane match keys).
    const bool small = prm->n + plan.tile_nodes + 32 < (1ull << 32);
    if (plan.u_split > plan.u_first) {
        // The start region, with slot-granular waits (pa_start.cu): its pairs
        // (ids, in SLOTS) start as all-ones; the start kernel writes them and
        // the seed edges.
        if (!prefilled) {
            uint64_t off = 0, len = 0;
            fill_region(*prm, plan, &off, &len);
            e = cudaMemsetAsync(reinterpret_cast<unsigned char *>(d_edges) + off, 0xff, len, stream);
            if (e != cudaSuccess) return set_cuda_error(e);
        }
        StartArgs sa;
        std::memset(&sa, 0, sizeof(sa));
        sa.one = a;
        sa.count = 1;
        sa.write_seeds = 1;
        sa.t_end = plan.start_tiles;
        sa.ticket = reinterpret_cast<unsigned long long *>(reinterpret_cast<unsigned char *>(d_scratch) +
                                                          plan.start_offset);
        sa.ctl = a.ctl;
        mrc = mark(1);
        if (mrc != PA_OK) return mrc;
        const int rc = launch_start(
            plan.id_bytes, sa, blocks, stream, plan.slots,
            start_min_blocks(plan.u_split - plan.u_first, plan.pth == 0 && plan.model == PA_MODEL_COPY));
        if (rc != PA_OK) return rc;
        if (plan.u_split >= prm->n) {
            mrc = mark(2);
            return mrc != PA_OK ? mrc : mark(3);
        }
        // u_split - u_first is a whole number of superblocks
        a.tile_begin = (plan.u_split - plan.u_first) / plan.tile_nodes;
        a.water_init = a.tile_begin / kSbTiles;
    }
    if (plan.slots && plan.u_split <= plan.u_first) {
        // a seed-only graph stores nothing in SLOTS
        for (int i = 1; i < 4; ++i)
            if ((mrc = mark(i)) != PA_OK) return mrc;
        return PA_OK;
    }
    if (plan.u_split <= plan.u_first) {
        mrc = mark(1);
        if (mrc != PA_OK) return mrc;
    }
    mrc = mark(2);
    if (mrc != PA_OK) return mrc;
    int rc;
    if (plan.id_bytes == 8)
        rc = small ? launch_passes<int64_t, uint32_t>(a, plan.passes, blocks, stream)
                   : launch_passes<int64_t, uint64_t>(a, plan.passes, blocks, stream);
    else
        rc = launch_passes<int32_t, uint32_t>(a, plan.passes, blocks, stream);
    return rc != PA_OK ? rc : mark(3);
}

}  // namespace pa
