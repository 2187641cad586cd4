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
#include "pa_device.cuh"
#include "pa_internal.h"

namespace pa {

namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kThreads = 256;
constexpr uint32_t kMinBlocks = 4;   // 32 resident warps per SM: at most 64 registers

enum : uint32_t { ST_KNOWN = 0, ST_PEND_GLOBAL = 1, ST_PEND_TILE = 2 };

struct GenArgs {
    void *edges;
    GenCtl *ctl;
    GenRep *reps;
    uint32_t *flags;
    uint32_t *sbcnt;      // tiles completed per superblock
    uint64_t n_sb;
    uint64_t sb_nodes;    // nodes per superblock
    uint64_t n;
    uint64_t u_first;
    uint64_t n_tiles;
    uint64_t seed_edges;
    int64_t slot_off;     // pair index of slot (v, k) = v*d + k + slot_off, for v > d
    uint64_t pth;
    uint64_t spin_limit_ns;
    uint32_t key0, key1;
    uint32_t d;
    uint32_t groups;
    uint32_t tile_nodes;
    uint32_t seed_mode;
    uint32_t withhold_first;   // test-only: never publish tile 0
    uint64_t *trace;           // progress samples (elapsed ns, nodes complete)
    uint64_t trace_step;       // superblocks between samples
    uint32_t window_shift;     // start gate: a tile at node tb waits for the watermark
    uint64_t min_window;       //   to reach tb - max(min_window, tb >> window_shift)
};

// Record a device-side error once, in the control block and every replica.
__device__ __forceinline__ void raise_error(const GenArgs &a, uint32_t code)
{
    if (atomicCAS(&a.ctl->error, 0u, code) == 0u)
        for (uint32_t r = 0; r < kReps; ++r) st_relaxed_u32(&a.reps[r].error, code);
}

// The replica a warp reads.
__device__ __forceinline__ const GenRep *my_rep(const GenArgs &a)
{
    return a.reps + ((blockIdx.x * (kThreads / 32) + (threadIdx.x >> 5)) % kReps);
}

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

// One draw in node arithmetic of width NodeT (see draw_slot in pa_device.cuh;
// identical values: for u < 2^32, floor(x*u / 2^64) with x = w1:w0 equals
// floor((w1*u + floor(w0*u / 2^32)) / 2^32)).
template <typename NodeT>
struct DrawT {
    NodeT v;
    uint32_t k;
    bool direct;
};

template <typename NodeT>
__device__ __forceinline__ DrawT<NodeT> draw(NodeT u, uint32_t i, uint32_t r, const GenArgs &a)
{
    DrawT<NodeT> out;
    if constexpr (sizeof(NodeT) == 4) {
        const uint4 w = philox4x32_10(make_uint4(u, 0u, i, r), a.key0, a.key1);
        const uint64_t lo = (uint64_t)w.x * u;
        const uint64_t hi = (uint64_t)w.y * u + (lo >> 32);
        out.v = (uint32_t)(hi >> 32);
        out.k = __umulhi(w.w, a.d);
        out.direct = (uint64_t)w.z < a.pth;
    } else {
        const Draw dr = draw_slot(u, i, r, a.key0, a.key1, a.pth, a.d);
        out.v = dr.v;
        out.k = dr.k;
        out.direct = dr.direct;
    }
    return out;
}

// Per-slot resolution state held in registers.
template <typename NodeT>
struct Slot {
    NodeT val;      // candidate value, or the pending source node v
    uint32_t meta;  // state (bits 0-1) | k (bits 2-7) | retry (bits 8-31)
};

__device__ __forceinline__ uint32_t meta_st(uint32_t m) { return m & 3u; }
__device__ __forceinline__ uint32_t meta_k(uint32_t m) { return (m >> 2) & 63u; }
__device__ __forceinline__ uint32_t meta_r(uint32_t m) { return m >> 8; }

template <typename Id, typename NodeT>
__device__ __forceinline__ const Id *slot_addr(const Id *E, const GenArgs &a, NodeT v, uint32_t k)
{
    const int64_t idx = (int64_t)((uint64_t)v * a.d) + (int64_t)k + a.slot_off;
    return E + 2 * idx + 1;
}

// Where the candidate of a fresh draw comes from.
template <typename Id, typename NodeT>
__device__ __forceinline__ void classify(Slot<NodeT> &s, const DrawT<NodeT> &dr, uint32_t r,
                                         const GenArgs &a, const Id *E, NodeT tb,
                                         NodeT water_node, uint32_t &n_pend)
{
    uint32_t st;
    if (dr.direct) {
        s.val = dr.v;
        st = ST_KNOWN;
    } else if (dr.v <= a.d) {
        s.val = (NodeT)seed_slot(dr.v, dr.k, a.d, a.seed_mode);
        st = ST_KNOWN;
    } else if (dr.v < water_node) {
        s.val = (NodeT)ld_slot(slot_addr(E, a, dr.v, dr.k));
        st = ST_KNOWN;
    } else if (dr.v < tb) {
        s.val = dr.v;
        st = ST_PEND_GLOBAL;
        ++n_pend;
    } else {
        s.val = dr.v;
        st = ST_PEND_TILE;
    }
    s.meta = st | (dr.k << 2) | (r << 8);
}

// Per-warp constants of one launch.
struct Lane {
    uint32_t lane, g, slot, gmask, lt, le;
    bool used;
};

// Stage 1: retry-0 draws of every slot of tile t, early copy loads.
template <typename Id, typename NodeT, int P>
__device__ __forceinline__ void stage1(Slot<NodeT> (&s)[P], uint64_t t, const GenArgs &a,
                                       const Id *E, const Lane &L, NodeT water_node,
                                       uint32_t &n_pend)
{
    const NodeT tb = (NodeT)(a.u_first + t * a.tile_nodes);
    const NodeT te = (NodeT)min(a.n, (uint64_t)tb + a.tile_nodes);
#pragma unroll
    for (int j = 0; j < P; ++j) {
        const NodeT u = tb + (NodeT)(j * a.groups + L.g);
        s[j].val = 0;
        s[j].meta = ST_KNOWN;
        if (L.used && u < te)
            classify(s[j], draw<NodeT>(u, L.slot, 0u, a), 0u, a, E, tb, water_node, n_pend);
    }
}

// Resolve the slots of one warp pass until every active lane is final.
// Returns false when the warp must stop (wait limit, or another warp failed).
template <typename Id, typename NodeT>
__device__ __forceinline__ bool resolve_pass(Slot<NodeT> &s, const GenArgs &a, const Id *E,
                                             const Id *tilebuf, NodeT tb, NodeT pbase,
                                             uint32_t pass_off, NodeT u, bool active,
                                             const Lane &L, NodeT &water_node,
                                             uint32_t &n_retry, uint32_t &n_wait,
                                             uint32_t &n_pend, uint32_t &n_poll)
{
    const uint32_t d = a.d;
    uint64_t spin_t0 = 0;
    uint32_t sleep_ns = 64;
    for (;;) {
        bool changed = false;
        const uint32_t st0 = meta_st(s.meta);
        const uint32_t k = meta_k(s.meta);
        if (active && st0 == ST_PEND_GLOBAL) {
            const NodeT v = s.val;
            bool ready = v < water_node;
            if (!ready)
                ready = ld_acquire_u32(a.flags + ((uint64_t)v - a.u_first) / a.tile_nodes) != 0u;
            if (!ready) ++n_poll;
            if (ready) {
                s.val = (NodeT)ld_slot(slot_addr(E, a, v, k));
                s.meta &= ~3u;
                changed = true;
            }
        } else if (active && st0 == ST_PEND_TILE) {
            const NodeT off = s.val - tb;
            if (off < (NodeT)pass_off) {   // a finished earlier pass of this tile
                s.val = (NodeT)tilebuf[(uint32_t)off * d + k];
                s.meta &= ~3u;
                changed = true;
            }
        }

        const bool known = active && meta_st(s.meta) == ST_KNOWN;
        uint32_t eq;
        if constexpr (sizeof(NodeT) == 4) {
            // values < 2^32 - 32: the lane-unique keys of unknown lanes never collide
            eq = __match_any_sync(kFull, known ? (uint32_t)s.val : (0xffffffe0u | L.lane));
        } else {
            eq = __match_any_sync(kFull, known ? (unsigned long long)s.val
                                               : (0x8000000000000000ull | L.lane));
        }
        const bool bad = active && (!known || (eq & L.lt & L.gmask) != 0u);
        const uint32_t badm = __ballot_sync(kFull, bad);
        const bool fin = active && (badm & L.gmask & L.le) == 0u;
        const uint32_t finm = __ballot_sync(kFull, fin || !active);
        if (finm == kFull) return true;

        // Copy targets in this same pass: take the source lane's value once
        // that lane is final.
        const bool same = active && meta_st(s.meta) == ST_PEND_TILE && s.val >= pbase;
        const uint32_t src = same ? (uint32_t)(s.val - pbase) * d + k : L.lane;
        const NodeT sv = __shfl_sync(kFull, s.val, src);
        if (same && ((finm >> src) & 1u)) {
            s.val = sv;
            s.meta &= ~3u;
            changed = true;
        }

        // A candidate equal to a final lower slot is rejected for certain.
        if (known && !fin && (eq & L.lt & L.gmask & finm) != 0u) {
            const uint32_t r = meta_r(s.meta) + 1u;
            classify(s, draw<NodeT>(u, L.slot, r, a), r, a, E, tb, water_node, n_pend);
            changed = true;
            ++n_retry;
        }

        if (!__any_sync(kFull, changed)) {
            // Nothing moved: every open slot waits on another tile.
            unsigned long long now = 0, w2 = 0;
            uint32_t err = 0;
            if (L.lane == 0) {
                now = globaltimer_ns();
                const GenRep *rp = my_rep(a);
                err = ld_relaxed_u32(&rp->error);
                w2 = ld_acquire_u64(&rp->water);
                ++n_wait;
            }
            now = __shfl_sync(kFull, now, 0);
            err = __shfl_sync(kFull, err, 0);
            w2 = __shfl_sync(kFull, w2, 0);
            __syncwarp();
            water_node = (NodeT)(a.u_first + w2 * a.sb_nodes);
            if (spin_t0 == 0) spin_t0 = now;
            if (err != 0) return false;
            if (now - spin_t0 > a.spin_limit_ns) {
                if (L.lane == 0) raise_error(a, (uint32_t)PA_ERR_SPIN_TIMEOUT);
                return false;
            }
            __nanosleep(sleep_ns);
            sleep_ns = min(sleep_ns * 2u, 1024u);
        } else {
            spin_t0 = 0;
            sleep_ns = 64;
        }
    }
}

// Stage 2: resolve, store and publish tile t.
template <typename Id, typename NodeT, int P>
__device__ __forceinline__ bool stage2(Slot<NodeT> (&s)[P], uint64_t t, const GenArgs &a, Id *E,
                                       Id *tilebuf, const Lane &L, NodeT &water_node,
                                       uint32_t &n_retry, uint32_t &n_wait, uint32_t &n_pend,
                                       uint32_t &n_poll)
{
    const uint32_t d = a.d, G = a.groups;
    const NodeT tb = (NodeT)(a.u_first + t * a.tile_nodes);
    const NodeT te = (NodeT)min(a.n, (uint64_t)tb + a.tile_nodes);
#pragma unroll
    for (int j = 0; j < P; ++j) {
        const NodeT pbase = tb + (NodeT)(j * G);   // first node of the pass
        const NodeT u = pbase + (NodeT)L.g;
        const bool active = L.used && u < te;
        if (!resolve_pass(s[j], a, E, tilebuf, tb, pbase, (uint32_t)j * G, u, active, L,
                          water_node, n_retry, n_wait, n_pend, n_poll))
            return false;
        // Finished pass: keep it for in-tile copy reads, then emit the edges.
        if (active) tilebuf[(uint32_t)j * G * d + L.lane] = (Id)s[j].val;
        __syncwarp();
        const uint64_t e0 = a.seed_edges + ((uint64_t)pbase - a.u_first) * d;
        if constexpr (sizeof(Id) == 8) {
            if (active) st_pair(E + 2 * (e0 + L.lane), (uint64_t)u, (uint64_t)s[j].val);
        } else {
            const uint32_t nu = __shfl_down_sync(kFull, (uint32_t)u, 1);
            const uint32_t nv = __shfl_down_sync(kFull, (uint32_t)s[j].val, 1);
            const uint32_t na = __shfl_down_sync(kFull, (uint32_t)active, 1);
            const bool leader = ((L.lane + (uint32_t)(e0 & 1u)) & 1u) == 0u;
            if (active) {
                Id *p = E + 2 * (e0 + L.lane);
                if (leader) {
                    if (L.lane < 31u && na) st_pair2(p, u, s[j].val, nu, nv);
                    else st_pair(p, u, s[j].val);
                } else if (L.lane == 0) {
                    st_pair(p, u, s[j].val);
                }
            }
        }
    }

    // Publish.  The warp barrier orders every lane's stores before lane 0's
    // release fence; the flag and the superblock count are written after it.
    __syncwarp();
    if (L.lane == 0 && !(a.withhold_first && t == 0)) {
        fence_acq_rel_gpu();
        st_relaxed_u32(a.flags + t, 1u);
        red_add_relaxed_u32(a.sbcnt + t / kSbTiles, 1u);
    }
    return true;
}

// The single writer of the completion watermark.  Each round trip reads the
// tile counts of 128 consecutive superblocks (one 16-byte load per lane),
// advances over the complete prefix and publishes it with a release store.  It
// stops when every superblock is complete, when a worker has raised an error,
// or after spin_limit_ns without progress (the workers' own waits are bounded by
// the same limit, so a stall that long means they have stopped).
__device__ __forceinline__ void advance_watermark(const GenArgs &a, uint32_t lane)
{
    uint64_t w = 0;
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

// Tiles are claimed kClaimTiles at a time: one ticket names a chunk of
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
    if (c.idx == kClaimTiles) {
        const uint64_t chunk = __shfl_sync(kFull, c.pre, 0);
        if (L.lane == 0) c.pre = atomicAdd(&a.ctl->ticket, 1ull);
        c.base = chunk * kClaimTiles;
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
    cl.idx = kClaimTiles;
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

int launch_generate(const pa_params *prm, const GenPlan &plan, void *d_edges, void *d_scratch,
                    cudaStream_t stream, uint32_t blocks_override)
{
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
    a.seed_edges = plan.seed_edges;
    a.slot_off = (int64_t)plan.seed_edges - (int64_t)(plan.u_first * prm->d);
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
    a.window_shift = 3;
    a.min_window = 16384;

    const uint32_t blocks = blocks_override ? blocks_override : prm->blocks;
    // 32-bit node arithmetic needs every node id, and tile base + tile_nodes,
    // below 2^32 - 32 (the top 32 values are the unknown-lane match keys).
    const bool small = prm->n + plan.tile_nodes + 32 < (1ull << 32);
    if (plan.id_bytes == 8)
        return small ? launch_passes<int64_t, uint32_t>(a, plan.passes, blocks, stream)
                     : launch_passes<int64_t, uint64_t>(a, plan.passes, blocks, stream);
    return launch_passes<int32_t, uint32_t>(a, plan.passes, blocks, stream);
}

}  // namespace pa
