// pa_gen_core.cuh -- the generation device code shared by the single-graph
// kernel (pa_generate.cu) and the batched kernel (pa_batch.cu): launch
// arguments, the draw, slot classification, the per-pass resolution loop and the
// two pipeline stages.  See pa_generate.cu for the algorithm.
#pragma once

#include <vector>

#include "pa_device.cuh"
#include "pa_internal.h"

namespace pa {
namespace gen {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kThreads = 256;
constexpr uint32_t kMinBlocks = 4;   // 32 resident warps per SM: at most 64 registers
// The start kernel: 40 warps per SM (at most 51 registers; a few bytes spill).
// More warps put more copy reads in flight: C3 69.4 -> 68.2 ms at p = 0.5.
constexpr uint32_t kStartMinBlocks = 5;
// p = 0 (every slot a copy, several retries per node): 48 warps per SM pay off
// there (C3 270 -> 259 ms) though they cost at p = 0.5 (68.1 -> 71.7 ms).
constexpr uint32_t kStartMinBlocksCopy = 6;
// A single graph with a small start region is bound by its dependency chains'
// latency, which the spills of the wider variants lengthen: four blocks, 64
// registers, no spills.
constexpr uint32_t kStartMinBlocksSmall = 4;
constexpr uint64_t kStartLargeNodes = 1ull << 24;

// The start-kernel variant for one graph: start region nodes, copy-only (p = 0).
inline uint32_t start_min_blocks(uint64_t start_nodes, bool copy_only)
{
    if (start_nodes < kStartLargeNodes) return kStartMinBlocksSmall;
    return copy_only ? kStartMinBlocksCopy : kStartMinBlocks;
}

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
    int64_t slot_off;     // index of slot (v, k) = v*d + k + slot_off, for v > d (a pair
                          // index in PAIRS; the id index in SLOTS, where seed_edges = 0)
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
    uint32_t max_sleep_ns;     // back-off cap of dependency waits
    uint64_t tile_begin;       // first tile of the persistent launch (earlier ones: start kernel)
    uint64_t water_init;       // superblocks complete when the persistent launch starts
    uint32_t window_shift;     // start gate: a tile at node tb waits for the watermark
    uint64_t min_window;       //   to reach tb - max(min_window, tb >> window_shift)
    uint64_t start_end;        // start kernel: nodes [u_first, start_end) are its work
    uint32_t claim_tiles;      // tiles per claim-counter atomic
    uint32_t model;            // PA_MODEL_COPY or PA_MODEL_BA
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

// e-th canonical seed edge (seed_edge_of in pa_device.cuh).
__device__ __forceinline__ void seed_edge(uint64_t e, uint32_t d, uint32_t mode, uint64_t &src,
                                          uint64_t &dst)
{
    seed_edge_of(e, d, mode, src, dst);
}

// One draw in node arithmetic of width NodeT (see draw_slot in pa_device.cuh;
// identical values: for u < 2^32, floor(x*u / 2^64) with x = w1:w0 equals
// floor((w1*u + floor(w0*u / 2^32)) / 2^32)).
//
// BA model (src/PA/SPA/SerialBA.cpp:145-157): the endpoint index is R =
// floor(x * 2du / 2^64), uniform over the 2du endpoints before node u.  With
// x*u = v*2^64 + f, R = 2d*v + floor(2d*f / 2^64), so v = floor(x*u / 2^64) is
// the node of the endpoint pair (v < d: a seed block entry, which is v itself),
// q = floor(2d*f / 2^64) < 2d its position: odd -> v, even -> v's slot q/2.
// Seed slots of STAR_REF already map v < d to v and node d to slot k, so the
// draw becomes (v, k = q/2, direct = q odd) and the rest of the kernel is the
// copy model's.
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
        if (a.model == PA_MODEL_BA) {
            const uint64_t f = (hi << 32) | (uint32_t)lo;   // x*u mod 2^64
            const uint32_t q = (uint32_t)__umul64hi(f, 2ull * a.d);
            out.k = q >> 1;
            out.direct = q & 1u;
        } else {
            out.k = __umulhi(w.w, a.d);
            out.direct = (uint64_t)w.z < a.pth;
        }
    } else {
        const Draw dr = a.model == PA_MODEL_BA ? draw_slot_ba(u, i, r, a.key0, a.key1, a.d)
                                               : draw_slot(u, i, r, a.key0, a.key1, a.pth, a.d);
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

// Address of the target of slot (v, k): the second field of its pair (PAIRS)
// or the id itself (SLOTS).
template <typename Id, typename NodeT, bool Slots = false>
__device__ __forceinline__ const Id *slot_addr(const Id *E, const GenArgs &a, NodeT v, uint32_t k)
{
    const int64_t idx = (int64_t)((uint64_t)v * a.d) + (int64_t)k + a.slot_off;
    return Slots ? E + idx : E + 2 * idx + 1;
}

// Whether the superblock holding node v has all its tiles published (the
// batched kernel's substitute for a watermark: the counts are L2-resident).
template <typename NodeT>
__device__ __forceinline__ bool sb_complete(const GenArgs &a, NodeT v)
{
    const uint64_t t = ((uint64_t)v - a.u_first) / a.tile_nodes;
    const uint64_t sb = t / kSbTiles;
    const uint32_t need = (uint32_t)min((uint64_t)kSbTiles, a.n_tiles - sb * kSbTiles);
    return ld_acquire_u32(a.sbcnt + sb) == need;
}

// Where the candidate of a fresh draw comes from.  With SbCheck, a source node
// at or above the watermark is still read at once when its superblock is
// complete.
template <typename Id, typename NodeT, bool SbCheck = false>
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
    } else if (dr.v < water_node || (SbCheck && dr.v < tb && sb_complete(a, dr.v))) {
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
template <typename Id, typename NodeT, int P, bool SbCheck = false>
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
            classify<Id, NodeT, SbCheck>(s[j], draw<NodeT>(u, L.slot, 0u, a), 0u, a, E, tb,
                                         water_node, n_pend);
    }
}

// Resolve the slots of one warp pass until every active lane is final.
// Returns false when the warp must stop (wait limit, or another warp failed).
template <typename Id, typename NodeT, bool SbCheck = false>
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
        // Lanes waiting on the same unfinished tile share one flag poll: the
        // lowest lane of each group polls and passes the answer on.
        const bool want = active && st0 == ST_PEND_GLOBAL && !(s.val < water_node);
        uint32_t flag = 0;
        if (__any_sync(kFull, want)) {
            const NodeT want_tile = want ? (NodeT)(((uint64_t)s.val - a.u_first) / a.tile_nodes)
                                         : (NodeT)(~(NodeT)0 - L.lane);
            const uint32_t peers = __match_any_sync(kFull, want_tile);
            const uint32_t leader = __ffs(peers) - 1;
            if (want && L.lane == leader) {
                flag = ld_acquire_u32(a.flags + want_tile);
                if (!flag) ++n_poll;
            }
            flag = __shfl_sync(kFull, flag, leader);
        }
        if (active && st0 == ST_PEND_GLOBAL) {
            const NodeT v = s.val;
            const bool ready = v < water_node || flag != 0u;
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
            classify<Id, NodeT, SbCheck>(s, draw<NodeT>(u, L.slot, r, a), r, a, E, tb,
                                         water_node, n_pend);
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
            const NodeT wn2 = (NodeT)(a.u_first + w2 * a.sb_nodes);
            if (wn2 > water_node) water_node = wn2;
            if (spin_t0 == 0) spin_t0 = now;
            if (err != 0) return false;
            if (now - spin_t0 > a.spin_limit_ns) {
                if (L.lane == 0) raise_error(a, (uint32_t)PA_ERR_SPIN_TIMEOUT);
                return false;
            }
            __nanosleep(sleep_ns);
            sleep_ns = min(sleep_ns * 2u, a.max_sleep_ns);
        } else {
            spin_t0 = 0;
            sleep_ns = 64;
        }
    }
}

// Stage 2: resolve, store and publish tile t.
template <typename Id, typename NodeT, int P, bool SbCheck = false>
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
        if (!resolve_pass<Id, NodeT, SbCheck>(s[j], a, E, tilebuf, tb, pbase, (uint32_t)j * G, u,
                                              active, L, water_node, n_retry, n_wait, n_pend,
                                              n_poll))
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

}  // namespace gen
}  // namespace pa

// ---------------------------------------------------------------------------
// Level-ordered index spaces of several graphs, and the two extra launches.
//
// Level l of a graph covers nodes [B_l, B_{l+1}), B_{l+1} = B_l +
// max(kLevelMinNodes, B_l >> kLevelShift).  The units (tiles or passes) of
// several graphs form one index space ordered by level and, within a level, by
// graph, so the start of every graph is worked on first and side by side.
// Within one graph the order is increasing, which is what deadlock freedom
// needs (a unit waits only on lower units of its own graph).
// ---------------------------------------------------------------------------
namespace pa {
namespace gen {

constexpr uint64_t kLevelMinNodes = 4096;
constexpr uint32_t kLevelShift = 3;
constexpr uint32_t kMaxLevels = 160;

// Device copies of the level tables of a set of graphs.
struct LevelTables {
    const unsigned long long *lvl_base;    // levels + 1: first global unit of each level
    const unsigned long long *inst_base;   // levels x (count + 1): prefix within a level
    const unsigned long long *loc_start;   // levels x count: graph's first unit of a level
    uint32_t levels;
};

// Unit bounds of a graph's levels over nodes [u_first, n_end) in units of
// unit_nodes: entry l is the first unit of level l, the last is n_units.
std::vector<uint64_t> level_bounds(uint64_t u_first, uint64_t n_end, uint64_t n_units,
                                   uint64_t unit_nodes);

// Largest index i in [0, len) with a[i] <= x (a ascending, a[0] <= x).
__device__ __forceinline__ uint32_t last_le(const unsigned long long *a, uint32_t len,
                                            unsigned long long x)
{
    uint32_t lo = 0, hi = len;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Global unit T -> (graph, unit of the graph).
__device__ __forceinline__ void map_unit(const LevelTables &tab, uint32_t count,
                                         unsigned long long T, uint32_t &inst, uint64_t &t)
{
    const uint32_t l = last_le(tab.lvl_base, tab.levels, T);
    const unsigned long long r = T - __ldg(tab.lvl_base + l);
    const unsigned long long *ib = tab.inst_base + (uint64_t)l * (count + 1);
    inst = last_le(ib, count, r);
    t = __ldg(tab.loc_start + (uint64_t)l * count + inst) + (r - __ldg(ib + inst));
}

// map_unit, plus the segment that T falls in: the global units [lo, hi) of
// (level, graph inst), whose unit lo is the graph's local unit t0.  Every T in
// it maps to (inst, t0 + T - lo) without a search.
__device__ __forceinline__ void map_unit_seg(const LevelTables &tab, uint32_t count,
                                             unsigned long long T, uint32_t &inst,
                                             unsigned long long &lo, unsigned long long &hi,
                                             unsigned long long &t0)
{
    const uint32_t l = last_le(tab.lvl_base, tab.levels, T);
    const unsigned long long base = __ldg(tab.lvl_base + l);
    const unsigned long long *ib = tab.inst_base + (uint64_t)l * (count + 1);
    inst = last_le(ib, count, T - base);
    lo = base + __ldg(ib + inst);
    hi = base + __ldg(ib + inst + 1);
    t0 = __ldg(tab.loc_start + (uint64_t)l * count + inst);
}

// The start kernel's claim counters: warp w of a block claims from counter w,
// which hands out start tiles w, w + 8, w + 16, ... (one atomic per tile, eight
// addresses instead of one).
constexpr uint32_t kStartCounters = kThreads / 32;

// Start kernel (pa_start.cu): start tiles of one graph (count == 1, arguments in
// `one`) or of `count` graphs in level order (arguments in `inst`).
struct StartArgs {
    GenArgs one;
    const GenArgs *inst;
    LevelTables tab;
    uint32_t count;
    uint32_t write_seeds;          // also write every graph's seed edges
    unsigned long long t_end;      // start tiles of the launch
    unsigned long long *ticket;    // kStartCounters claim counters, 128 bytes apart (zero)
    GenCtl *ctl;                   // shared status and counters
};

// Launch the start kernel; `blocks` 0 = one wave.  The claim counters must be
// zero and every pair of the graphs' start regions all-ones (fill_start).
// min_blocks: the variant's resident blocks per SM (start_min_blocks picks it).
int launch_start(uint32_t id_bytes, const StartArgs &b, uint32_t blocks, cudaStream_t s,
                 bool slots = false, uint32_t min_blocks = kStartMinBlocks);

// Set every byte of the pairs of nodes [u_first, start_end) of each of `count`
// graphs to 0xff (one launch).
int fill_start(uint32_t id_bytes, const GenArgs *d_inst, uint32_t count, uint64_t max_pairs,
               cudaStream_t s);

// Batch kernel (pa_batch.cu) over global tiles [t_begin, t_end) of `count`
// graphs; every node of graph i below node u_first + loc_start[l_begin][i] *
// tile_nodes is complete when it starts.
int launch_tail(uint32_t id_bytes, uint32_t passes, const GenArgs *d_inst, const LevelTables &tabs,
                uint32_t count, unsigned long long t_begin, unsigned long long t_end,
                unsigned long long *d_ticket, GenCtl *ctl, uint32_t claim_tiles, cudaStream_t s);

}  // namespace gen
}  // namespace pa
