// pa_start.cu -- graphs generated with waits on single slots.
//
// Early in a graph most copy reads land on nodes that are still being
// generated.  The persistent kernel publishes completion per tile, and a tile
// is complete only once the sources of all of its nodes are, so a dependency
// chain counted in tiles is far longer than the same chain counted in nodes:
// the longest chain of a random recursive graph grows like c*ln(u) in nodes,
// while a tile takes the maximum over the chains of all its ~2*tile_nodes copy
// sources at every step (a simulation of d = 4, p = 1/2 gives 28 node steps but
// 136 tile steps at 8192 nodes, 49 against 365 at 2^18).  With each step a
// poll round trip, the first few million nodes of a graph cost milliseconds.
//
// This kernel takes the tile out of the chain.  Before it runs, every pair of
// its region is set to all-ones (a memset), which is never a node id.  A lane
// stores its slot's pair the moment the slot is final -- every lower slot of
// its node final and its candidate distinct from theirs -- and a copy read of
// slot (v, k) re-reads that pair's target field until it is not all-ones.  The
// datum is its own completion flag: it is written once, with its final value,
// so a gpu-scope relaxed load returns either the fill or that value, and no
// fence, flag or watermark is involved.  Copy sources inside the lane's own
// warp pass are taken from the source lane by shuffle once it is final, as in
// the persistent kernel.  (Filling inside the kernel instead -- each warp
// filling the tile it claims, with per-tile opened flags and a watermark for
// readers -- measured slower on B200 than the memset it saves: 88.7 against
// 68.0 ms for n = 2^30, d = 4.)
//
// Work is claimed one start tile at a time: kStartPasses warp passes of G =
// 32/d nodes each (lane = node-in-pass * d + slot), resolved together, so a
// wait in one pass does not hold back the others.  Warp w of a block claims
// from counter w (of kStartCounters), which hands out tiles w, w + 8, ... in
// increasing order: eight counter lines instead of one, since a single counter
// saturates at one atomic every few nanoseconds.  Several graphs share one
// launch in level order (pa_gen_core.cuh).
//
// Draws, the slot order and the rejection rule are the persistent kernel's, so
// the output is bit-identical to it and to the sequential definition
// (src/PA/SPA/SerialCopyModel3.cpp:50-92 of the reference, with Philox draws).
#include <algorithm>

#include "pa_gen_core.cuh"

namespace pa {
namespace gen {
namespace {

template <typename Id>
struct Sentinel {
    static constexpr uint64_t value = sizeof(Id) == 8 ? ~0ull : 0xffffffffull;
};

// Read slot (v, k) into s: true with its value, or false (s.val = v) while it
// still holds the fill.
template <typename Id, bool Slots>
__device__ __forceinline__ bool read_slot(Slot<uint32_t> &s, const GenArgs &a, const Id *E,
                                          uint32_t v, uint32_t k)
{
    const uint64_t x = ld_slot(slot_addr<Id, uint32_t, Slots>(E, a, v, k));
    if (x != Sentinel<Id>::value) {
        s.val = (uint32_t)x;
        return true;
    }
    s.val = v;
    return false;
}

// Where the candidate of a fresh draw comes from (32-bit node arithmetic: the
// start region ends below 2^31).
template <typename Id, bool Slots>
__device__ __forceinline__ void classify_start(Slot<uint32_t> &s, const DrawT<uint32_t> &dr,
                                               uint32_t r, const GenArgs &a, const Id *E,
                                               uint32_t pbase, uint32_t &n_pend)
{
    uint32_t st = ST_KNOWN;
    if (dr.direct) {
        s.val = dr.v;
    } else if (dr.v <= a.d) {
        s.val = (uint32_t)seed_slot(dr.v, dr.k, a.d, a.seed_mode);
    } else if (dr.v < pbase) {
        if (!read_slot<Id, Slots>(s, a, E, dr.v, dr.k)) {
            st = ST_PEND_GLOBAL;
            ++n_pend;
        }
    } else {
        s.val = dr.v;   // an earlier node of this same pass
        st = ST_PEND_TILE;
    }
    s.meta = st | (dr.k << 2) | (r << 8);
}

// Resolve the kStartPasses warp passes of one start tile together; every slot is
// stored as soon as it is final.  Copy sources in the lane's own pass come from
// the source lane by shuffle; sources in an earlier pass of the tile are polled
// in memory like any other.  Returns false when the warp must stop (wait limit,
// or another warp failed).
template <typename Id, bool Slots>
__device__ __forceinline__ bool resolve_start(Slot<uint32_t> (&s)[kStartPasses], const GenArgs &a,
                                              Id *E, uint32_t tb, bool withhold, const Lane &L,
                                              uint32_t &n_retry, uint32_t &n_wait,
                                              uint32_t &n_pend, uint32_t &n_poll)
{
    const uint32_t d = a.d, G = a.groups;
    // this lane's slot of pass 0: a pair (PAIRS) or an id (SLOTS, seed_edges = 0)
    const uint64_t e_lane = a.seed_edges + (uint64_t)(tb - (uint32_t)a.u_first) * d + L.lane;
    Id *pair0 = Slots ? E + e_lane : E + 2 * e_lane;
    uint32_t stored = 0;   // bit j: pass j's slot is stored (or inactive)
#pragma unroll
    for (int j = 0; j < kStartPasses; ++j)
        if (!(L.used && tb + j * G + L.g < a.start_end)) stored |= 1u << j;
    const uint32_t max_sleep = min(a.max_sleep_ns, 512u);
    uint64_t spin_t0 = 0;
    uint32_t sleep_ns = 32;
    // bit j: every active slot of pass j is final and stored (warp-uniform); a
    // finished pass costs no more match or ballot while the others wait
    uint32_t done = 0;
    // bit j: this lane's slot of pass j changed after the pass's last match; a
    // pass in which no lane changed would match and vote exactly as before, so
    // only its pending reads are polled (one vote per pass and round)
    uint32_t dirty = (1u << kStartPasses) - 1u;
    for (;;) {
        bool changed = false;
#pragma unroll
        for (int j = 0; j < kStartPasses; ++j) {
            if ((done >> j) & 1u) continue;
            const uint32_t pbase = tb + j * G;
            const uint32_t u = pbase + L.g;
            const bool active = L.used && u < a.start_end;
            bool ch = (dirty >> j) & 1u;
            if (active && meta_st(s[j].meta) == ST_PEND_GLOBAL) {
                if (read_slot<Id, Slots>(s[j], a, E, s[j].val, meta_k(s[j].meta))) {
                    s[j].meta &= ~3u;
                    ch = true;
                    changed = true;
                } else {
                    ++n_poll;
                }
            }
            if (!__any_sync(kFull, ch)) continue;
            dirty &= ~(1u << j);
            const bool known = active && meta_st(s[j].meta) == ST_KNOWN;
            // node values are < 2^31: the lane-unique keys of unknown lanes never collide
            const uint32_t eq = __match_any_sync(kFull, known ? s[j].val : (0xffffffe0u | L.lane));
            const bool bad = active && (!known || (eq & L.lt & L.gmask) != 0u);
            const uint32_t badm = __ballot_sync(kFull, bad);
            const bool fin = active && (badm & L.gmask & L.le) == 0u;
            if (fin && !((stored >> j) & 1u)) {
                if (!withhold) {
                    if constexpr (Slots) st_relaxed_id(pair0 + (uint64_t)(j * G * d), s[j].val);
                    else st_relaxed_pair(pair0 + 2 * (uint64_t)(j * G * d), u, s[j].val);
                }
                stored |= 1u << j;
            }
            const uint32_t finm = __ballot_sync(kFull, fin || !active);
            if (finm == kFull) {
                done |= 1u << j;
                continue;
            }

            // copy sources in this pass: the source lane's value once it is final
            const bool same = active && meta_st(s[j].meta) == ST_PEND_TILE;
            const uint32_t src = same ? (s[j].val - pbase) * d + meta_k(s[j].meta) : L.lane;
            const uint32_t sv = __shfl_sync(kFull, s[j].val, src);
            if (same && ((finm >> src) & 1u)) {
                s[j].val = sv;
                s[j].meta &= ~3u;
                dirty |= 1u << j;
                changed = true;
            }

            // a candidate equal to a final lower slot of the node is rejected
            if (known && !fin && (eq & L.lt & L.gmask & finm) != 0u) {
                const uint32_t r = meta_r(s[j].meta) + 1u;
                classify_start<Id, Slots>(s[j], draw<uint32_t>(u, L.slot, r, a), r, a, E, pbase,
                                          n_pend);
                dirty |= 1u << j;
                changed = true;
                ++n_retry;
            }
        }
        if (done == (1u << kStartPasses) - 1u) return true;

        if (!__any_sync(kFull, changed)) {
            unsigned long long now = 0;
            uint32_t err = 0;
            if (L.lane == 0) {
                now = globaltimer_ns();
                err = ld_relaxed_u32(&my_rep(a)->error);
                ++n_wait;
            }
            now = __shfl_sync(kFull, now, 0);
            err = __shfl_sync(kFull, err, 0);
            if (err != 0) return false;
            if (spin_t0 == 0) spin_t0 = now;
            if (now - spin_t0 > a.spin_limit_ns) {
                if (L.lane == 0) raise_error(a, (uint32_t)PA_ERR_SPIN_TIMEOUT);
                return false;
            }
            __nanosleep(sleep_ns);
            sleep_ns = min(sleep_ns * 2u, max_sleep);
        } else {
            spin_t0 = 0;
            sleep_ns = 32;
        }
    }
}

__device__ __forceinline__ void set_lane(Lane &L, const GenArgs &a)
{
    L.g = L.lane / a.d;
    L.slot = L.lane - L.g * a.d;
    L.used = L.lane < a.groups * a.d;
    L.gmask = L.used ? (a.d == 32 ? kFull : (((1u << a.d) - 1u) << (L.g * a.d))) : 0u;
}

template <typename Id, bool Slots, uint32_t MinBlocks>
__global__ void __launch_bounds__(kThreads, MinBlocks) start_kernel(const StartArgs b)
{
    __shared__ GenArgs s_args[kThreads / 32];
    // per warp: the (level, graph) segment of its last claim, [lo, hi) and the
    // local unit of lo -- a warp's claims T, T + 8, ... mostly stay inside one,
    // and the two searches of map_unit cost as much as a tile's own work
    __shared__ unsigned long long s_seg[kThreads / 32][3];
    const uint32_t warp = threadIdx.x >> 5;
    GenArgs &a = s_args[warp];
    if ((threadIdx.x & 31u) == 0) {
        s_seg[warp][0] = 1;   // empty segment
        s_seg[warp][1] = 0;
    }
    __syncwarp();

    Lane L;
    L.lane = threadIdx.x & 31u;
    L.lt = lanemask_lt();
    L.le = L.lt | (1u << L.lane);
    uint32_t cur = 0xffffffffu;
    if (b.count == 1) {
        if (L.lane == 0) a = b.one;
        __syncwarp();
        set_lane(L, a);
        cur = 0;
    }

    if (!Slots && b.write_seeds) {
        // closed forms; nothing reads them back (SLOTS does not store them)
        const uint32_t gw = blockIdx.x * (kThreads / 32) + warp;
        const uint32_t nw = gridDim.x * (kThreads / 32);
        for (uint32_t i = gw; i < b.count; i += nw) {
            const GenArgs *ai = b.count == 1 ? &a : b.inst + i;
            Id *Ei = reinterpret_cast<Id *>(ai->edges);
            const uint32_t di = ai->d, mode = ai->seed_mode;
            const uint64_t se = ai->seed_edges;
            for (uint64_t e = L.lane; e < se; e += 32) {
                uint64_t src, dst;
                seed_edge(e, di, mode, src, dst);
                st_pair(Ei + 2 * e, src, dst);
            }
        }
    }

    uint32_t n_retry = 0, n_wait = 0, n_pend = 0, n_poll = 0;
    bool ok = true;
    // Counter `warp` hands out tiles warp, warp + 8, ... in increasing order.
    // Let T* be the lowest unfinished tile.  If it is claimed, its warp is
    // working on it (a warp holds one tile at a time) and every tile it reads
    // is lower, hence finished: it progresses.  If not, every tile its counter has handed out is lower,
    // hence finished, so the warps of that counter are free and the next of
    // them to claim takes T*.  Any resident block has a warp on every counter,
    // so this holds for any grid.
    unsigned long long *my_ticket = b.ticket + 16 * warp;
    while (ok) {
        unsigned long long c = 0;
        if (L.lane == 0) c = atomicAdd(my_ticket, 1ull);
        c = __shfl_sync(kFull, c, 0);
        const unsigned long long T = c * kStartCounters + warp;
        if (T >= b.t_end) break;
        uint32_t i = 0;
        uint64_t t = T;
        if (b.count != 1) {
            const unsigned long long lo = s_seg[warp][0], hi = s_seg[warp][1];
            if (T >= lo && T < hi) {
                i = cur;   // the segment's graph is the one loaded
                t = s_seg[warp][2] + (T - lo);
            } else {
                unsigned long long nlo, nhi, t0;
                map_unit_seg(b.tab, b.count, T, i, nlo, nhi, t0);
                t = t0 + (T - nlo);
                __syncwarp();
                if (L.lane == 0) {
                    s_seg[warp][0] = nlo;
                    s_seg[warp][1] = nhi;
                    s_seg[warp][2] = t0;
                }
                __syncwarp();
            }
        }
        if (i != cur) {
            __syncwarp();
            const uint32_t *src = reinterpret_cast<const uint32_t *>(b.inst + i);
            uint32_t *dst = reinterpret_cast<uint32_t *>(&a);
            for (uint32_t w = L.lane; w < sizeof(GenArgs) / 4; w += 32) dst[w] = __ldg(src + w);
            __syncwarp();
            cur = i;
            set_lane(L, a);
        }
        Id *E = reinterpret_cast<Id *>(a.edges);
        const uint32_t tb = (uint32_t)(a.u_first + t * (kStartPasses * a.groups));
        Slot<uint32_t> s[kStartPasses];
#pragma unroll
        for (int j = 0; j < kStartPasses; ++j) {
            const uint32_t pbase = tb + j * a.groups;
            const uint32_t u = pbase + L.g;
            s[j].val = 0;
            s[j].meta = ST_KNOWN;
            if (L.used && u < a.start_end)
                classify_start<Id, Slots>(s[j], draw<uint32_t>(u, L.slot, 0u, a), 0u, a, E, pbase,
                                          n_pend);
        }
        ok = resolve_start<Id, Slots>(s, a, E, tb, a.withhold_first && t == 0, L, n_retry, n_wait, n_pend,
                               n_poll);
    }

#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_retry += __shfl_down_sync(kFull, n_retry, o);
        n_pend += __shfl_down_sync(kFull, n_pend, o);
        n_poll += __shfl_down_sync(kFull, n_poll, o);
    }
    if (L.lane == 0) {
        if (n_pend) atomicAdd(&b.ctl->pending_reads, (unsigned long long)n_pend);
        if (n_poll) atomicAdd(&b.ctl->pending_polls, (unsigned long long)n_poll);
        if (n_retry) atomicAdd(&b.ctl->retries, (unsigned long long)n_retry);
        if (n_wait) atomicAdd(&b.ctl->waits, (unsigned long long)n_wait);
    }
}

// All-ones over the start-region pairs of graph blockIdx.y (+ y0), 16 bytes per
// store.  Pair regions start 16-byte aligned for 64-bit ids; for 32-bit ids the
// region's ragged 8-byte ends are written separately.
__global__ void fill_start_kernel(const GenArgs *inst, uint32_t y0, uint32_t id_bytes)
{
    const GenArgs &a = inst[y0 + blockIdx.y];
    const uint64_t pair_bytes = 2ull * id_bytes;
    const uint64_t n_pairs = (a.start_end - a.u_first) * a.d;
    unsigned char *base = reinterpret_cast<unsigned char *>(a.edges) + a.seed_edges * pair_bytes;
    uint64_t lo = 0, hi = n_pairs * pair_bytes;
    if (hi == 0) return;
    const uint64_t mis = reinterpret_cast<uintptr_t>(base) & 15u;   // 0 or 8
    if (mis) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            *reinterpret_cast<unsigned long long *>(base) = ~0ull;
        lo = 16 - mis;
    }
    if ((hi - lo) & 15u) {
        if (blockIdx.x == 0 && threadIdx.x == 0)
            *reinterpret_cast<unsigned long long *>(base + hi - 8) = ~0ull;
        hi -= 8;
    }
    uint4 *p = reinterpret_cast<uint4 *>(base + lo);
    const uint64_t n16 = (hi - lo) >> 4;
    const uint4 ones = make_uint4(~0u, ~0u, ~0u, ~0u);
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n16;
         x += (uint64_t)gridDim.x * blockDim.x)
        p[x] = ones;
}

template <typename Id, bool Slots, uint32_t MinBlocks>
int launch_start_t(const StartArgs &b, uint32_t blocks, cudaStream_t s)
{
    auto kern = start_kernel<Id, Slots, MinBlocks>;
    if (blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)kThreads, 0);
        if (e != cudaSuccess) return set_cuda_error(e);
        uint64_t g = (uint64_t)sms * (uint64_t)(per_sm > 0 ? per_sm : 1);
        // no more warps than start tiles (but one block at least, for the seed edges)
        const uint64_t need = (b.t_end + kThreads / 32 - 1) / (kThreads / 32);
        if (need < g) g = need > 0 ? need : 1;
        blocks = (uint32_t)g;
    }
    kern<<<blocks, kThreads, 0, s>>>(b);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

}  // namespace

template <uint32_t MinBlocks>
int launch_start_m(uint32_t id_bytes, const StartArgs &b, uint32_t blocks, cudaStream_t s,
                   bool slots)
{
    if (slots)
        return id_bytes == 8 ? launch_start_t<int64_t, true, MinBlocks>(b, blocks, s)
                             : launch_start_t<int32_t, true, MinBlocks>(b, blocks, s);
    return id_bytes == 8 ? launch_start_t<int64_t, false, MinBlocks>(b, blocks, s)
                         : launch_start_t<int32_t, false, MinBlocks>(b, blocks, s);
}

int launch_start(uint32_t id_bytes, const StartArgs &b, uint32_t blocks, cudaStream_t s,
                 bool slots, uint32_t min_blocks)
{
    if (min_blocks == kStartMinBlocksCopy)
        return launch_start_m<kStartMinBlocksCopy>(id_bytes, b, blocks, s, slots);
    if (min_blocks == kStartMinBlocksSmall)
        return launch_start_m<kStartMinBlocksSmall>(id_bytes, b, blocks, s, slots);
    return launch_start_m<kStartMinBlocks>(id_bytes, b, blocks, s, slots);
}

int fill_start(uint32_t id_bytes, const GenArgs *d_inst, uint32_t count, uint64_t max_pairs,
               cudaStream_t s)
{
    if (count == 0 || max_pairs == 0) return PA_OK;
    const uint64_t n16 = max_pairs * 2ull * id_bytes / 16 + 1;
    const uint32_t gx = (uint32_t)std::min<uint64_t>(4096, (n16 + 255) / 256);
    for (uint32_t y0 = 0; y0 < count; y0 += 65535) {
        const uint32_t gy = std::min<uint32_t>(65535, count - y0);
        fill_start_kernel<<<dim3(gx, gy), 256, 0, s>>>(d_inst, y0, id_bytes);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    return PA_OK;
}

}  // namespace gen
}  // namespace pa
