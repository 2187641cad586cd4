// pa_wide.cu -- graphs whose nodes have more than 32 edges (32 < d <= 32767).
//
// The reference keeps each node's slots in a per-node unique set with up to M
// entries, M an int16 EdgeIndexType (cuBSTVertex::insertItem,
// src/Graph/Vertex/CUDA/cuBSTVertex.cuh:153-217; src/Common/DataTypes.h:11-28).
// For d <= 32 the start kernel holds a node's set in the lanes of a warp; here a
// node has more slots than a warp has lanes, so:
//
//  * one warp generates one node at a time, its slots 32 at a time (chunk c =
//    slots 32c .. 32c+31, lane = slot - 32c);
//  * the final values of the node's earlier chunks sit in a per-warp
//    open-addressing hash set in shared memory; a candidate found there is
//    rejected at once (every slot it is compared with is final);
//  * within a chunk the lanes resolve as the start kernel's do: a lane is
//    final when every lower lane is known and distinct and its own candidate
//    differs from theirs (__match_any_sync + ballots), and a candidate equal to
//    a final lower lane is redrawn;
//  * a copy read of slot (v, k) re-reads it while it holds the all-ones fill
//    (the slot-granular completion of the start kernel: the value is its own
//    flag), and every slot is stored the moment it is final;
//  * the first candidate (retry 0) of every slot of the node is drawn and read
//    before the chunks are resolved (kept in shared memory beside the set, up
//    to d = 8192), so the chunks' copy reads are in flight together.
//
// The draws (Philox counter (u_lo, u_hi, slot, retry)), the slot order and the
// rejection rule are the start kernel's, so the output is bit-identical to the
// sequential definition (src/PA/SPA/SerialCopyModel3.cpp:52-78 with Philox
// draws) for any d.  Nodes are claimed in increasing order from one counter; a
// warp holds one node and waits only on lower nodes, so the lowest unfinished
// node always progresses, for any grid.  Every wait is bounded by
// spin_limit_ns.
//
// Also here: canonical rows and CSR out parts of such graphs (each row ranked
// by one warp from a copy in shared memory), for d <= kWideRankMaxD.
#include <algorithm>

#include "pa_gen_core.cuh"
#include "pa_wide.h"

namespace pa {
namespace gen {
namespace {

constexpr uint32_t kEmpty = 0xffffffffu;   // never a node id (ids are below 2^31)

template <typename Id>
struct WideSentinel {
    static constexpr uint64_t value = sizeof(Id) == 8 ? ~0ull : 0xffffffffull;
};

__device__ __forceinline__ uint32_t set_hash(uint32_t x, uint32_t cap_log2)
{
    return (x * 0x9E3779B1u) >> (32 - cap_log2);
}

__device__ __forceinline__ bool set_contains(const uint32_t *set, uint32_t cap_log2, uint32_t x)
{
    const uint32_t mask = (1u << cap_log2) - 1u;
    for (uint32_t h = set_hash(x, cap_log2);; h = (h + 1) & mask) {
        const uint32_t y = set[h];
        if (y == x) return true;
        if (y == kEmpty) return false;
    }
}

__device__ __forceinline__ void set_insert(uint32_t *set, uint32_t cap_log2, uint32_t x)
{
    const uint32_t mask = (1u << cap_log2) - 1u;
    for (uint32_t h = set_hash(x, cap_log2);; h = (h + 1) & mask) {
        const uint32_t old = atomicCAS(set + h, kEmpty, x);
        if (old == kEmpty || old == x) return;
    }
}

// State of one lane's slot: its candidate (or the pending source node), the
// source slot k of a pending copy read, its retry, and whether it is known.
struct WSlot {
    uint32_t val, k, r;
    bool known;
};

// A fresh draw of slot i of node u at retry r.
template <typename Id, bool Slots>
__device__ __forceinline__ void wide_classify(WSlot &s, uint32_t u, uint32_t i, uint32_t r,
                                              const GenArgs &a, const Id *E, uint32_t &n_pend)
{
    const DrawT<uint32_t> dr = draw<uint32_t>(u, i, r, a);
    s.r = r;
    s.k = dr.k;
    s.known = true;
    if (dr.direct) {
        s.val = dr.v;
    } else if (dr.v <= a.d) {
        s.val = (uint32_t)seed_slot(dr.v, dr.k, a.d, a.seed_mode);
    } else {
        const uint64_t x = ld_slot(slot_addr<Id, uint32_t, Slots>(E, a, dr.v, dr.k));
        if (x != WideSentinel<Id>::value) {
            s.val = (uint32_t)x;
        } else {
            s.val = dr.v;
            s.known = false;
            ++n_pend;
        }
    }
}

// Retry-0 candidates of all of a node's slots, fetched before its chunks are
// resolved: the draws do not depend on the resolution, so the copy reads of
// every chunk are in flight together instead of one chunk's at a time.  kPre
// slots per lane are drawn, then their reads issued, then classified.
template <typename Id, bool Slots>
__device__ __forceinline__ void wide_prefetch(uint32_t *pre_val, uint32_t *pre_meta, uint32_t u,
                                              const GenArgs &a, const Id *E, uint32_t lane,
                                              uint32_t &n_pend)
{
    constexpr uint32_t kPre = 4;
    const uint32_t d = a.d;
    for (uint32_t i0 = lane; i0 < d; i0 += 32 * kPre) {
        DrawT<uint32_t> dr[kPre];
        uint64_t x[kPre];
#pragma unroll
        for (uint32_t q = 0; q < kPre; ++q) {
            const uint32_t i = i0 + 32 * q;
            if (i < d) dr[q] = draw<uint32_t>(u, i, 0u, a);
        }
#pragma unroll
        for (uint32_t q = 0; q < kPre; ++q) {
            const uint32_t i = i0 + 32 * q;
            x[q] = 0;
            if (i < d && !dr[q].direct && dr[q].v > d)
                x[q] = ld_slot(slot_addr<Id, uint32_t, Slots>(E, a, dr[q].v, dr[q].k));
        }
#pragma unroll
        for (uint32_t q = 0; q < kPre; ++q) {
            const uint32_t i = i0 + 32 * q;
            if (i >= d) continue;
            uint32_t val, known = 1u;
            if (dr[q].direct) {
                val = dr[q].v;
            } else if (dr[q].v <= d) {
                val = (uint32_t)seed_slot(dr[q].v, dr[q].k, d, a.seed_mode);
            } else if (x[q] != WideSentinel<Id>::value) {
                val = (uint32_t)x[q];
            } else {
                val = dr[q].v;   // pending: polled while its chunk is resolved
                known = 0u;
                ++n_pend;
            }
            pre_val[i] = val;
            pre_meta[i] = dr[q].k | (known << 31);
        }
    }
}

template <typename Id, bool Slots>
__global__ void wide_kernel(const GenArgs a, unsigned long long *ticket, uint32_t cap_log2,
                            uint32_t write_seeds, uint32_t prefetch)
{
    extern __shared__ uint32_t wide_smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t cap = 1u << cap_log2;
    // per warp: the hash set, then (with prefetch) each slot's retry-0 candidate
    // and its source slot k with a known bit
    const size_t warp_words = cap + (prefetch ? 2ull * a.d : 0ull);
    uint32_t *set = wide_smem + (size_t)warp * warp_words;
    uint32_t *pre_val = set + cap;
    uint32_t *pre_meta = pre_val + a.d;
    const uint32_t lt = lanemask_lt(), le = lt | (1u << lane);
    const uint32_t d = a.d;
    Id *E = reinterpret_cast<Id *>(a.edges);
    const uint32_t gw = blockIdx.x * (blockDim.x >> 5) + warp;
    const uint32_t nw = gridDim.x * (blockDim.x >> 5);

    if (!Slots && write_seeds) {
        for (uint64_t e = (uint64_t)gw * 32 + lane; e < a.seed_edges; e += (uint64_t)nw * 32) {
            uint64_t src, dst;
            seed_edge(e, d, a.seed_mode, src, dst);
            st_pair(E + 2 * e, src, dst);
        }
    }

    uint32_t n_retry = 0, n_wait = 0, n_pend = 0, n_poll = 0;
    const uint32_t max_sleep = min(a.max_sleep_ns, 512u);
    bool ok = true;
    while (ok) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(ticket, 1ull);
        c = __shfl_sync(kFull, c, 0);
        const uint64_t u64 = a.u_first + c;
        if (u64 >= a.start_end) break;
        const uint32_t u = (uint32_t)u64;
        const uint64_t row = c;
        const bool withhold = a.withhold_first && row == 0;
        __syncwarp();
        for (uint32_t x = lane; x < cap; x += 32) set[x] = kEmpty;
        if (prefetch) wide_prefetch<Id, Slots>(pre_val, pre_meta, u, a, E, lane, n_pend);
        __syncwarp();
        for (uint32_t c0 = 0; c0 < d && ok; c0 += 32) {
            const uint32_t i = c0 + lane;
            const bool active = i < d;
            WSlot s{0u, 0u, 0u, true};
            if (active && prefetch) {
                const uint32_t m = pre_meta[i];
                s.val = pre_val[i];
                s.k = m & 0x7fffffffu;
                s.known = (m >> 31) != 0u;
            } else if (active) {
                wide_classify<Id, Slots>(s, u, i, 0u, a, E, n_pend);
            }
            bool stored = !active;
            const uint64_t e = a.seed_edges + row * d + i;
            uint64_t spin_t0 = 0;
            uint32_t sleep_ns = 32;
            for (;;) {
                bool changed = false;
                if (active && !s.known) {
                    const uint64_t x = ld_slot(slot_addr<Id, uint32_t, Slots>(E, a, s.val, s.k));
                    if (x != WideSentinel<Id>::value) {
                        s.val = (uint32_t)x;
                        s.known = true;
                        changed = true;
                    } else {
                        ++n_poll;
                    }
                }
                // a candidate among the earlier chunks' final values is rejected
                // now, as often as it takes (every value in the set is final)
                while (active && s.known && set_contains(set, cap_log2, s.val)) {
                    wide_classify<Id, Slots>(s, u, i, s.r + 1u, a, E, n_pend);
                    ++n_retry;
                    changed = true;
                }
                const bool known = active && s.known;
                const uint32_t eq = __match_any_sync(kFull, known ? s.val : (0xffffffe0u | lane));
                const bool bad = active && (!known || (eq & lt) != 0u);
                const uint32_t badm = __ballot_sync(kFull, bad);
                const bool fin = active && (badm & le) == 0u;
                if (fin && !stored) {
                    if (!withhold) {
                        if constexpr (Slots) st_relaxed_id(E + e, s.val);
                        else st_relaxed_pair(E + 2 * e, u, s.val);
                    }
                    stored = true;
                }
                const uint32_t finm = __ballot_sync(kFull, fin || !active);
                if (finm == kFull) break;
                // a candidate equal to a final lower slot of the chunk is rejected
                if (known && !fin && (eq & lt & finm) != 0u) {
                    wide_classify<Id, Slots>(s, u, i, s.r + 1u, a, E, n_pend);
                    ++n_retry;
                    changed = true;
                }
                if (!__any_sync(kFull, changed)) {
                    unsigned long long now = 0;
                    uint32_t err = 0;
                    if (lane == 0) {
                        now = globaltimer_ns();
                        err = ld_relaxed_u32(&my_rep(a)->error);
                        ++n_wait;
                    }
                    now = __shfl_sync(kFull, now, 0);
                    err = __shfl_sync(kFull, err, 0);
                    if (err != 0) {
                        ok = false;
                        break;
                    }
                    if (spin_t0 == 0) spin_t0 = now;
                    if (now - spin_t0 > a.spin_limit_ns) {
                        if (lane == 0) raise_error(a, (uint32_t)PA_ERR_SPIN_TIMEOUT);
                        ok = false;
                        break;
                    }
                    __nanosleep(sleep_ns);
                    sleep_ns = min(sleep_ns * 2u, max_sleep);
                } else {
                    spin_t0 = 0;
                    sleep_ns = 32;
                }
            }
            // the chunk's final values join the node's set
            if (ok && active) set_insert(set, cap_log2, s.val);
            __syncwarp();
        }
    }

#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_retry += __shfl_down_sync(kFull, n_retry, o);
        n_pend += __shfl_down_sync(kFull, n_pend, o);
        n_poll += __shfl_down_sync(kFull, n_poll, o);
    }
    if (lane == 0) {
        if (n_pend) atomicAdd(&a.ctl->pending_reads, (unsigned long long)n_pend);
        if (n_poll) atomicAdd(&a.ctl->pending_polls, (unsigned long long)n_poll);
        if (n_retry) atomicAdd(&a.ctl->retries, (unsigned long long)n_retry);
        if (n_wait) atomicAdd(&a.ctl->waits, (unsigned long long)n_wait);
    }
}

// Slots of the hash set of one warp: a power of two holding every value of a
// node but the last chunk's with at least one slot empty, at most half full
// while that fits kWideSetMaxBytes.
uint32_t set_cap_log2(uint32_t d)
{
    uint32_t lg = 5;
    while ((1u << lg) < 2u * d && (4u << (lg + 1)) <= kWideSetMaxBytes) ++lg;
    while ((1u << lg) <= d) ++lg;   // d <= 32767: at most 2^15 slots, 128 KB
    return lg;
}

template <typename Id, bool Slots>
int launch_wide_t(const GenArgs &a, unsigned long long *ticket, uint32_t blocks, cudaStream_t s)
{
    const uint32_t lg = set_cap_log2(a.d);
    // fetch every slot's first candidate up front when it fits beside the set
    const bool prefetch = (4ull << lg) + 8ull * a.d <= kWideSetMaxBytes;
    const size_t warp_bytes = (4ull << lg) + (prefetch ? 8ull * a.d : 0ull);
    const uint32_t warps = (uint32_t)std::max<size_t>(
        1, std::min<size_t>(8, kWideBlockSetBytes / warp_bytes));
    const size_t smem = warp_bytes * warps;
    auto kern = wide_kernel<Id, Slots>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (blocks == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        e = cudaGetDevice(&dev);
        if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess)
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)(32 * warps), smem);
        if (e != cudaSuccess) return set_cuda_error(e);
        uint64_t g = (uint64_t)sms * (uint64_t)(per_sm > 0 ? per_sm : 1);
        const uint64_t nodes = a.start_end - a.u_first;
        const uint64_t need = (nodes + warps - 1) / warps;
        if (need < g) g = need > 0 ? need : 1;
        blocks = (uint32_t)g;
    }
    kern<<<blocks, 32 * warps, smem, s>>>(a, ticket, lg, 1u, prefetch ? 1u : 0u);
    e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

// ---------------------------------------------------------------------------
// Row ranking for d > 32: one warp per generated row, the row's targets copied
// to shared memory first, each lane ranking its slots against the copy (the
// values of a row are distinct).  rows_out: canonical pairs (src, dst sorted);
// CSR: the targets at rowptr[row] + rank.
// ---------------------------------------------------------------------------
template <typename Id, bool Csr>
__global__ void rank_rows_wide_kernel(const Id *E, Id *out, const int64_t *rowptr, uint64_t n,
                                      uint32_t d, uint64_t seed_edges, uint64_t out_len)
{
    extern __shared__ unsigned char rank_smem[];
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    Id *rowbuf = reinterpret_cast<Id *>(rank_smem) + (size_t)warp * d;
    const uint64_t rows = n - (d + 1);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + warp;
    const uint64_t nw = (uint64_t)gridDim.x * (blockDim.x >> 5);
    if (!Csr && E != out)
        for (uint64_t e = w0 * 32 + lane; e < seed_edges; e += nw * 32) {
            out[2 * e] = E[2 * e];
            out[2 * e + 1] = E[2 * e + 1];
        }
    for (uint64_t row = w0; row < rows; row += nw) {
        const uint64_t e0 = seed_edges + row * d;
        __syncwarp();
        for (uint32_t i = lane; i < d; i += 32) rowbuf[i] = E[2 * (e0 + i) + 1];
        __syncwarp();
        const uint64_t base = Csr ? (uint64_t)rowptr[row + d + 1] : e0;
        for (uint32_t i = lane; i < d; i += 32) {
            const Id x = rowbuf[i];
            uint32_t rank = 0;
            for (uint32_t j = 0; j < d; ++j) rank += rowbuf[j] < x ? 1u : 0u;
            if constexpr (Csr) {
                if (base + rank < out_len) out[base + rank] = x;
            } else {
                out[2 * (base + rank)] = (Id)(row + d + 1);
                out[2 * (base + rank) + 1] = x;
            }
        }
    }
}

template <typename Id, bool Csr>
int launch_rank_t(const Id *E, Id *out, const int64_t *rowptr, uint64_t n, uint32_t d,
                  uint64_t seed_edges, uint64_t out_len, cudaStream_t s)
{
    const uint32_t warps = (uint32_t)std::max<uint64_t>(
        1, std::min<uint64_t>(8, kWideBlockSetBytes / ((uint64_t)d * sizeof(Id))));
    const size_t smem = (size_t)warps * d * sizeof(Id);
    auto kern = rank_rows_wide_kernel<Id, Csr>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_cuda_error(e);
    int dev = 0, sms = 0;
    e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return set_cuda_error(e);
    const uint64_t rows = n - (d + 1);
    uint64_t blocks = std::min<uint64_t>((uint64_t)sms * 4, (rows + warps - 1) / warps);
    if (blocks == 0) blocks = 1;
    kern<<<(unsigned)blocks, 32 * warps, smem, s>>>(E, out, rowptr, n, d, seed_edges, out_len);
    e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

}  // namespace

int launch_wide(uint32_t id_bytes, bool slots, const GenArgs &a, unsigned long long *ticket,
                uint32_t blocks, cudaStream_t s)
{
    if (slots)
        return id_bytes == 8 ? launch_wide_t<int64_t, true>(a, ticket, blocks, s)
                             : launch_wide_t<int32_t, true>(a, ticket, blocks, s);
    return id_bytes == 8 ? launch_wide_t<int64_t, false>(a, ticket, blocks, s)
                         : launch_wide_t<int32_t, false>(a, ticket, blocks, s);
}

int canon_wide(uint32_t id_bytes, const void *E, void *out, uint64_t n, uint32_t d,
               uint64_t seed_edges, cudaStream_t s)
{
    if (d > kWideRankMaxD) return PA_ERR_NOT_SUPPORTED;
    if (id_bytes == 8)
        return launch_rank_t<int64_t, false>((const int64_t *)E, (int64_t *)out, nullptr, n, d,
                                             seed_edges, 0, s);
    return launch_rank_t<int32_t, false>((const int32_t *)E, (int32_t *)out, nullptr, n, d,
                                         seed_edges, 0, s);
}

int csr_out_wide(uint32_t id_bytes, const void *E, const int64_t *rowptr, void *col, uint64_t n,
                 uint32_t d, uint64_t seed_edges, uint64_t col_len, cudaStream_t s)
{
    if (d > kWideRankMaxD) return PA_ERR_NOT_SUPPORTED;
    if (id_bytes == 8)
        return launch_rank_t<int64_t, true>((const int64_t *)E, (int64_t *)col, rowptr, n, d,
                                            seed_edges, col_len, s);
    return launch_rank_t<int32_t, true>((const int32_t *)E, (int32_t *)col, rowptr, n, d,
                                        seed_edges, col_len, s);
}

}  // namespace gen
}  // namespace pa
