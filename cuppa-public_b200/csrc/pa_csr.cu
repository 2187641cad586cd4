// pa_csr.cu -- undirected CSR of a generated graph: every edge in both rows,
// every row sorted ascending.  No reference counterpart (the reference never
// hands its graph out); the degree pass is the device side of
// src/PA/cuPPA/cuPPA.cu:103-165.
//
// Row x is [x's own targets, all < x, ascending] ++ [x's in-neighbours, all > x,
// ascending], so it comes out sorted when both parts are:
//   1. in parts: the pairs, taken as (destination, source) items, are sorted by
//      destination with a stable LSD radix sort; the pairs are in source order,
//      so every destination's sources come out ascending, back to back;
//   2. rowptr[x] = (out entries of rows below x: a closed form) + (items with
//      destination below x: read off the run boundaries of the sorted items);
//   3. in part entries: sorted item i with destination v goes to position
//      outprefix(v + 1) + i;
//   4. out part: each generated row's d targets ranked in registers and stored;
//      the seed rows' targets are 0, 1, ... (both seed graphs).
// Steps 3 and 4 run in one row writer for d <= 32 (a warp writes 32 whole
// rows), with the in parts of hub rows copied in pieces spread over all warps.
// Items pack (v, u) in 8 bytes, so graphs of 2^32 nodes and more are refused.
//
// The sort reads the pairs once and the items twice per pass: one histogram
// kernel counts the digits of every pass while it turns the pairs into items,
// and each pass is one kernel that keeps its tile on chip from the load to the
// store, taking each digit's offset from the tiles before it by decoupled
// look-back (Merrill and Garland's single-pass prefix scan, as in Adinets and
// Merrill's one-sweep radix sort) instead of a per-pass histogram and scan.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "pa_device.cuh"
#include "pa_internal.h"
#include "pa_wide.h"

namespace pa {
namespace {

constexpr uint32_t kFull = 0xffffffffu;
// ---------------------------------------------------------------------------
// Seed rows' out parts for the path of d > 32 (rows_kernel writes them for
// d <= 32; csr_out_wide writes the generated rows): the seed rows' out-edges go
// to targets 0, 1, ... in order in both seed graphs (CLIQUE row v: 0..v-1;
// STAR_REF row d: 0..d-1), so an edge's position in its row is its target.
// ---------------------------------------------------------------------------
template <typename Id>
__global__ void seed_out_part_kernel(const Id *E, const int64_t *rowptr, Id *col, uint64_t n,
                                     uint64_t seed_edges, uint64_t col_len)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < seed_edges; e += stride) {
        const uint64_t u = (uint64_t)E[2 * e], t = (uint64_t)E[2 * e + 1];
        if (u < n && t < u) {
            const uint64_t pos = (uint64_t)rowptr[u] + t;
            if (pos < col_len) col[pos] = E[2 * e + 1];
        }
    }
}

// Out-degree of each seed node: CLIQUE row v holds v edges (to 0..v-1),
// STAR_REF node d holds d (to 0..d-1).
__global__ void seed_out_kernel(uint32_t d, uint32_t seed_mode, uint32_t *seed_out)
{
    for (uint32_t v = threadIdx.x; v <= d; v += blockDim.x)
        seed_out[v] = seed_mode == PA_SEED_CLIQUE ? v : (v == d ? d : 0u);
}

// ---------------------------------------------------------------------------
// Sorted in parts by a stable LSD radix sort (graphs below 2^32 nodes).
//
// Item = (destination v) << 32 | (source u), one per pair.  The pairs are in
// non-decreasing source order (seed rows, then node d+1, d+2, ...), so a
// stable sort by v leaves every v's sources ascending: the sorted items are
// the in parts, in order, back to back.  Item i of the sorted array (key v)
// goes to col[outprefix(v + 1) + i], where outprefix(x) is the number of out
// entries of rows below x -- a closed form -- and rowptr[x] = outprefix(x) +
// (number of items with key < x), read off the run boundaries.  No atomics on
// the node range and no per-row sorting.
//
// A pass sorts 8 or 9 key bits (the fewest passes for the key).  Its
// kernel claims tiles of 8192 items in order from a counter; a tile's 512
// threads load 16 items each and park them in shared memory, rank them stably
// -- each of 16 warps walks its 512 items in order, 32 at a time, with
// __match_any_sync for equal digits and 16-bit per-warp counters in shared
// memory -- publish the tile's count of every digit, and look back over the
// tiles before it (their counts, or the running total the nearest finished
// one published) for each digit's global offset.  The tile is then staged in
// shared memory in digit order and every digit's run is written contiguously.
// ---------------------------------------------------------------------------
constexpr uint32_t kRadixThreads = 512, kRadixWarps = kRadixThreads / 32;
constexpr uint32_t kRadixBuckets = 512;   // the widest digit in use: 9 bits
constexpr uint32_t kRadixRounds = 16;     // items per lane per tile
constexpr uint32_t kRadixTile = kRadixThreads * kRadixRounds;
constexpr uint32_t kMaxPasses = 4;
constexpr unsigned long long kBadKey = 0xffffffffull;   // sorts after every node id

// Look-back status word of (tile, digit): bits 63-62 kind (1 = the tile's own
// count, 2 = the running total through the tile), bits 61-56 the pass's epoch
// (a word of another pass reads as not yet published), bits 55-0 the value.
constexpr unsigned long long kLbAgg = 1ull << 62, kLbInc = 2ull << 62;
constexpr unsigned long long kLbValMask = (1ull << 56) - 1;
constexpr uint32_t kLbEpochShift = 56;
constexpr uint32_t kLbWindow = 4;   // predecessors read per look-back step

// Item of pair i (ids above the node range, never produced by the generator,
// become kBadKey and raise an error).
template <typename Id>
__device__ __forceinline__ unsigned long long pair_item(const Id *E, uint64_t i, uint64_t n,
                                                        uint32_t *err)
{
    const uint64_t u = (uint64_t)E[2 * i], v = (uint64_t)E[2 * i + 1];
    if (u >= n || v >= n) {
        atomicCAS(err, 0u, (uint32_t)PA_ERR_INVALID);
        return (kBadKey << 32) | 0xffffffffull;
    }
    return (v << 32) | u;
}

// The items, in pair order, and the digit counts of every pass over them (the
// pairs read once): per-block shared counters, flushed with one global atomic
// per nonzero digit.  (Combining a warp's equal digits with __match_any_sync
// first measured far slower than the shared atomics it saves: 32 against ~5 ms
// at n = 10^8, d = 16.)  Writing the items here lets every pass read 8 bytes
// per item instead of the first one reading the 16-byte pairs.
template <typename Id, uint32_t DB>
__global__ void __launch_bounds__(kRadixThreads) radix_hist_all_kernel(const Id *E, uint64_t n_items,
                                                                       uint64_t n, uint32_t passes,
                                                                       unsigned long long *items,
                                                                       unsigned long long *hist,
                                                                       uint32_t *err)
{
    constexpr uint32_t NB = 1u << DB, MASK = NB - 1;
    __shared__ uint32_t cnt[kMaxPasses * NB];
    for (uint32_t b = threadIdx.x; b < kMaxPasses * NB; b += kRadixThreads) cnt[b] = 0;
    __syncthreads();
    constexpr uint32_t U = 4;   // items per thread per step, loaded together
    const uint64_t stride = (uint64_t)gridDim.x * kRadixThreads * U;
    for (uint64_t base = (uint64_t)blockIdx.x * kRadixThreads * U; base < n_items; base += stride) {
        uint32_t key[U];
#pragma unroll
        for (uint32_t j = 0; j < U; ++j) {
            const uint64_t i = base + j * kRadixThreads + threadIdx.x;
            key[j] = 0u;
            if (i < n_items) {
                const unsigned long long it = pair_item(E, i, n, err);
                items[i] = it;
                key[j] = (uint32_t)(it >> 32);
            }
        }
#pragma unroll
        for (uint32_t j = 0; j < U; ++j) {
            if (base + j * kRadixThreads + threadIdx.x >= n_items) continue;
            for (uint32_t q = 0; q < passes; ++q)
                atomicAdd(&cnt[q * NB + ((key[j] >> (DB * q)) & MASK)], 1u);
        }
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < passes * NB; b += kRadixThreads)
        if (cnt[b]) atomicAdd(hist + b, (unsigned long long)cnt[b]);
}

// Exclusive prefix of each pass's digit counts: base[q*NB + b] = items whose
// pass-q digit is below b.  One block, one thread per pass.
template <uint32_t DB>
__global__ void radix_base_kernel(const unsigned long long *hist, uint32_t passes,
                                  unsigned long long *base)
{
    constexpr uint32_t NB = 1u << DB;
    const uint32_t q = threadIdx.x;
    if (q >= passes) return;
    unsigned long long acc = 0;
    for (uint32_t b = 0; b < NB; ++b) {
        base[q * NB + b] = acc;
        acc += hist[q * NB + b];
    }
}

// Dynamic shared memory of the pass kernel: the tile in digit order, each
// digit's global offset less its start within the tile, the per-warp digit
// counts (then the warps' bases within the tile), the claimed tile.
template <uint32_t NB>
struct RadixSmem {
    unsigned long long stage[kRadixTile];
    unsigned long long goff[NB];
    uint16_t wcnt[kRadixWarps][NB];
    uint32_t wsum[kRadixWarps];
    unsigned long long tile;
};

// Two CTAs per SM (84 KB of shared memory each at 9-bit digits, 64 registers).
// Measured at n = 2^30, d = 4 (C3 CSR) and n = 10^8, d = 16 (C2): 8,192-item
// tiles at two CTAs 224-227 / 75.6 ms; 6,144-item tiles at three CTAs and 40
// registers (which spill) 231 / 76.0 ms; 7,168, 9,216 and 10,240-item tiles at
// two CTAs 231 / 74.2, 238 / 76.8 and 241 / 77.1 ms.
template <uint32_t DB>
__global__ void __launch_bounds__(kRadixThreads, 2) radix_pass_kernel(
    const unsigned long long *src, unsigned long long *dst, uint64_t n_items, uint32_t shift,
    const unsigned long long *digit_base, unsigned long long *status, uint32_t epoch,
    unsigned long long *tile_ctr, uint64_t spin_limit_ns, uint32_t *err)
{
    constexpr uint32_t NB = 1u << DB, MASK = NB - 1;
    // digits per thread in the per-digit steps (10-bit digits: two)
    constexpr uint32_t DPT = NB > kRadixThreads ? NB / kRadixThreads : 1;
    static_assert(NB <= kRadixBuckets && DPT * kRadixThreads >= NB, "digit width");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RadixSmem<NB> &S = *reinterpret_cast<RadixSmem<NB> *>(smem_raw);
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31u;
    const uint32_t lt = lanemask_lt();
    const bool owner = tid * DPT < NB;
    for (uint32_t w = 0; w < kRadixWarps; ++w)
        for (uint32_t b = tid; b < NB; b += kRadixThreads) S.wcnt[w][b] = 0;
    if (tid == 0) S.tile = atomicAdd(tile_ctr, 1ull);
    __syncthreads();
    const uint64_t t = S.tile;
    const uint64_t tb = t * kRadixTile;
    const uint32_t tcount = (uint32_t)min((uint64_t)kRadixTile, n_items - tb);
    const uint32_t wo = warp * (kRadixRounds * 32);

    // 1. the tile's items, loaded together, parked in the stage in their own
    // order (conflict-free); only their digits stay in registers through the
    // ranking and the look-back, which keeps the kernel free of spills
    uint32_t dgp[kRadixRounds / 2];   // two digits per register
    // loaded in two halves: all of a thread's items at once spill registers
#pragma unroll
    for (uint32_t h = 0; h < kRadixRounds; h += kRadixRounds / 2) {
        unsigned long long its[kRadixRounds / 2];
#pragma unroll
        for (uint32_t q = 0; q < kRadixRounds / 2; ++q) {
            const uint32_t k = wo + (h + q) * 32 + lane;
            its[q] = k < tcount ? src[tb + k] : 0ull;
        }
#pragma unroll
        for (uint32_t q = 0; q < kRadixRounds / 2; ++q) {
            const uint32_t r = h + q;
            const uint32_t k = wo + r * 32 + lane;
            S.stage[k] = its[q];
            const uint32_t dg = k < tcount ? (uint32_t)(its[q] >> (32 + shift)) & MASK : NB + lane;
            if (r & 1) dgp[r / 2] |= dg << 16;
            else dgp[r / 2] = dg;
        }
    }
    // stable ranks within the warp's items (in order, 32 per round); two ranks
    // per register
    uint32_t rk[kRadixRounds / 2];
#pragma unroll
    for (uint32_t r = 0; r < kRadixRounds; ++r) {
        const uint32_t k = wo + r * 32 + lane;
        const bool valid = k < tcount;
        const uint32_t dg = (dgp[r / 2] >> ((r & 1) * 16)) & 0xffffu;
        const uint32_t peers = __match_any_sync(kFull, dg);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (valid && lane == leader) {
            old = S.wcnt[warp][dg];
            S.wcnt[warp][dg] = (uint16_t)(old + __popc(peers));
        }
        old = __shfl_sync(kFull, old, leader);
        const uint32_t rank = old + __popc(peers & lt);
        if (r & 1) rk[r / 2] |= rank << 16;
        else rk[r / 2] = rank;
        // the next round's leader for a digit may be another lane: order this
        // round's counter stores before the next round's loads
        __syncwarp();
    }
    __syncthreads();

    // 2. thread j owns digits j*DPT .. j*DPT+DPT-1: their warps' bases in warp
    // order and their counts in the tile, published for the tiles after this one
    uint32_t tot[DPT];
#pragma unroll
    for (uint32_t j = 0; j < DPT; ++j) {
        tot[j] = 0;
        if (owner) {
            const uint32_t dig = tid * DPT + j;
            for (uint32_t w = 0; w < kRadixWarps; ++w) {
                const uint32_t c = S.wcnt[w][dig];
                S.wcnt[w][dig] = (uint16_t)tot[j];
                tot[j] += c;
            }
        }
    }
    const unsigned long long ep = (unsigned long long)epoch << kLbEpochShift;
    unsigned long long before[DPT];   // each digit's items in the tiles before t
#pragma unroll
    for (uint32_t j = 0; j < DPT; ++j) before[j] = 0;
    if (owner) {
        unsigned long long *mine = status + t * NB + tid * DPT;
#pragma unroll
        for (uint32_t j = 0; j < DPT; ++j)
            st_relaxed_u64(mine + j, (t == 0 ? kLbInc : kLbAgg) | ep | tot[j]);
        if (t > 0) {
            // 3. look back: add the counts of earlier tiles until one of them
            // carries its running total (bounded wait on tiles not yet ranked).
            // kLbWindow predecessors of each owned digit are read at once: one
            // at a time, the running totals would advance one tile per L2
            // round trip, far slower than tiles are ranked.
            uint64_t p[DPT];   // tiles [p, t) are accounted for
            bool done[DPT];
#pragma unroll
            for (uint32_t j = 0; j < DPT; ++j) {
                p[j] = t;
                done[j] = false;
            }
            const uint64_t t0 = globaltimer_ns();
            while (true) {
                bool open = false;
#pragma unroll
                for (uint32_t j = 0; j < DPT; ++j) open |= !done[j] && p[j] > 0;
                if (!open) break;
                unsigned long long w[DPT][kLbWindow];
#pragma unroll
                for (uint32_t j = 0; j < DPT; ++j)
#pragma unroll
                    for (uint32_t k = 0; k < kLbWindow; ++k)
                        w[j][k] = !done[j] && k < p[j]
                                      ? ld_relaxed_u64(status + (p[j] - 1 - k) * NB + tid * DPT + j)
                                      : 0ull;
                bool waiting = false;
#pragma unroll
                for (uint32_t j = 0; j < DPT; ++j) {
                    uint32_t used = 0;
                    bool stop = done[j];
#pragma unroll
                    for (uint32_t k = 0; k < kLbWindow; ++k) {
                        if (stop || k >= p[j]) continue;
                        const bool ready = (w[j][k] >> 62) != 0 &&
                                           ((w[j][k] >> kLbEpochShift) & 63ull) == epoch;
                        if (!ready) {
                            waiting = true;
                            stop = true;
                            continue;
                        }
                        before[j] += w[j][k] & kLbValMask;
                        ++used;
                        if ((w[j][k] >> 62) == 2) done[j] = stop = true;
                    }
                    p[j] -= used;
                }
                if (waiting) {
                    if (globaltimer_ns() - t0 > spin_limit_ns) {
                        atomicCAS(err, 0u, (uint32_t)PA_ERR_SPIN_TIMEOUT);
                        break;
                    }
                    __nanosleep(32);
                }
            }
#pragma unroll
            for (uint32_t j = 0; j < DPT; ++j)
                st_relaxed_u64(mine + j, kLbInc | ep | (before[j] + tot[j]));
        }
    }
    // 4. digit starts within the tile (exclusive scan of the counts over
    // digits: within the thread, then over threads)
    uint32_t mysum = 0;
#pragma unroll
    for (uint32_t j = 0; j < DPT; ++j) mysum += tot[j];
    uint32_t x = mysum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) S.wsum[warp] = x;
    __syncthreads();
    uint32_t start = x - mysum;
    for (uint32_t w = 0; w < warp; ++w) start += S.wsum[w];
    if (owner) {
#pragma unroll
        for (uint32_t j = 0; j < DPT; ++j) {
            const uint32_t dig = tid * DPT + j;
            for (uint32_t w = 0; w < kRadixWarps; ++w)   // <= tile size: fits 16 bits
                S.wcnt[w][dig] = (uint16_t)(S.wcnt[w][dig] + start);
            // the digit's global start less its start in the tile (the tile's
            // items of smaller digits are counted in digit_base, so this is >= 0)
            S.goff[dig] = digit_base[dig] + before[j] - start;
            start += tot[j];
        }
    }
    __syncthreads();
    // 5. the tile back from its parking place, then into the stage in digit order
    {
        unsigned long long its[kRadixRounds];
#pragma unroll
        for (uint32_t r = 0; r < kRadixRounds; ++r) its[r] = S.stage[wo + r * 32 + lane];
        __syncthreads();
#pragma unroll
        for (uint32_t r = 0; r < kRadixRounds; ++r) {
            const uint32_t k = wo + r * 32 + lane;
            if (k < tcount) {
                const uint32_t dg = (dgp[r / 2] >> ((r & 1) * 16)) & 0xffffu;
                const uint32_t rank = (rk[r / 2] >> ((r & 1) * 16)) & 0xffffu;
                S.stage[S.wcnt[warp][dg] + rank] = its[r];
            }
        }
    }
    __syncthreads();
    // 6. out in digit runs: consecutive threads write consecutive addresses
    for (uint32_t k = tid; k < tcount; k += kRadixThreads) {
        const unsigned long long it = S.stage[k];
        const uint32_t dg = (uint32_t)(it >> (32 + shift)) & MASK;
        dst[S.goff[dg] + k] = it;
    }
}

// Out entries of rows below x: seed rows from their prefix table, then d per row.
__device__ __forceinline__ uint64_t outprefix(uint64_t x, uint32_t d, uint64_t seed_edges,
                                              const int64_t *seed_pre)
{
    return x <= (uint64_t)d + 1 ? (uint64_t)seed_pre[x] : seed_edges + (x - d - 1) * d;
}

// seed_pre[x] = out entries of seed rows below x, x = 0..d+1.
__global__ void seed_prefix_kernel(const uint32_t *seed_out, uint32_t d, int64_t *seed_pre)
{
    if (threadIdx.x == 0) {
        int64_t acc = 0;
        for (uint32_t x = 0; x <= d + 1; ++x) {
            seed_pre[x] = acc;
            if (x <= d) acc += seed_out[x];
        }
    }
}

// One pass over the sorted items (the path of d > 32): rowptr[x] = outprefix(x)
// + #items with key < x is written for every x in (key(i-1), key(i)] (i =
// n_items closes the range up to n; keys >= n -- only after an input error --
// count as n), and in part entry i (key v, value u) goes to
// col[outprefix(v + 1) + i].
// Consecutive threads take consecutive items (coalesced stores); a thread's U
// items of one step are a grid stride apart, their loads issued together.
template <typename Id>
__global__ void in_sorted_kernel(const unsigned long long *items, uint64_t n_items, uint64_t n,
                                 uint32_t d, uint64_t seed_edges, const int64_t *seed_pre, Id *col,
                                 uint64_t col_len, int64_t *rowptr)
{
    constexpr uint32_t U = 4;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 <= n_items;
         i0 += U * stride) {
        unsigned long long it[U], pv[U];
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint64_t i = i0 + q * stride;
            it[q] = i < n_items ? items[i] : ~0ull;
            pv[q] = i > 0 && i <= n_items ? items[i - 1] : ~0ull;
        }
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint64_t i = i0 + q * stride;
            if (i > n_items) break;
            const uint64_t v = i < n_items ? min((uint64_t)(it[q] >> 32), n) : n;
            const uint64_t lo = i > 0 ? min((uint64_t)(pv[q] >> 32), n) + 1 : 0;
            for (uint64_t x = lo; x <= v && x <= n; ++x)
                rowptr[x] = (int64_t)(outprefix(x, d, seed_edges, seed_pre) + i);
            if (i < n_items && v < n) {
                const uint64_t pos = outprefix(v + 1, d, seed_edges, seed_pre) + i;
                if (pos < col_len) col[pos] = (Id)(it[q] & 0xffffffffull);
            }
        }
    }
}

// rowptr alone (the row writer's input): rowptr[x] = outprefix(x) + the first
// position k in [0, n_items] whose key is >= x (key(n_items) = n; keys >= n,
// only after an input error, count as n).  A warp takes 32 * U consecutive
// positions; for each 32 of them it writes rows (key(k0 - 1), key(k0 + 31)]
// one per lane, each from the first lane whose key reaches it (a five-step
// search over the lanes' keys), so a run of rows without in-edges costs one
// coalesced store per row instead of a loop in one lane.
__global__ void __launch_bounds__(256) rowptr_kernel(const unsigned long long *items, uint64_t n_items,
                                                     uint64_t n, uint32_t d, uint64_t seed_edges,
                                                     const int64_t *seed_pre, int64_t *rowptr)
{
    constexpr uint32_t U = 8;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint64_t positions = n_items + 1;
    // keys, rows and the search in 32 bits (n < 2^32); rows beyond key(k) are
    // never written by the lane of k
    const uint32_t n32 = (uint32_t)n;
    for (uint64_t c0 = w0 * 32 * U; c0 < positions; c0 += warps * 32 * U) {
        uint32_t key[U];
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint64_t k = c0 + q * 32 + lane;
            key[q] = k < n_items ? (uint32_t)min(items[k] >> 32, (unsigned long long)n) : n32;
        }
        // the first row not yet written: rows up to key(c0 - 1) belong to the
        // warp holding position c0 - 1
        uint64_t nxt = c0 == 0 ? 0 : min(items[c0 - 1] >> 32, (unsigned long long)n) + 1;
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint64_t kb = c0 + q * 32;
            if (kb >= positions) break;   // warp-uniform
            const uint32_t v = key[q];
            const uint32_t last = __shfl_sync(kFull, v, 31);
            for (uint64_t x0 = nxt; x0 <= last; x0 += 32) {
                const uint64_t x = x0 + lane;
                const uint32_t xs = (uint32_t)min(x, (uint64_t)last);
                uint32_t lo = 0;   // lanes whose key is below x
#pragma unroll
                for (uint32_t step = 16; step > 0; step >>= 1)
                    if (__shfl_sync(kFull, v, lo + step - 1) < xs) lo += step;
                if (x <= last)
                    rowptr[x] = (int64_t)(outprefix(x, d, seed_edges, seed_pre) + kb + lo);
            }
            if ((uint64_t)last + 1 > nxt) nxt = (uint64_t)last + 1;
        }
    }
}

// ---------------------------------------------------------------------------
// Whole rows (d <= 32), once rowptr is known: a warp writes 32 consecutive rows,
// each out part then in part, so every 32-byte sector of col between the
// chunk's first and last entry is written by one warp within a short time.
// (Out parts and in parts written by two kernels share a partial sector at
// every row boundary, which DRAM then reads and writes back twice.)
//
// Row x's in part is sorted items [lb(x), lb(x+1)), lb(x) = rowptr[x] -
// outprefix(x); entry k of it (item index) goes to col[outprefix(x+1) + k].
// A row whose in part is longer than kHeavyIn items is listed here and its in
// part copied in pieces of kPiece items spread over all warps (heavy_scan_kernel,
// heavy_in_kernel), so that hub rows -- up to every item at p = 0 -- hold no
// single warp or block.
// ---------------------------------------------------------------------------
constexpr uint32_t kRowsChunk = 32;        // rows per warp step: one per lane
constexpr uint64_t kHeavyIn = 512;         // longest in part a row warp copies
constexpr uint32_t kPiece = 512;           // items per piece of a longer one

__device__ __forceinline__ uint64_t clamp_items(int64_t v, uint64_t n_items)
{
    return v < 0 ? 0ull : ((uint64_t)v > n_items ? n_items : (uint64_t)v);
}

// Out degree of row x: seed rows from the prefix table, d for the others.
__device__ __forceinline__ uint32_t outdeg(uint64_t x, uint32_t d, const int64_t *seed_pre)
{
    return x <= (uint64_t)d ? (uint32_t)(seed_pre[x + 1] - seed_pre[x]) : d;
}

// Copy sorted items [a, b) -- the in parts of some of a row warp's rows -- into
// their places in col; U loads per lane in flight.
template <typename Id>
__device__ __forceinline__ void copy_in_items(const unsigned long long *items, uint64_t a, uint64_t b,
                                              uint32_t lane, uint64_t n, uint32_t d,
                                              uint64_t seed_edges, const int64_t *seed_pre, Id *col,
                                              uint64_t col_len)
{
    constexpr uint32_t U = 4;
    for (uint64_t k0 = a; k0 < b; k0 += 32 * U) {
        unsigned long long it[U];
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint64_t k = k0 + q * 32 + lane;
            it[q] = k < b ? items[k] : ~0ull;
        }
#pragma unroll
        for (uint32_t q = 0; q < U; ++q) {
            const uint64_t k = k0 + q * 32 + lane;
            const uint64_t v = it[q] >> 32;
            if (k < b && v < n) {
                const uint64_t pos = outprefix(v + 1, d, seed_edges, seed_pre) + k;
                if (pos < col_len) col[pos] = (Id)(it[q] & 0xffffffffull);
            }
        }
    }
}

template <typename Id>
__global__ void __launch_bounds__(256) rows_kernel(const Id *E, const unsigned long long *items,
                                                   uint64_t n_items, const int64_t *rowptr, Id *col,
                                                   uint64_t n, uint32_t d, uint64_t seed_edges,
                                                   const int64_t *seed_pre, uint64_t col_len,
                                                   unsigned long long *heavy, uint64_t heavy_cap,
                                                   unsigned long long *ctr)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint32_t G = 32u / d;   // rows per out part pass, d lanes each
    const uint32_t g = lane / d, i = lane - g * d;
    const bool used = lane < G * d;
    const uint64_t step = warps * kRowsChunk;
    // rowptr of each chunk's rows is loaded one chunk ahead
    int64_t rp_next = 0, rp1_next = 0;
    if (w0 * kRowsChunk + lane < n) {
        rp_next = rowptr[w0 * kRowsChunk + lane];
        rp1_next = rowptr[w0 * kRowsChunk + lane + 1];
    }
    for (uint64_t x0 = w0 * kRowsChunk; x0 < n; x0 += step) {
        // lane j: row x0 + j, its rowptr and its in part's item range
        const uint64_t x = x0 + lane;
        const bool row_ok = x < n;
        const int64_t rp = row_ok ? rp_next : 0, rp1 = row_ok ? rp1_next : 0;
        if (x + step < n) {
            rp_next = rowptr[x + step];
            rp1_next = rowptr[x + step + 1];
        }
        uint64_t lb = n_items, lb1 = n_items;
        if (row_ok) {
            lb = clamp_items(rp - (int64_t)outprefix(x, d, seed_edges, seed_pre), n_items);
            lb1 = clamp_items(rp1 - (int64_t)outprefix(x + 1, d, seed_edges, seed_pre), n_items);
            if (lb1 < lb) lb1 = lb;
        }
        const bool heavy_row = row_ok && lb1 - lb > kHeavyIn;
        if (heavy_row) {
            // listed in any order: every entry's place is fixed by its index
            const unsigned long long slot = atomicAdd(ctr, 1ull);
            if (slot < heavy_cap) heavy[slot] = x;
        }
        uint32_t hv = __ballot_sync(kFull, heavy_row);
        uint64_t a = __shfl_sync(kFull, lb, 0);
        const uint64_t end = __shfl_sync(kFull, lb1, 31);
        // without hub rows the chunk's in parts are items [a, end): their first
        // kPre * 32 loads go out now, beside the out parts' loads below
        constexpr uint32_t kPre = 4;
        unsigned long long pre[kPre];
#pragma unroll
        for (uint32_t q = 0; q < kPre; ++q) {
            const uint64_t k = a + q * 32 + lane;
            pre[q] = hv == 0 && k < end ? items[k] : ~0ull;
        }

        // (a) out parts, G rows per pass, each row's d targets ranked in
        // registers (as 32-bit node ids: n < 2^32); U passes' loads issued
        // together.  Seed rows hold targets 0, 1, ... (both seed graphs); their
        // absent slots sort last.
        constexpr uint32_t U = 4;
        for (uint32_t r0 = 0; r0 < kRowsChunk; r0 += U * G) {
            uint32_t t[U];
            bool have[U];
            int64_t rrp[U];
#pragma unroll
            for (uint32_t q = 0; q < U; ++q) {
                const uint32_t rj = r0 + q * G + g;
                rrp[q] = __shfl_sync(kFull, rp, rj & 31u);
                const uint64_t row = x0 + rj;
                const bool act = used && rj < kRowsChunk && row < n;
                t[q] = 0xffffffffu;
                have[q] = false;
                if (act && row > d) {
                    t[q] = (uint32_t)E[2 * (seed_edges + (row - d - 1) * d + i) + 1];
                    have[q] = true;
                } else if (act && i < outdeg(row, d, seed_pre)) {
                    t[q] = i;
                    have[q] = true;
                }
            }
            // the U passes' ranks in one loop: U independent shuffles per step
            uint32_t rank[U];
#pragma unroll
            for (uint32_t q = 0; q < U; ++q) rank[q] = 0;
            const uint32_t gb = g * d;
#pragma unroll 2
            for (uint32_t j = 0; j < d; ++j) {
                const uint32_t src = (gb + j) & 31u;
#pragma unroll
                for (uint32_t q = 0; q < U; ++q)
                    rank[q] += __shfl_sync(kFull, t[q], src) < t[q] ? 1u : 0u;
            }
#pragma unroll
            for (uint32_t q = 0; q < U; ++q) {
                if (have[q]) {
                    const uint64_t pos = (uint64_t)rrp[q] + rank[q];
                    if (pos < col_len) col[pos] = (Id)t[q];
                }
            }
        }

        // (b) in parts of the chunk's rows, the heavy rows' ranges skipped
        if (hv == 0) {
#pragma unroll
            for (uint32_t q = 0; q < kPre; ++q) {
                const uint64_t k = a + q * 32 + lane;
                const uint64_t v = pre[q] >> 32;
                if (k < end && v < n) {
                    const uint64_t pos = outprefix(v + 1, d, seed_edges, seed_pre) + k;
                    if (pos < col_len) col[pos] = (Id)(pre[q] & 0xffffffffull);
                }
            }
            a = min(a + kPre * 32, end);
        }
        while (true) {
            uint64_t b = end, next = end;
            if (hv) {
                const uint32_t h = __ffs(hv) - 1;
                b = __shfl_sync(kFull, lb, h);
                next = __shfl_sync(kFull, lb1, h);
                hv &= hv - 1;
            }
            if (b > a) copy_in_items(items, a, b, lane, n, d, seed_edges, seed_pre, col, col_len);
            if (b == end && next == end) break;
            a = next;
        }
    }
}

// Row x's in part: sorted items [lb, lb1), entry k at col[base + k].
struct InPart {
    uint64_t lb, lb1, base;
};

__device__ __forceinline__ InPart in_part(uint64_t x, const int64_t *rowptr, uint64_t n_items,
                                          uint32_t d, uint64_t seed_edges, const int64_t *seed_pre)
{
    InPart r;
    r.base = outprefix(x + 1, d, seed_edges, seed_pre);
    r.lb = clamp_items(rowptr[x] - (int64_t)outprefix(x, d, seed_edges, seed_pre), n_items);
    r.lb1 = clamp_items(rowptr[x + 1] - (int64_t)r.base, n_items);
    if (r.lb1 < r.lb) r.lb1 = r.lb;
    return r;
}

// The first piece of every listed row: pref[h] = pieces of rows 0..h-1 of the
// list, pref[K] = all pieces (one block; the list holds at most one entry per
// kHeavyIn items).
__global__ void __launch_bounds__(1024) heavy_scan_kernel(const unsigned long long *heavy,
                                                          uint64_t heavy_cap,
                                                          const unsigned long long *ctr,
                                                          const int64_t *rowptr, uint64_t n,
                                                          uint32_t d, uint64_t seed_edges,
                                                          const int64_t *seed_pre,
                                                          uint64_t n_items,
                                                          unsigned long long *pref)
{
    __shared__ unsigned long long wsum[32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint64_t K = min((uint64_t)ctr[0], heavy_cap);
    unsigned long long carry = 0;
    for (uint64_t h0 = 0; h0 < K; h0 += 1024) {
        const uint64_t h = h0 + threadIdx.x;
        unsigned long long pc = 0;
        if (h < K && heavy[h] < n) {
            const InPart r = in_part(heavy[h], rowptr, n_items, d, seed_edges, seed_pre);
            pc = (r.lb1 - r.lb + kPiece - 1) / kPiece;
        }
        unsigned long long x = pc;   // inclusive scan over the block
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long y = __shfl_up_sync(kFull, x, o);
            if (lane >= (uint32_t)o) x += y;
        }
        if (lane == 31) wsum[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned long long w = wsum[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long y = __shfl_up_sync(kFull, w, o);
                if (lane >= (uint32_t)o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        const unsigned long long before = warp > 0 ? wsum[warp - 1] : 0ull;
        if (h < K) pref[h] = carry + before + x - pc;
        carry += wsum[31];
        __syncthreads();   // wsum is rewritten by the next chunk
    }
    if (threadIdx.x == 0) pref[K] = carry;
}

// In parts of the listed rows, in pieces of kPiece items: a warp takes runs of
// kPieceRun consecutive pieces (over all listed rows, in list order), finds the
// row of its first piece by binary search over pref and copies each piece with
// all 32 lanes (kPiece / 32 items each, loads issued together).
constexpr uint32_t kPieceRun = 16;

template <typename Id>
__global__ void __launch_bounds__(256) heavy_in_kernel(const unsigned long long *items,
                                                       uint64_t n_items, const int64_t *rowptr,
                                                       Id *col, uint64_t n, uint32_t d,
                                                       uint64_t seed_edges, const int64_t *seed_pre,
                                                       uint64_t col_len,
                                                       const unsigned long long *heavy,
                                                       uint64_t heavy_cap,
                                                       const unsigned long long *ctr,
                                                       const unsigned long long *pref)
{
    constexpr uint32_t PL = kPiece / 32;   // items per lane per piece
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const uint64_t K = min((uint64_t)ctr[0], heavy_cap);
    if (K == 0) return;
    const uint64_t T = pref[K];
    for (uint64_t t0 = w0 * kPieceRun; t0 < T; t0 += warps * kPieceRun) {
        // the last h with pref[h] <= t0 (pref[0] = 0, pref is non-decreasing)
        uint64_t lo = 0, hi = K;
        while (hi - lo > 1) {
            const uint64_t mid = lo + (hi - lo) / 2;
            if (pref[mid] <= t0) lo = mid;
            else hi = mid;
        }
        uint64_t h = lo, next = pref[h + 1];
        InPart r{0, 0, 0};
        if (heavy[h] < n) r = in_part(heavy[h], rowptr, n_items, d, seed_edges, seed_pre);
        const uint64_t t1 = min(t0 + kPieceRun, T);
        for (uint64_t t = t0; t < t1; ++t) {
            while (t >= next && h + 1 < K) {   // rows of one piece or more: a few steps
                ++h;
                next = pref[h + 1];
                r = heavy[h] < n ? in_part(heavy[h], rowptr, n_items, d, seed_edges, seed_pre)
                                 : InPart{0, 0, 0};
            }
            const uint64_t k0 = r.lb + (t - pref[h]) * kPiece;
            unsigned long long it[PL];
#pragma unroll
            for (uint32_t q = 0; q < PL; ++q) {
                const uint64_t k = k0 + q * 32 + lane;
                it[q] = k < r.lb1 ? items[k] : 0ull;
            }
#pragma unroll
            for (uint32_t q = 0; q < PL; ++q) {
                const uint64_t k = k0 + q * 32 + lane, pos = r.base + k;
                if (k < r.lb1 && pos < col_len) col[pos] = (Id)(it[q] & 0xffffffffull);
            }
        }
    }
}

int grid_for(uint64_t items, uint32_t threads, uint32_t per_sm = 8)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t want = (items + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sms * per_sm;
    return (int)(want == 0 ? 1 : (want > cap ? cap : want));
}

struct CsrLayout {
    uint64_t items_off, status_off, hist_off, base_off, ctr_off, err_off, seed_out_off,
        seed_pre_off, heavy_off, pref_off, total;
    uint64_t r_tiles;               // radix tiles
    uint64_t heavy_cap;             // rows with in parts above kHeavyIn items
    uint32_t db, passes;            // digit bits and passes of the sort
    uint64_t status_bytes;
    bool status_in_col;             // status words in the column buffer's second half
};

// Graphs below 2^32 nodes: items pack (v, u) in 8 bytes.
bool csr_supported(uint64_t n) { return n < (1ull << 32); }

// Digit width of the sort: keys < n need bits(n - 1) bits (a pair with an id
// outside the node range raises an error; its key, all ones in those bits, then
// sorts last or among the keys n - 1).  The fewest passes of 8 or 9 bits; on
// a tie, as measured: 9-bit digits for three passes (24-bit keys: 6.01 against
// 6.22 ms at n = 1.6 * 10^7, d = 9; 22-bit: 3.08 against 3.11 ms), 8-bit ones
// otherwise (30-bit keys, four passes: 214.1 against 227.3 ms at n = 2^30).
void radix_digits(uint64_t n, uint32_t *db, uint32_t *passes)
{
    uint32_t bits = 1;
    while (bits < 32 && ((n - 1) >> bits) != 0) ++bits;
    // (10-bit digits -- the pass kernel's per-digit steps take two digits per
    // thread when kRadixBuckets allows it -- measured twice as slow per pass as
    // 8-bit ones at n = 2^30 with 6,144-item tiles: 88 KB of shared memory,
    // 64 registers, runs of ~6 items per digit and tile.  Three of them lost
    // to four 8-bit passes, 306 against 238 ms.)
    *db = 8;
    *passes = (bits + 7) / 8;
    const uint32_t nine = (bits + 8) / 9;
    if (nine < *passes || (nine == *passes && *passes == 3)) {
        *db = 9;
        *passes = nine;
    }
}

CsrLayout csr_layout(uint64_t n, uint32_t d, uint64_t n_edges, uint32_t id_bytes)
{
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    CsrLayout L{};
    radix_digits(n, &L.db, &L.passes);
    L.r_tiles = (n_edges + kRadixTile - 1) / kRadixTile;
    L.status_bytes = 8ull * (1u << L.db) * std::max<uint64_t>(L.r_tiles, 1);
    // with 8-byte ids the column buffer (16 bytes per pair) holds the sort's
    // second item array (8 per pair) and, behind it, the look-back words
    L.status_in_col = id_bytes == 8 && L.status_bytes <= 8 * n_edges;
    uint64_t o = 0;
    L.items_off = o;    o += al(8 * std::max<uint64_t>(n_edges, 1));
    L.status_off = o;   o += L.status_in_col ? 0 : al(L.status_bytes);
    L.hist_off = o;     o += al(8 * kMaxPasses * kRadixBuckets);
    L.base_off = o;     o += al(8 * kMaxPasses * kRadixBuckets);
    L.ctr_off = o;      o += 256;   // one tile counter per pass, then the hub rows'
    L.err_off = o;      o += 256;
    L.seed_out_off = o; o += al(4 * (d + 1));
    L.seed_pre_off = o; o += al(8 * (d + 2));
    // more than cap rows cannot each hold more than kHeavyIn of the n_edges items
    L.heavy_cap = n_edges / (kHeavyIn + 1) + 1;

    L.heavy_off = o;    o += al(8 * L.heavy_cap);
    L.pref_off = o;     o += al(8 * (L.heavy_cap + 1));
    L.total = o;
    return L;
}

// Every pass of the sort: the histogram of all passes' digits, their bases,
// then one kernel per pass.  The last pass always lands in A.
template <typename Id, uint32_t DB>
int radix_sort(const Id *E, uint64_t m, uint64_t n, uint32_t passes, unsigned long long *A,
               unsigned long long *B, unsigned long long *status, unsigned char *scratch,
               const CsrLayout &L, uint32_t *err, cudaStream_t s)
{
    constexpr uint32_t NB = 1u << DB;
    unsigned long long *hist = (unsigned long long *)(scratch + L.hist_off);
    unsigned long long *base = (unsigned long long *)(scratch + L.base_off);
    unsigned long long *ctr = (unsigned long long *)(scratch + L.ctr_off);
    const size_t smem = sizeof(RadixSmem<NB>);
    cudaError_t e = cudaFuncSetAttribute(radix_pass_kernel<DB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // status words of an earlier call must not read as this call's
    if (e == cudaSuccess) e = cudaMemsetAsync(status, 0, 8 * (uint64_t)NB * L.r_tiles, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(hist, 0, 8 * kMaxPasses * kRadixBuckets, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctr, 0, 8 * kMaxPasses, s);
    if (e != cudaSuccess) return set_cuda_error(e);
    // pass q reads what pass q - 1 wrote; the histogram kernel writes the
    // items where pass 0 reads them, so that the last pass lands in A
    auto buf = [&](uint32_t k) { return (passes - k) % 2 == 0 ? A : B; };   // pass k - 1's output
    // four 512-thread blocks per SM (24 registers, 8 KB of counters each): at
    // n = 10^8, d = 16 the kernel took 8.44 ms with two blocks per SM, 5.96 ms
    // with four
    radix_hist_all_kernel<Id, DB><<<grid_for(m / 4 + 1, kRadixThreads, 4), kRadixThreads, 0, s>>>(
        E, m, n, passes, buf(0), hist, err);
    radix_base_kernel<DB><<<1, 32, 0, s>>>(hist, passes, base);
    const unsigned tiles = (unsigned)L.r_tiles;
    for (uint32_t q = 0; q < passes; ++q)
        radix_pass_kernel<DB><<<tiles, kRadixThreads, smem, s>>>(
            buf(q), buf(q + 1), m, DB * q, base + q * NB, status, q + 1, ctr + q, 2000000000ull, err);
    e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

// Sort, rowptr, in parts, out parts, queued on s; the device error word is at
// scratch + err_off (PA_OK, or PA_ERR_INVALID / PA_ERR_SPIN_TIMEOUT).
template <typename Id>
int csr_enqueue_t(const pa_params *prm, const GenPlan &p, const Id *E, int64_t *rowptr, Id *col,
                  unsigned char *scratch, const CsrLayout &L, cudaStream_t s)
{
    const uint64_t n = prm->n, m = p.n_edges;
    const uint32_t d = prm->d;
    uint32_t *seed_out = (uint32_t *)(scratch + L.seed_out_off);
    int64_t *seed_pre = (int64_t *)(scratch + L.seed_pre_off);
    uint32_t *err = (uint32_t *)(scratch + L.err_off);
    unsigned long long *A = (unsigned long long *)(scratch + L.items_off);
    // the column buffer (>= 8 bytes per pair) holds the other ping-pong array
    // while sorting; the last pass always lands in A
    unsigned long long *B = reinterpret_cast<unsigned long long *>(col);
    cudaError_t e = cudaMemsetAsync(err, 0, 4, s);
    if (e != cudaSuccess) return set_cuda_error(e);
    seed_out_kernel<<<1, 256, 0, s>>>(d, prm->seed_mode, seed_out);
    seed_prefix_kernel<<<1, 32, 0, s>>>(seed_out, d, seed_pre);
    unsigned long long *status =
        L.status_in_col ? reinterpret_cast<unsigned long long *>(col) + m
                        : (unsigned long long *)(scratch + L.status_off);
    if (m > 0) {
        int rc = PA_ERR_INVALID;
        if (L.db == 9)
            rc = radix_sort<Id, 9>(E, m, n, L.passes, A, B, status, scratch, L, err, s);
        else
            rc = radix_sort<Id, 8>(E, m, n, L.passes, A, B, status, scratch, L, err, s);
        if (rc != PA_OK) return rc;
    }
    const uint64_t col_len = 2 * m;
    if (p.wide) {
        // in parts and rowptr from the sorted items, the seed rows' out parts,
        // then the generated rows' out parts (ranked in shared memory)
        in_sorted_kernel<Id><<<grid_for(m / 4 + 1, 256), 256, 0, s>>>(
            A, m, n, d, p.seed_edges, seed_pre, col, col_len, rowptr);
        seed_out_part_kernel<Id><<<grid_for(p.seed_edges, 256), 256, 0, s>>>(E, rowptr, col, n,
                                                                             p.seed_edges, col_len);
        const int rc = gen::csr_out_wide(p.id_bytes, E, rowptr, col, n, d, p.seed_edges, col_len, s);
        if (rc != PA_OK) return rc;
    } else {
        // rowptr, then whole rows (the hub rows' in parts listed and copied last)
        unsigned long long *lists = (unsigned long long *)(scratch + L.ctr_off) + kMaxPasses;
        unsigned long long *heavy = (unsigned long long *)(scratch + L.heavy_off);
        unsigned long long *pref = (unsigned long long *)(scratch + L.pref_off);
        e = cudaMemsetAsync(lists, 0, 8, s);
        if (e != cudaSuccess) return set_cuda_error(e);
        rowptr_kernel<<<grid_for(m / 8 + 1, 256), 256, 0, s>>>(A, m, n, d, p.seed_edges,
                                                                seed_pre, rowptr);
        const int grid = grid_for(n / kRowsChunk + 1, 256 / 32);
        rows_kernel<Id><<<grid, 256, 0, s>>>(E, A, m, rowptr, col, n, d, p.seed_edges, seed_pre,
                                             col_len, heavy, L.heavy_cap, lists);
        heavy_scan_kernel<<<1, 1024, 0, s>>>(heavy, L.heavy_cap, lists, rowptr, n, d,
                                              p.seed_edges, seed_pre, m, pref);
        // one warp per run of kPieceRun pieces; at most m / kPiece + (listed rows) pieces
        heavy_in_kernel<Id><<<grid_for(m / (kPiece * kPieceRun) + 1, 256 / 32), 256, 0, s>>>(
            A, m, rowptr, col, n, d, p.seed_edges, seed_pre, col_len, heavy, L.heavy_cap, lists,
            pref);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

}  // namespace

int csr_enqueue(const pa_params *prm, const void *d_edges, int64_t *d_rowptr, void *d_col,
                void *d_scratch, uint64_t scratch_bytes, cudaStream_t s, uint64_t *err_offset)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !d_rowptr || !d_col || !d_scratch) return PA_ERR_INVALID;
    if (!csr_supported(prm->n) || p.slots || (p.wide && prm->d > gen::kWideRankMaxD))
        return PA_ERR_NOT_SUPPORTED;
    if ((reinterpret_cast<uintptr_t>(d_col) & 15u) || (reinterpret_cast<uintptr_t>(d_scratch) & 15u))
        return PA_ERR_INVALID;
    const CsrLayout L = csr_layout(prm->n, prm->d, p.n_edges, p.id_bytes);
    if (scratch_bytes < L.total) return PA_ERR_CAPACITY;
    if (err_offset) *err_offset = L.err_off;
    if (p.id_bytes == 8)
        return csr_enqueue_t<int64_t>(prm, p, (const int64_t *)d_edges, d_rowptr, (int64_t *)d_col,
                                      (unsigned char *)d_scratch, L, s);
    return csr_enqueue_t<int32_t>(prm, p, (const int32_t *)d_edges, d_rowptr, (int32_t *)d_col,
                                  (unsigned char *)d_scratch, L, s);
}

}  // namespace pa

using namespace pa;

extern "C" {

int pa_csr_bytes(const pa_params *prm, uint64_t *rowptr_bytes, uint64_t *col_bytes,
                 uint64_t *scratch_bytes)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!rowptr_bytes || !col_bytes || !scratch_bytes) return PA_ERR_INVALID;
    if (!csr_supported(prm->n) || p.slots || (p.wide && prm->d > gen::kWideRankMaxD))
        return PA_ERR_NOT_SUPPORTED;
    *rowptr_bytes = 8 * (prm->n + 1);
    *col_bytes = 2 * p.n_edges * p.id_bytes;
    *scratch_bytes = csr_layout(prm->n, prm->d, p.n_edges, p.id_bytes).total;
    return PA_OK;
}

int pa_build_csr(const pa_params *prm, const void *d_edges, int64_t *d_rowptr, void *d_col,
                 void *d_scratch, uint64_t scratch_bytes, void *stream)
{
    cudaStream_t s = (cudaStream_t)stream;
    uint64_t err_off = 0;
    const int rc = csr_enqueue(prm, d_edges, d_rowptr, d_col, d_scratch, scratch_bytes, s, &err_off);
    if (rc != PA_OK) return rc;
    uint32_t herr = 0;
    cudaError_t e = cudaMemcpyAsync(&herr, (const unsigned char *)d_scratch + err_off, 4,
                                    cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_cuda_error(e);
    return (int)herr;
}

}  // extern "C"
