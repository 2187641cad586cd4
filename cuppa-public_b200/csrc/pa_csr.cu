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
//      the seed rows' targets come from the (canonical) seed edges.
// Items pack (v, u) in 8 bytes, so graphs of 2^32 nodes and more are refused.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "pa_device.cuh"
#include "pa_internal.h"

namespace pa {
namespace {

constexpr uint32_t kFull = 0xffffffffu;
constexpr uint32_t kScanThreads = 256;
constexpr uint32_t kScanItems = 8;
constexpr uint32_t kScanTile = kScanThreads * kScanItems;

// ---------------------------------------------------------------------------
// Exclusive scan of int64 with decoupled look-back.  Tile status word:
// bits 62-63 = 0 (empty), 1 (aggregate), 2 (inclusive prefix); bits 0-61 value.
// ---------------------------------------------------------------------------
constexpr unsigned long long kStAgg = 1ull << 62, kStInc = 2ull << 62,
                             kValMask = (1ull << 62) - 1;

__device__ __forceinline__ unsigned long long ld_status(const unsigned long long *p)
{
    return ld_acquire_u64(p);
}

// Exclusive scan of in[0, n) into out[0, n) (in == out allowed: a tile reads its
// items before it writes them and touches no other tile's items).
__global__ void __launch_bounds__(kScanThreads) scan_kernel(const int64_t *in, int64_t *out,
                                                            uint64_t n, unsigned long long *status,
                                                            unsigned long long *tile_ctr,
                                                            uint64_t spin_limit_ns, uint32_t *err)
{
    __shared__ unsigned long long s_tile;
    __shared__ int64_t s_warp[kScanThreads / 32];
    __shared__ int64_t s_prefix;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1ull);
    __syncthreads();
    const uint64_t tile = s_tile;
    const uint64_t base = tile * kScanTile + (uint64_t)threadIdx.x * kScanItems;
    int64_t v[kScanItems];
    int64_t sum = 0;
#pragma unroll
    for (uint32_t i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? in[base + i] : 0;
        sum += v[i];
    }
    // block-wide exclusive scan of per-thread sums
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    int64_t x = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        int64_t w = lane < kScanThreads / 32 ? s_warp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(kFull, w, o);
            if (lane >= (uint32_t)o) w += y;
        }
        if (lane < kScanThreads / 32) s_warp[lane] = w;   // inclusive per warp
    }
    __syncthreads();
    const int64_t block_total = s_warp[kScanThreads / 32 - 1];
    int64_t thread_excl = x - sum + (warp ? s_warp[warp - 1] : 0);

    // look-back
    if (warp == 0) {
        int64_t prefix = 0;
        if (tile == 0) {
            if (lane == 0) {
                st_release_u64(status, kStInc | (unsigned long long)block_total);
            }
        } else {
            if (lane == 0) st_release_u64(status + tile, kStAgg | (unsigned long long)block_total);
            int64_t pred = (int64_t)tile - 1;
            const uint64_t t0 = globaltimer_ns();
            bool failed = false;
            while (true) {
                // each lane inspects one predecessor, newest first
                const int64_t t = pred - (int64_t)lane;
                unsigned long long st = t >= 0 ? ld_status(status + t) : (kStInc);
                const uint32_t empty = __ballot_sync(kFull, (st >> 62) == 0);
                const uint32_t inc = __ballot_sync(kFull, (st >> 62) == 2);
                // lanes before the first empty one are usable; stop at the first inclusive
                const uint32_t stop_empty = empty ? (uint32_t)(__ffs(empty) - 1) : 32u;
                const uint32_t stop_inc = inc ? (uint32_t)(__ffs(inc) - 1) : 32u;
                if (stop_inc < stop_empty) {
                    // sum lanes [0, stop_inc] (the inclusive one included)
                    const int64_t contrib = lane <= stop_inc ? (int64_t)(st & kValMask) : 0;
                    int64_t s = contrib;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
                    prefix += s;
                    break;
                }
                if (stop_empty > 0) {
                    const int64_t contrib = lane < stop_empty ? (int64_t)(st & kValMask) : 0;
                    int64_t s = contrib;
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(kFull, s, o);
                    prefix += s;
                    pred -= stop_empty;
                    continue;
                }
                if (globaltimer_ns() - t0 > spin_limit_ns) { failed = true; break; }
                __nanosleep(64);
            }
            if (failed) {
                if (lane == 0) atomicCAS(err, 0u, (uint32_t)PA_ERR_SPIN_TIMEOUT);
            } else if (lane == 0) {
                st_release_u64(status + tile, kStInc | (unsigned long long)(prefix + block_total));
            }
        }
        if (lane == 0) s_prefix = prefix;
    }
    __syncthreads();
    int64_t run = s_prefix + thread_excl;
#pragma unroll
    for (uint32_t i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
}

// ---------------------------------------------------------------------------
// Out parts.
// ---------------------------------------------------------------------------
template <typename Id>
__global__ void out_part_kernel(const Id *E, const int64_t *rowptr, Id *col, uint64_t n, uint32_t d,
                                uint64_t seed_edges, uint64_t col_len)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    // seed rows: canonical seed edges are grouped by src, ascending dst
    for (uint64_t e = w0 * 32 + lane; e < seed_edges; e += warps * 32) {
        const uint64_t u = (uint64_t)E[2 * e];
        // position of this edge among u's seed out-edges
        uint64_t first = e;
        while (first > 0 && (uint64_t)E[2 * (first - 1)] == u) --first;
        const uint64_t pos = (uint64_t)rowptr[u] + (e - first);
        if (u < n && pos < col_len) col[pos] = E[2 * e + 1];
    }
    const uint32_t G = 32u / d;
    const uint32_t g = lane / d, i = lane - g * d;
    const bool used = lane < G * d;
    const uint64_t rows = n - (d + 1);
    for (uint64_t r0 = w0 * G; r0 < rows; r0 += warps * G) {
        const uint64_t row = r0 + g;
        const bool act = used && row < rows;
        Id dst = 0;
        if (act) dst = E[2 * (seed_edges + row * d + i) + 1];
        uint32_t rank = 0;
        for (uint32_t j = 0; j < d; ++j) {
            const Id o = __shfl_sync(kFull, dst, (g * d + j) & 31u);
            rank += (o < dst) ? 1u : 0u;
        }
        if (act) {
            const uint64_t pos = (uint64_t)rowptr[row + d + 1] + rank;
            if (pos < col_len) col[pos] = dst;
        }
    }
}

// Out-degree of each seed node (its canonical seed edges).
template <typename Id>
__global__ void seed_out_kernel(const Id *E, uint64_t seed_edges, uint32_t d, uint32_t *seed_out)
{
    for (uint32_t v = threadIdx.x; v <= d; v += blockDim.x) {
        uint32_t c = 0;
        for (uint64_t e = 0; e < seed_edges; ++e) c += (uint64_t)E[2 * e] == v;
        seed_out[v] = c;
    }
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
// the node range, no per-row sorting, no special path for hub rows.
//
// A pass sorts 8 or 9 key bits: a histogram kernel counts the digits of every
// tile of 8192 items into a digit-major table, an exclusive scan of the table
// gives each (digit, tile) its output offset, and the scatter kernel ranks every
// item within its tile stably -- each of 16 warps walks its 512 items in order,
// 32 at a time, with __match_any_sync for equal digits and 16-bit per-warp
// counters in shared memory, then the warps' counts are prefixed per digit --
// stages the tile in shared memory in digit order and writes each digit's run
// contiguously.
// ---------------------------------------------------------------------------
constexpr uint32_t kRadixThreads = 512, kRadixWarps = kRadixThreads / 32;
constexpr uint32_t kRadixBuckets = 512;   // the widest digit: 9 bits
constexpr uint32_t kRadixRounds = 16;   // items per lane per tile
constexpr uint32_t kRadixTile = kRadixThreads * kRadixRounds;
constexpr unsigned long long kBadKey = 0xffffffffull;   // sorts after every node id

// Item i of a pass.  The first pass reads the pairs (ids above the node range,
// never produced by the generator, become kBadKey and raise an error).
template <typename Id, bool First>
__device__ __forceinline__ unsigned long long radix_item(const void *src, uint64_t i, uint64_t n,
                                                         uint32_t *err)
{
    if constexpr (First) {
        const Id *E = reinterpret_cast<const Id *>(src);
        const uint64_t u = (uint64_t)E[2 * i], v = (uint64_t)E[2 * i + 1];
        if (u >= n || v >= n) {
            atomicCAS(err, 0u, (uint32_t)PA_ERR_INVALID);
            return (kBadKey << 32) | 0xffffffffull;
        }
        return (v << 32) | u;
    } else {
        return reinterpret_cast<const unsigned long long *>(src)[i];
    }
}

template <typename Id, bool First, uint32_t DB>
__global__ void __launch_bounds__(kRadixThreads) radix_hist_kernel(const void *src, uint64_t n_items,
                                                                   uint32_t shift, uint64_t n,
                                                                   int64_t *table, uint64_t n_tiles,
                                                                   uint32_t *err)
{
    constexpr uint32_t NB = 1u << DB, MASK = NB - 1;
    __shared__ uint32_t cnt[NB];
    for (uint32_t b = threadIdx.x; b < NB; b += kRadixThreads) cnt[b] = 0;
    __syncthreads();
    const uint64_t t = blockIdx.x;
    const uint64_t base = t * kRadixTile;
    for (uint32_t r = 0; r < kRadixRounds; ++r) {
        const uint64_t i = base + (uint64_t)r * kRadixThreads + threadIdx.x;
        if (i < n_items) {
            const unsigned long long it = radix_item<Id, First>(src, i, n, err);
            atomicAdd(&cnt[(uint32_t)(it >> (32 + shift)) & MASK], 1u);
        }
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < NB; b += kRadixThreads) table[(uint64_t)b * n_tiles + t] = cnt[b];
}

// Dynamic shared memory of the scatter kernel: the tile's items in digit order,
// then the per-warp counts, ranks and bases.
template <uint32_t NB>
struct RadixSmem {
    unsigned long long stage[kRadixTile];
    unsigned long long goff[NB];                  // global offset of the digit's run, less its
                                                  // start within the tile
    uint16_t wcnt[kRadixWarps][NB];               // per-warp digit counts, then the warp's base
                                                  // within the tile (digit start included)
    uint16_t lrank[kRadixTile];                   // rank within the warp's items of its digit
};

template <typename Id, bool First, uint32_t DB>
__global__ void __launch_bounds__(kRadixThreads, 2) radix_scatter_kernel(const void *src,
                                                                      unsigned long long *dst,
                                                                      uint64_t n_items, uint32_t shift,
                                                                      uint64_t n, const int64_t *offs,
                                                                      uint64_t n_tiles, uint32_t *err)
{
    constexpr uint32_t NB = 1u << DB, MASK = NB - 1;
    constexpr uint32_t PER = NB > kRadixThreads ? NB / kRadixThreads : 1;   // digits per thread
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RadixSmem<NB> &S = *reinterpret_cast<RadixSmem<NB> *>(smem_raw);
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint32_t lt = lanemask_lt();
    for (uint32_t w = 0; w < kRadixWarps; ++w)
        for (uint32_t b = threadIdx.x; b < NB; b += kRadixThreads) S.wcnt[w][b] = 0;
    __syncthreads();
    const uint64_t t = blockIdx.x;
    const uint64_t tb = t * kRadixTile;
    const uint32_t tcount = (uint32_t)min((uint64_t)kRadixTile, n_items - tb);
    const uint32_t wo = warp * (kRadixRounds * 32);
    // 1. stable ranks within the warp's items (in order, 32 per round); the
    // loads of kBatch rounds are issued together
    constexpr uint32_t kBatch = 8;
    for (uint32_t r0 = 0; r0 < kRadixRounds; r0 += kBatch) {
        uint32_t dgs[kBatch];
#pragma unroll
        for (uint32_t q = 0; q < kBatch; ++q) {
            const uint32_t k = wo + (r0 + q) * 32 + lane;
            dgs[q] = k < tcount
                         ? (uint32_t)(radix_item<Id, First>(src, tb + k, n, err) >> (32 + shift)) & MASK
                         : NB + lane;   // unique for lanes past the end
        }
#pragma unroll
        for (uint32_t q = 0; q < kBatch; ++q) {
            const uint32_t k = wo + (r0 + q) * 32 + lane;
            const bool valid = k < tcount;
            const uint32_t dg = dgs[q];
            const uint32_t peers = __match_any_sync(kFull, dg);
            const uint32_t leader = __ffs(peers) - 1;
            uint32_t old = 0;
            if (valid && lane == leader) {
                old = S.wcnt[warp][dg];
                S.wcnt[warp][dg] = (uint16_t)(old + __popc(peers));
            }
            old = __shfl_sync(kFull, old, leader);
            if (valid) S.lrank[k] = (uint16_t)(old + __popc(peers & lt));
            // the next round's leader for a digit may be another lane: order
            // this round's counter stores before the next round's loads
            __syncwarp();
        }
    }
    __syncthreads();
    // 2. per digit (thread j owns digits j*PER .. j*PER+PER-1): warp bases in
    // warp order, the digit's total, then the digits' starts within the tile,
    // folded into the warp bases and the global offsets so that phases 3 and 4
    // make one randomly indexed shared access each per item (shared memory, not
    // DRAM, is what bounds this kernel)
    uint32_t tot[PER];
    uint32_t mine = 0;
#pragma unroll
    for (uint32_t q = 0; q < PER; ++q) {
        const uint32_t dg = threadIdx.x * PER + q;
        tot[q] = 0;
        if (dg < NB) {
            uint32_t acc = 0;
            for (uint32_t w = 0; w < kRadixWarps; ++w) {
                const uint32_t c = S.wcnt[w][dg];
                S.wcnt[w][dg] = (uint16_t)acc;
                acc += c;
            }
            tot[q] = acc;
            S.goff[dg] = (unsigned long long)offs[(uint64_t)dg * n_tiles + t];
        }
        mine += tot[q];
    }
    uint32_t x = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(kFull, x, o);
        if (lane >= (uint32_t)o) x += y;
    }
    __shared__ uint32_t s_wsum[kRadixWarps];
    if (lane == 31) s_wsum[warp] = x;
    __syncthreads();
    uint32_t run = x - mine;
    for (uint32_t w = 0; w < warp; ++w) run += s_wsum[w];
#pragma unroll
    for (uint32_t q = 0; q < PER; ++q) {
        const uint32_t dg = threadIdx.x * PER + q;
        if (dg < NB) {
            for (uint32_t w = 0; w < kRadixWarps; ++w)   // <= tile size: fits 16 bits
                S.wcnt[w][dg] = (uint16_t)(S.wcnt[w][dg] + run);
            S.goff[dg] -= run;    // the run's global start >= its start in the tile
        }
        run += tot[q];
    }
    __syncthreads();
    // 3. the tile's items into shared memory in digit order (read again, from L2)
    for (uint32_t r0 = 0; r0 < kRadixRounds; r0 += kBatch) {
        unsigned long long its[kBatch];
#pragma unroll
        for (uint32_t q = 0; q < kBatch; ++q) {
            const uint32_t k = wo + (r0 + q) * 32 + lane;
            its[q] = k < tcount ? radix_item<Id, First>(src, tb + k, n, err) : 0ull;
        }
#pragma unroll
        for (uint32_t q = 0; q < kBatch; ++q) {
            const uint32_t k = wo + (r0 + q) * 32 + lane;
            if (k < tcount) {
                const uint32_t dg = (uint32_t)(its[q] >> (32 + shift)) & MASK;
                S.stage[S.wcnt[warp][dg] + S.lrank[k]] = its[q];
            }
        }
    }
    __syncthreads();
    // 4. out in digit runs: consecutive threads write consecutive addresses
    for (uint32_t k = threadIdx.x; k < tcount; k += kRadixThreads) {
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

// One pass over the sorted items: in part entry i (key v, value u) goes to
// col[outprefix(v + 1) + i], and rowptr[x] = outprefix(x) + #items with key < x
// is written for every x in (key(i-1), key(i)] (i = n_items closes the range up
// to n; keys >= n -- only after an input error -- count as n).
template <typename Id>
__global__ void in_sorted_kernel(const unsigned long long *items, uint64_t n_items, uint64_t n,
                                 uint32_t d, uint64_t seed_edges, const int64_t *seed_pre, Id *col,
                                 uint64_t col_len, int64_t *rowptr)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n_items; i += stride) {
        const unsigned long long it = i < n_items ? items[i] : ~0ull;
        const uint64_t v = i < n_items ? min((uint64_t)(it >> 32), n) : n;
        const uint64_t lo = i > 0 ? min((uint64_t)(items[i - 1] >> 32), n) + 1 : 0;
        for (uint64_t x = lo; x <= v && x <= n; ++x)
            rowptr[x] = (int64_t)(outprefix(x, d, seed_edges, seed_pre) + i);
        if (i < n_items && v < n) {
            const uint64_t pos = outprefix(v + 1, d, seed_edges, seed_pre) + i;
            if (pos < col_len) col[pos] = (Id)(it & 0xffffffffull);
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
    uint64_t status_off, ctr_off, err_off, seed_out_off, seed_pre_off, items_off, table_off, total;
    uint64_t n_tiles;   // scan tiles the status region holds
    uint64_t r_tiles;   // radix tiles
};

// Graphs below 2^32 nodes: items pack (v, u) in 8 bytes.
bool csr_supported(uint64_t n) { return n < (1ull << 32); }

CsrLayout csr_layout(uint64_t n, uint32_t d, uint64_t n_edges)
{
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    CsrLayout L{};
    L.r_tiles = (n_edges + kRadixTile - 1) / kRadixTile;
    const uint64_t scan_len = std::max<uint64_t>(kRadixBuckets * L.r_tiles, n + 1);
    L.n_tiles = (scan_len + kScanTile - 1) / kScanTile;
    uint64_t o = 0;
    L.items_off = o;    o += al(8 * std::max<uint64_t>(n_edges, 1));
    L.table_off = o;    o += al(8 * kRadixBuckets * std::max<uint64_t>(L.r_tiles, 1));
    L.status_off = o;   o += al(8 * L.n_tiles);
    L.ctr_off = o;      o += 256;
    L.err_off = o;      o += 256;
    L.seed_out_off = o; o += al(4 * (d + 1));
    L.seed_pre_off = o; o += al(8 * (d + 2));
    L.total = o;
    return L;
}

// Exclusive scan of len items (reuses the scratch's tile-status region).
int run_scan(const int64_t *in, int64_t *out, uint64_t len, unsigned char *scratch,
             const CsrLayout &L, cudaStream_t s)
{
    const uint64_t tiles = (len + kScanTile - 1) / kScanTile;
    if (tiles == 0) return PA_OK;
    if (tiles > L.n_tiles) return PA_ERR_CAPACITY;
    unsigned long long *status = (unsigned long long *)(scratch + L.status_off);
    unsigned long long *ctr = (unsigned long long *)(scratch + L.ctr_off);
    cudaError_t e = cudaMemsetAsync(status, 0, 8 * tiles, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(ctr, 0, 8, s);
    if (e != cudaSuccess) return set_cuda_error(e);
    scan_kernel<<<(unsigned)tiles, kScanThreads, 0, s>>>(in, out, len, status, ctr, 2000000000ull,
                                                         (uint32_t *)(scratch + L.err_off));
    e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

// One stable pass over DB key bits from `shift` (histogram, scan, scatter).
template <typename Id, uint32_t DB>
int radix_pass(bool first, const void *src, unsigned long long *dst, uint64_t m, uint32_t shift,
               uint64_t n, int64_t *table, unsigned char *scratch, const CsrLayout &L, uint32_t *err,
               cudaStream_t s)
{
    constexpr uint32_t NB = 1u << DB;
    const unsigned tiles = (unsigned)L.r_tiles;
    const size_t smem = sizeof(RadixSmem<NB>);
    cudaError_t e = cudaFuncSetAttribute(radix_scatter_kernel<Id, true, DB>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(radix_scatter_kernel<Id, false, DB>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (first)
        radix_hist_kernel<Id, true, DB><<<tiles, kRadixThreads, 0, s>>>(src, m, shift, n, table,
                                                                        L.r_tiles, err);
    else
        radix_hist_kernel<Id, false, DB><<<tiles, kRadixThreads, 0, s>>>(src, m, shift, n, table,
                                                                         L.r_tiles, err);
    const int rc = run_scan(table, table, (uint64_t)NB * L.r_tiles, scratch, L, s);
    if (rc != PA_OK) return rc;
    if (first)
        radix_scatter_kernel<Id, true, DB><<<tiles, kRadixThreads, smem, s>>>(src, dst, m, shift, n,
                                                                              table, L.r_tiles, err);
    else
        radix_scatter_kernel<Id, false, DB><<<tiles, kRadixThreads, smem, s>>>(src, dst, m, shift, n,
                                                                               table, L.r_tiles, err);
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
    int64_t *table = (int64_t *)(scratch + L.table_off);
    unsigned long long *A = (unsigned long long *)(scratch + L.items_off);
    // the column buffer (>= 8 bytes per pair) holds the other ping-pong array
    // while sorting; the last pass always lands in A
    unsigned long long *B = reinterpret_cast<unsigned long long *>(col);
    cudaError_t e = cudaMemsetAsync(err, 0, 4, s);
    if (e != cudaSuccess) return set_cuda_error(e);
    seed_out_kernel<Id><<<1, 64, 0, s>>>(E, p.seed_edges, d, seed_out);
    seed_prefix_kernel<<<1, 32, 0, s>>>(seed_out, d, seed_pre);
    uint32_t bits = 1;
    while (bits < 32 && (n >> bits) != 0) ++bits;   // keys < n need bits(n) bits; kBadKey sorts last
    // 9-bit digits when three passes cover the key (n < 2^27), else 8-bit ones
    const uint32_t db = bits <= 27 ? 9u : 8u;
    const uint32_t passes = (bits + db - 1) / db;
    int rc = PA_OK;
    for (uint32_t q = 0; q < passes && m > 0; ++q) {
        const uint32_t shift = db * q;
        unsigned long long *dst = ((passes - 1 - q) % 2 == 0) ? A : B;
        const void *src = q == 0 ? (const void *)E : (const void *)(((passes - q) % 2 == 0) ? A : B);
        rc = db == 9 ? radix_pass<Id, 9>(q == 0, src, dst, m, shift, n, table, scratch, L, err, s)
                     : radix_pass<Id, 8>(q == 0, src, dst, m, shift, n, table, scratch, L, err, s);
        if (rc != PA_OK) return rc;
    }
    const uint64_t col_len = 2 * m;
    in_sorted_kernel<Id><<<grid_for(m + 1, 256), 256, 0, s>>>(A, m, n, d, p.seed_edges, seed_pre, col,
                                                              col_len, rowptr);
    out_part_kernel<Id><<<grid_for(n * d, 256), 256, 0, s>>>(E, rowptr, col, n, d, p.seed_edges,
                                                             col_len);
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
    if (!csr_supported(prm->n) || p.slots) return PA_ERR_NOT_SUPPORTED;
    if ((reinterpret_cast<uintptr_t>(d_col) & 15u) || (reinterpret_cast<uintptr_t>(d_scratch) & 15u))
        return PA_ERR_INVALID;
    const CsrLayout L = csr_layout(prm->n, prm->d, p.n_edges);
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
    if (!csr_supported(prm->n) || p.slots) return PA_ERR_NOT_SUPPORTED;
    *rowptr_bytes = 8 * (prm->n + 1);
    *col_bytes = 2 * p.n_edges * p.id_bytes;
    *scratch_bytes = csr_layout(prm->n, prm->d, p.n_edges).total;
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
