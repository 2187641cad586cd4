// pa_csr.cu -- undirected CSR of a generated graph: every edge in both rows,
// every row sorted ascending.  No reference counterpart (the reference never
// hands its graph out); the degree pass is the device side of
// src/PA/cuPPA/cuPPA.cu:103-165.
//
// Row x is [x's own targets, all < x, ascending] ++ [x's in-neighbours, all > x,
// ascending], so it comes out sorted when both parts are:
//   1. in-degrees: one warp-aggregated atomic per pair on its destination; the
//      value the atomic returns is the pair's rank in the destination's in part,
//      kept (4 bytes per pair) so that step 4 needs no atomics;
//   2. rowptr = exclusive scan of out-degree + in-degree: a single-pass scan with
//      decoupled look-back (tiles take ids in launch order from an atomic counter,
//      publish their aggregate, then their inclusive prefix);
//   3. out part: each generated row's d targets ranked in registers and stored;
//      the seed rows' targets come from the (canonical) seed edges;
//   4. in part: every pair (u, v) stores u at its rank in v's in part (order
//      arbitrary across warps) ...
//   5. ... then every in part is sorted: a warp per part of <= 32 entries (rank
//      by counting; entries of a part are distinct), a warp bitonic network in
//      registers for <= 256 entries, a CTA bitonic sort in shared memory for
//      <= 8192, and the few larger hub parts by a bitmap over the node range
//      (set, then compact in order).
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
constexpr uint32_t kMidMax = 8192;   // largest in part sorted in shared memory

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

// ---------------------------------------------------------------------------
// In-degrees and in-part ranks.
// ---------------------------------------------------------------------------
template <typename Id>
__global__ void in_degree_kernel(const Id *E, uint64_t n_edges, uint64_t n, uint32_t *cnt,
                                 uint32_t *rank)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n_edges; base += stride) {
        const uint64_t e = base + threadIdx.x;
        unsigned long long v = e < n_edges ? (unsigned long long)E[2 * e + 1] : ~0ull;
        const bool act = v < n;   // ids are used as addresses: never trust them
        if (!act) v = ~0ull - lane;
        const uint32_t peers = __match_any_sync(kFull, v);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t old = 0;
        if (act && lane == leader) old = atomicAdd(cnt + v, (uint32_t)__popc(peers));
        old = __shfl_sync(kFull, old, leader);
        if (act) rank[e] = old + __popc(peers & lanemask_lt());
    }
}

// deg[x] = out-degree(x) + in-degree(x); deg[n] = 0 (so rowptr[n] is the total).
__global__ void deg_fill_kernel(const uint32_t *cnt, const uint32_t *seed_out, uint64_t n,
                                uint32_t d, int64_t *deg)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x <= n; x += stride)
        deg[x] = x == n ? 0 : (int64_t)cnt[x] + (x <= d ? seed_out[x] : d);
}

// ---------------------------------------------------------------------------
// In parts: store u at its rank in v's in part (no atomics).
// ---------------------------------------------------------------------------
template <typename Id>
__global__ void in_part_kernel(const Id *E, uint64_t n_edges, uint64_t n, uint32_t d,
                               const int64_t *rowptr, const uint32_t *rank,
                               const uint32_t *seed_out, Id *col, uint64_t col_len)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < n_edges; e += stride) {
        const uint64_t u = (uint64_t)E[2 * e], v = (uint64_t)E[2 * e + 1];
        if (u >= n || v >= n) continue;   // never trust ids used as addresses
        const uint64_t outdeg = v <= d ? seed_out[v] : d;
        const uint64_t pos = (uint64_t)rowptr[v] + outdeg + rank[e];
        if (pos < (uint64_t)rowptr[v + 1] && pos < col_len) col[pos] = (Id)u;
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
// Sorting the in parts.
// ---------------------------------------------------------------------------
template <typename Id>
__device__ __forceinline__ void in_range(uint64_t x, uint32_t d, const int64_t *rowptr,
                                         const uint32_t *seed_out, uint64_t &b, uint64_t &len)
{
    const uint64_t outdeg = x <= d ? seed_out[x] : d;
    b = rowptr[x] + outdeg;
    len = rowptr[x + 1] - b;
}

// Small parts (<= 32 entries): one warp each, rank by counting.  Hub parts
// (> 8192 entries) are queued for the bitmap pass.
template <typename Id>
__global__ void sort_small_kernel(uint64_t n, uint32_t d, const int64_t *rowptr,
                                  const uint32_t *seed_out, Id *col, unsigned long long *big_list,
                                  unsigned long long *big_count, uint64_t big_cap)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (uint64_t x0 = w0 * 32; x0 < n; x0 += warps * 32) {
        // each lane classifies one row; then the warp sorts the small ones
        const uint64_t x = x0 + lane;
        uint64_t b = 0, len = 0;
        if (x < n) in_range<Id>(x, d, rowptr, seed_out, b, len);
        if (len > kMidMax) {
            const unsigned long long slot = atomicAdd(big_count, 1ull);
            if (slot < big_cap) big_list[slot] = x;
        }
        uint32_t todo = __ballot_sync(kFull, len > 1 && len <= 32);
        while (todo) {
            const uint32_t src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint64_t sb = __shfl_sync(kFull, b, src);
            const uint32_t sl = (uint32_t)__shfl_sync(kFull, len, src);
            Id val = lane < sl ? col[sb + lane] : (Id)0;
            uint32_t rank = 0;
            for (uint32_t j = 0; j < sl; ++j) {
                const Id o = __shfl_sync(kFull, val, j);
                rank += (o < val) ? 1u : 0u;
            }
            __syncwarp();
            if (lane < sl) col[sb + rank] = val;
            __syncwarp();
        }
    }
}

// Bitonic sort of N = 32*EL values held by a warp, element i = j*32 + lane in
// v[j]; ascending.  Partners at distance s < 32 are in other lanes (shuffle),
// at s >= 32 in the same lane.
template <typename Id, int EL>
__device__ __forceinline__ void warp_bitonic(Id (&v)[EL], uint32_t lane)
{
    constexpr uint32_t N = 32u * EL;
#pragma unroll
    for (uint32_t k = 2; k <= N; k <<= 1) {
#pragma unroll
        for (uint32_t s = k >> 1; s > 0; s >>= 1) {
            if (s >= 32) {
                const uint32_t js = s >> 5;
#pragma unroll
                for (uint32_t j = 0; j < (uint32_t)EL; ++j) {
                    const uint32_t jp = j ^ js;
                    if (jp > j) {
                        const uint32_t i = j * 32 + lane;
                        const bool up = (i & k) == 0;
                        const Id a = v[j], b = v[jp];
                        if ((a > b) == up) {
                            v[j] = b;
                            v[jp] = a;
                        }
                    }
                }
            } else {
#pragma unroll
                for (uint32_t j = 0; j < (uint32_t)EL; ++j) {
                    const uint32_t i = j * 32 + lane;
                    const Id o = __shfl_xor_sync(kFull, v[j], s);
                    const bool up = (i & k) == 0;
                    const bool lower = (i & s) == 0;   // i < partner
                    v[j] = (lower == up) ? (v[j] < o ? v[j] : o) : (v[j] > o ? v[j] : o);
                }
            }
        }
    }
}

template <typename Id, int EL>
__device__ __forceinline__ void warp_sort_part(Id *col, uint64_t b, uint32_t len, uint32_t lane)
{
    const Id pad = (Id)(~(typename std::make_unsigned<Id>::type)0 >> 1);
    Id v[EL];
#pragma unroll
    for (int j = 0; j < EL; ++j) {
        const uint32_t i = j * 32 + lane;
        v[j] = i < len ? col[b + i] : pad;
    }
    warp_bitonic<Id, EL>(v, lane);
#pragma unroll
    for (int j = 0; j < EL; ++j) {
        const uint32_t i = j * 32 + lane;
        if (i < len) col[b + i] = v[j];
    }
}

// Parts of 33..256 entries: one warp each, the register bitonic network.
template <typename Id>
__global__ void sort_warp_kernel(uint64_t n, uint32_t d, const int64_t *rowptr,
                                 const uint32_t *seed_out, Id *col)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    for (uint64_t x0 = w0 * 32; x0 < n; x0 += warps * 32) {
        const uint64_t x = x0 + lane;
        uint64_t b = 0, len = 0;
        if (x < n) in_range<Id>(x, d, rowptr, seed_out, b, len);
        uint32_t todo = __ballot_sync(kFull, len > 32 && len <= 256);
        while (todo) {
            const uint32_t src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint64_t sb = __shfl_sync(kFull, b, src);
            const uint32_t sl = (uint32_t)__shfl_sync(kFull, len, src);
            if (sl <= 64) warp_sort_part<Id, 2>(col, sb, sl, lane);
            else if (sl <= 128) warp_sort_part<Id, 4>(col, sb, sl, lane);
            else warp_sort_part<Id, 8>(col, sb, sl, lane);
        }
    }
}

// Parts of 257..8192 entries: a CTA tests 512 rows at a time, queues those in
// shared memory and bitonic-sorts each in shared memory.
template <typename Id>
__global__ void __launch_bounds__(512) sort_mid_kernel(uint64_t n, uint32_t d, const int64_t *rowptr,
                                                       const uint32_t *seed_out, Id *col)
{
    extern __shared__ __align__(16) unsigned char smem[];
    Id *buf = reinterpret_cast<Id *>(smem);
    __shared__ unsigned long long s_rows[512];
    __shared__ unsigned int s_cnt;
    for (uint64_t r0 = (uint64_t)blockIdx.x * blockDim.x; r0 < n; r0 += (uint64_t)gridDim.x * blockDim.x) {
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        const uint64_t x = r0 + threadIdx.x;
        if (x < n) {
            uint64_t b, len;
            in_range<Id>(x, d, rowptr, seed_out, b, len);
            if (len > 256 && len <= kMidMax) s_rows[atomicAdd(&s_cnt, 1u)] = x;
        }
        __syncthreads();
        const uint32_t cnt = s_cnt;
        for (uint32_t m = 0; m < cnt; ++m) {
            uint64_t b, len;
            in_range<Id>(s_rows[m], d, rowptr, seed_out, b, len);
            uint32_t N = 512;
            while (N < len) N <<= 1;
            for (uint32_t i = threadIdx.x; i < N; i += blockDim.x)
                buf[i] = i < len ? col[b + i] : (Id)(~(typename std::make_unsigned<Id>::type)0 >> 1);
            __syncthreads();
            for (uint32_t k = 2; k <= N; k <<= 1) {
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t i = threadIdx.x; i < N; i += blockDim.x) {
                        const uint32_t ixj = i ^ j;
                        if (ixj > i) {
                            const bool up = (i & k) == 0;
                            const Id a = buf[i], c = buf[ixj];
                            if ((a > c) == up) {
                                buf[i] = c;
                                buf[ixj] = a;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
            for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) col[b + i] = buf[i];
            __syncthreads();
        }
    }
}

// Large parts: bitmap over node ids (x, n): set one bit per entry, then write the
// set bits in order.  The entries of an in part are distinct and all > x.
template <typename Id>
__global__ void bitmap_set_kernel(const Id *col, uint64_t b, uint64_t len, uint64_t lo,
                                  uint64_t n, uint32_t *bits)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += stride) {
        const uint64_t x = (uint64_t)col[b + i];
        if (x < lo || x >= n) continue;
        const uint64_t v = x - lo;
        atomicOr(bits + (v >> 5), 1u << (v & 31));
    }
}

// Per 32-bit word: population count (pass 1) then ordered write (pass 2) using
// an exclusive scan of the word counts computed by scan_kernel on int64 counts.
__global__ void bitmap_count_kernel(const uint32_t *bits, uint64_t words, int64_t *counts)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride)
        counts[w] = __popc(bits[w]);
}

template <typename Id>
__global__ void bitmap_write_kernel(const uint32_t *bits, uint64_t words, const int64_t *offs,
                                    uint64_t lo, Id *col, uint64_t b, uint64_t len)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += stride) {
        uint32_t m = bits[w];
        uint64_t o = (uint64_t)offs[w];
        while (m && o < len) {
            const uint32_t bit = __ffs(m) - 1;
            m &= m - 1;
            col[b + o++] = (Id)(lo + w * 32 + bit);
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
    uint64_t deg_off, status_off, ctr_off, err_off, seed_out_off, cursor_off, rank_off, lists_off,
        bits_off, counts_off, total;
    uint64_t n_tiles, big_cap, bit_words;
};

CsrLayout csr_layout(uint64_t n, uint32_t d, uint64_t n_edges)
{
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    CsrLayout L{};
    L.n_tiles = (n + 1 + kScanTile - 1) / kScanTile;
    L.big_cap = (n * d) / 4096 + 16;   // hub parts above 8192 entries: at most 2E / 8192
    L.bit_words = (n + 31) / 32 + 1;
    uint64_t o = 0;
    L.deg_off = o;        o += al(8 * (n + 1));
    L.status_off = o;     o += al(8 * L.n_tiles);
    L.ctr_off = o;        o += 256;                       // scan tile counter + list counters
    L.err_off = o;        o += 256;
    L.seed_out_off = o;   o += al(4 * (d + 1));
    L.cursor_off = o;     o += al(4 * n);                  // in-degree counts
    L.rank_off = o;       o += al(4 * n_edges);            // rank of each pair in its in part
    L.lists_off = o;      o += al(8 * L.big_cap);
    L.bits_off = o;       o += al(4 * L.bit_words);
    L.counts_off = o;     o += al(8 * (L.bit_words + 1));
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

template <typename Id>
int build_csr(const pa_params *prm, const GenPlan &p, const Id *E, int64_t *rowptr, Id *col,
              unsigned char *scratch, const CsrLayout &L, cudaStream_t s)
{
    const uint64_t n = prm->n;
    const uint32_t d = prm->d;
    int64_t *deg = (int64_t *)(scratch + L.deg_off);
    uint32_t *seed_out = (uint32_t *)(scratch + L.seed_out_off);
    uint32_t *cursor = (uint32_t *)(scratch + L.cursor_off);
    unsigned long long *lists = (unsigned long long *)(scratch + L.lists_off);
    unsigned long long *ctrs = (unsigned long long *)(scratch + L.ctr_off);
    uint32_t *err = (uint32_t *)(scratch + L.err_off);

    uint32_t *rank = (uint32_t *)(scratch + L.rank_off);
    cudaError_t e = cudaMemsetAsync(err, 0, 4, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(cursor, 0, 4 * n, s);
    if (e != cudaSuccess) return set_cuda_error(e);

    seed_out_kernel<Id><<<1, 64, 0, s>>>(E, p.seed_edges, d, seed_out);
    if (p.n_edges)
        in_degree_kernel<Id><<<grid_for(p.n_edges, 256), 256, 0, s>>>(E, p.n_edges, n, cursor, rank);
    deg_fill_kernel<<<grid_for(n + 1, 256), 256, 0, s>>>(cursor, seed_out, n, d, deg);
    int rc = run_scan(deg, rowptr, n + 1, scratch, L, s);   // deg[n] = 0: rowptr[n] = total
    if (rc != PA_OK) return rc;

    const uint64_t col_len = 2 * p.n_edges;
    out_part_kernel<Id><<<grid_for(n * d, 256), 256, 0, s>>>(E, rowptr, col, n, d, p.seed_edges,
                                                             col_len);
    in_part_kernel<Id><<<grid_for(p.n_edges, 256), 256, 0, s>>>(E, p.n_edges, n, d, rowptr, rank,
                                                                seed_out, col, col_len);
    // list counters live after the scan tile counter
    e = cudaMemsetAsync(ctrs + 1, 0, 16, s);
    if (e != cudaSuccess) return set_cuda_error(e);
    unsigned long long *big_list = lists;
    sort_small_kernel<Id><<<grid_for(n, 256), 256, 0, s>>>(n, d, rowptr, seed_out, col, big_list,
                                                           ctrs + 2, L.big_cap);
    sort_warp_kernel<Id><<<grid_for(n, 256), 256, 0, s>>>(n, d, rowptr, seed_out, col);
    const size_t smem = kMidMax * sizeof(Id);
    e = cudaFuncSetAttribute(sort_mid_kernel<Id>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
    if (e != cudaSuccess) return set_cuda_error(e);
    sort_mid_kernel<Id><<<grid_for(n, 512, 4), 512, smem, s>>>(n, d, rowptr, seed_out, col);
    e = cudaGetLastError();
    if (e != cudaSuccess) return set_cuda_error(e);

    // Large parts: few; the host reads their list and handles them one by one.
    unsigned long long counts[2] = {0, 0};
    e = cudaMemcpyAsync(counts, ctrs + 1, 16, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (counts[1] > L.big_cap) return PA_ERR_CAPACITY;
    if (counts[1]) {
        std::vector<unsigned long long> big(counts[1]);
        big_list = lists;
        e = cudaMemcpyAsync(big.data(), big_list, 8 * counts[1], cudaMemcpyDeviceToHost, s);
        std::vector<int64_t> rp(2);
        std::vector<uint32_t> so(d + 1);
        if (e == cudaSuccess) e = cudaMemcpyAsync(so.data(), seed_out, 4 * (d + 1), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return set_cuda_error(e);
        uint32_t *bits = (uint32_t *)(scratch + L.bits_off);
        int64_t *wcounts = (int64_t *)(scratch + L.counts_off);
        for (unsigned long long x : big) {
            e = cudaMemcpyAsync(rp.data(), rowptr + x, 16, cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
            if (e != cudaSuccess) return set_cuda_error(e);
            const uint64_t outdeg = x <= d ? so[x] : d;
            const uint64_t b = rp[0] + outdeg, len = rp[1] - b;
            const uint64_t lo = x + 1, words = (n - lo + 31) / 32;
            e = cudaMemsetAsync(bits, 0, 4 * words, s);
            if (e != cudaSuccess) return set_cuda_error(e);
            bitmap_set_kernel<Id><<<grid_for(len, 256), 256, 0, s>>>(col, b, len, lo, n, bits);
            bitmap_count_kernel<<<grid_for(words, 256), 256, 0, s>>>(bits, words, wcounts);
            rc = run_scan(wcounts, wcounts, words, scratch, L, s);
            if (rc != PA_OK) return rc;
            bitmap_write_kernel<Id><<<grid_for(words, 256), 256, 0, s>>>(bits, words, wcounts, lo,
                                                                         col, b, len);
            e = cudaGetLastError();
            if (e != cudaSuccess) return set_cuda_error(e);
        }
    }
    uint32_t herr = 0;
    e = cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_cuda_error(e);
    return (int)herr;
}

}  // namespace
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
    *rowptr_bytes = 8 * (prm->n + 1);
    *col_bytes = 2 * p.n_edges * p.id_bytes;
    *scratch_bytes = csr_layout(prm->n, prm->d, p.n_edges).total;
    return PA_OK;
}

int pa_build_csr(const pa_params *prm, const void *d_edges, int64_t *d_rowptr, void *d_col,
                 void *d_scratch, uint64_t scratch_bytes, void *stream)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !d_rowptr || !d_col || !d_scratch) return PA_ERR_INVALID;
    const CsrLayout L = csr_layout(prm->n, prm->d, p.n_edges);
    if (scratch_bytes < L.total) return PA_ERR_CAPACITY;
    if (p.id_bytes == 8)
        return build_csr<int64_t>(prm, p, (const int64_t *)d_edges, d_rowptr, (int64_t *)d_col,
                                  (unsigned char *)d_scratch, L, (cudaStream_t)stream);
    return build_csr<int32_t>(prm, p, (const int32_t *)d_edges, d_rowptr, (int32_t *)d_col,
                              (unsigned char *)d_scratch, L, (cudaStream_t)stream);
}

}  // extern "C"
