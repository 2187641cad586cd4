// pa_stream.cu -- the edge list out of the device: formatted on the device,
// copied out in chunks, handed to a sink in order.
//
// The reference writes a graph with one ostream insertion per number
// (PAHelper::writeGraphToDisk, src/PA/SPA/PAHelper.hpp:163-177: rows u = M..N-1,
// one "u v" line per slot) and never writes the cuPPA graph at all
// (src/PA/cuPPA/cuPPA_1.cu:247-250).  Here the "u v\n" text (or the binary
// (src, dst) pairs) is produced by the GPU, and the host only moves bytes:
//
//   stream F (the caller's):  format chunk c into device staging buffer c&1
//   stream C (internal):      copy chunk c to pinned host buffer c&1
//   writer thread:            sink(pinned buffer c&1) once its copy is done
//
// so formatting chunk c+1, copying chunk c and the sink of chunk c-1 overlap;
// the host link and the sink are the bounds, not the formatting.  Text is made
// in two passes over a chunk -- each tile's byte count, an exclusive scan of the
// tile counts, then each tile formats its lines in shared memory and copies them
// to its offset -- which reads the ids twice instead of waiting on neighbouring
// tiles.  Seed edges (at most 528) are formatted on the host, from their closed
// form, ahead of the first chunk.
//
// Both layouts stream in the PAIRS order: the seed edges, then rows u =
// d+1..n-1 in slot order.  A row's source is its node id, so SLOTS needs no
// stored sources; PAIRS binary output is copied straight from the edge list.
#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "pa_device.cuh"
#include "pa_internal.h"

namespace pa {
namespace {

constexpr uint32_t kFmtThreads = 256;
constexpr uint32_t kTileEdges = 2048;              // edges per tile at most (8 per thread)
constexpr uint32_t kPerThread = kTileEdges / kFmtThreads;
constexpr uint64_t kChunkEdgesAuto = 1ull << 24;

// Decimal digits of x (ids are below 2^40: at most 13 digits).
__host__ __device__ __forceinline__ uint32_t dec_digits(uint64_t x)
{
    uint32_t n = 1;
    uint64_t p = 10;
    for (int i = 1; i < 13; ++i) {
        n += x >= p ? 1u : 0u;
        p *= 10;
    }
    return n;
}

__device__ __forceinline__ void put_dec(unsigned char *p, uint64_t x, uint32_t len)
{
    for (uint32_t i = len; i > 0; --i) {
        p[i - 1] = (unsigned char)('0' + x % 10);
        x /= 10;
    }
}

struct FmtArgs {
    const void *edges;        // PAIRS: the pair list; SLOTS: the id array
    unsigned char *out;       // this chunk's staging buffer
    unsigned long long *tile_len;   // per tile: byte count, then (after the scan) offset
    unsigned long long *total;      // the chunk's byte count
    uint64_t row0;            // first row of the chunk (row r = node u_first + r)
    uint64_t rows;            // rows in the chunk
    uint64_t u_first;
    uint64_t seed_edges;      // PAIRS offset of row 0
    uint32_t d;
    uint32_t tile_rows;       // rows per tile (tile_rows * d <= kTileEdges)
    uint64_t n_tiles;
};

// Target of slot k of row r.
template <typename Id, bool Slots>
__device__ __forceinline__ uint64_t target(const FmtArgs &f, uint64_t r, uint32_t k)
{
    const Id *E = reinterpret_cast<const Id *>(f.edges);
    const uint64_t g = r * f.d + k;
    return (uint64_t)(Slots ? E[g] : E[2 * (f.seed_edges + g) + 1]);
}

// Line lengths of this thread's edges of tile t (kPerThread, strided by the
// block), and their sum.
template <typename Id, bool Slots>
__device__ __forceinline__ uint32_t line_lengths(const FmtArgs &f, uint64_t t, uint32_t (&len)[kPerThread],
                                                 uint64_t (&src)[kPerThread],
                                                 uint64_t (&dst)[kPerThread])
{
    const uint64_t r_begin = f.row0 + t * f.tile_rows;
    const uint64_t r_end = min(f.row0 + f.rows, r_begin + f.tile_rows);
    const uint32_t n_edges = (uint32_t)(r_end - r_begin) * f.d;
    uint32_t sum = 0;
#pragma unroll
    for (uint32_t j = 0; j < kPerThread; ++j) {
        const uint32_t x = threadIdx.x + j * kFmtThreads;
        len[j] = 0;
        if (x < n_edges) {
            const uint32_t rr = x / f.d;
            const uint64_t r = r_begin + rr;
            src[j] = f.u_first + r;
            dst[j] = target<Id, Slots>(f, r, x - rr * f.d);
            len[j] = dec_digits(src[j]) + dec_digits(dst[j]) + 2;
            sum += len[j];
        }
    }
    return sum;
}

__device__ __forceinline__ uint32_t block_sum(uint32_t v, uint32_t *red)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    uint32_t t = 0;
    if (threadIdx.x == 0)
        for (uint32_t w = 0; w < kFmtThreads / 32; ++w) t += red[w];
    return t;   // valid in thread 0
}

// Pass 1: bytes of every tile of the chunk.
template <typename Id, bool Slots>
__global__ void __launch_bounds__(kFmtThreads) text_len_kernel(const FmtArgs f)
{
    __shared__ uint32_t red[kFmtThreads / 32];
    for (uint64_t t = blockIdx.x; t < f.n_tiles; t += gridDim.x) {
        uint32_t len[kPerThread];
        uint64_t src[kPerThread], dst[kPerThread];
        const uint32_t s = line_lengths<Id, Slots>(f, t, len, src, dst);
        const uint32_t tot = block_sum(s, red);
        if (threadIdx.x == 0) f.tile_len[t] = tot;
        __syncthreads();
    }
}

// Exclusive scan of the tile byte counts in place (one block), and the total.
__global__ void __launch_bounds__(1024) tile_scan_kernel(unsigned long long *v, uint64_t n,
                                                         unsigned long long *total)
{
    __shared__ unsigned long long part[1024];
    const uint64_t per = (n + 1023) / 1024;
    const uint64_t b = threadIdx.x * per, e = min(n, b + per);
    unsigned long long s = 0;
    for (uint64_t i = b; i < e; ++i) s += v[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (uint32_t o = 1; o < 1024; o <<= 1) {   // Hillis-Steele inclusive scan
        const unsigned long long add = threadIdx.x >= o ? part[threadIdx.x - o] : 0ull;
        __syncthreads();
        part[threadIdx.x] += add;
        __syncthreads();
    }
    unsigned long long run = part[threadIdx.x] - s;
    for (uint64_t i = b; i < e; ++i) {
        const unsigned long long x = v[i];
        v[i] = run;
        run += x;
    }
    if (threadIdx.x == 1023) *total = part[1023];
}

// The four 32-bit words starting s bytes (s < 16, a multiple-of-4 part ws = s/4
// and a byte part) into the 32 bytes a:b.
__device__ __forceinline__ uint4 shift_bytes(const uint4 &a, const uint4 &b, uint32_t ws,
                                             uint32_t bits)
{
    uint32_t x[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    uint4 r;
    // ws is the same for the whole block: the branches do not diverge, and the
    // constant indices keep x in registers
    switch (ws) {
    case 0:
        r = make_uint4(__funnelshift_r(x[0], x[1], bits), __funnelshift_r(x[1], x[2], bits),
                       __funnelshift_r(x[2], x[3], bits), __funnelshift_r(x[3], x[4], bits));
        break;
    case 1:
        r = make_uint4(__funnelshift_r(x[1], x[2], bits), __funnelshift_r(x[2], x[3], bits),
                       __funnelshift_r(x[3], x[4], bits), __funnelshift_r(x[4], x[5], bits));
        break;
    case 2:
        r = make_uint4(__funnelshift_r(x[2], x[3], bits), __funnelshift_r(x[3], x[4], bits),
                       __funnelshift_r(x[4], x[5], bits), __funnelshift_r(x[5], x[6], bits));
        break;
    default:
        r = make_uint4(__funnelshift_r(x[3], x[4], bits), __funnelshift_r(x[4], x[5], bits),
                       __funnelshift_r(x[5], x[6], bits), __funnelshift_r(x[6], x[7], bits));
        break;
    }
    return r;
}

// Copy `len` bytes of the tile text to out (any alignment): the bytes up to the
// first 16-byte boundary of out and after the last one go one by one, the rest
// as aligned 16-byte stores, each assembled from two aligned 16-byte shared
// loads (the shared buffer carries 32 bytes of slack past the text).
__device__ __forceinline__ void copy_out(unsigned char *out, const unsigned char *s_text,
                                         uint32_t len)
{
    uint32_t head = (uint32_t)((16u - (reinterpret_cast<uintptr_t>(out) & 15u)) & 15u);
    if (head > len) head = len;
    const uint32_t chunks = (len - head) / 16u;
    const uint32_t tail0 = head + chunks * 16u;
    if (threadIdx.x < head) out[threadIdx.x] = s_text[threadIdx.x];
    if (threadIdx.x < len - tail0) out[tail0 + threadIdx.x] = s_text[tail0 + threadIdx.x];
    const uint32_t ws = (head & 15u) >> 2, bits = (head & 3u) * 8u;
    const uint4 *src = reinterpret_cast<const uint4 *>(s_text) + (head >> 4);
    uint4 *dst = reinterpret_cast<uint4 *>(out + head);
    for (uint32_t k = threadIdx.x; k < chunks; k += kFmtThreads)
        dst[k] = shift_bytes(src[k], src[k + 1], ws, bits);
}

// Pass 2: each tile formats its lines into shared memory at their block-scanned
// offsets, then copies the bytes to the chunk buffer at the tile's offset.
template <typename Id, bool Slots>
__global__ void __launch_bounds__(kFmtThreads) text_write_kernel(const FmtArgs f)
{
    extern __shared__ __align__(16) unsigned char s_text[];
    __shared__ uint32_t s_warp[kFmtThreads / 32];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (uint64_t t = blockIdx.x; t < f.n_tiles; t += gridDim.x) {
        uint32_t len[kPerThread];
        uint64_t src[kPerThread], dst[kPerThread];
        line_lengths<Id, Slots>(f, t, len, src, dst);
        // Lines go out in edge order.  Stripe j is edges [256j, 256j + 256) of
        // the tile, one per thread, so a line's offset is the bytes of the
        // earlier stripes plus an exclusive scan across the block in its stripe.
        uint32_t base = 0;   // bytes of all earlier stripes
#pragma unroll
        for (uint32_t j = 0; j < kPerThread; ++j) {
            uint32_t x = len[j];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= (uint32_t)o) x += y;
            }
            if (lane == 31) s_warp[warp] = x;
            __syncthreads();
            uint32_t before = 0, stripe = 0;
#pragma unroll
            for (uint32_t w = 0; w < kFmtThreads / 32; ++w) {
                const uint32_t v = s_warp[w];
                before += w < warp ? v : 0u;
                stripe += v;
            }
            const uint32_t off = base + before + x - len[j];
            if (len[j]) {
                const uint32_t ls = dec_digits(src[j]);
                unsigned char *p = s_text + off;
                put_dec(p, src[j], ls);
                p[ls] = ' ';
                put_dec(p + ls + 1, dst[j], len[j] - ls - 2);
                p[len[j] - 1] = '\n';
            }
            base += stripe;
            __syncthreads();
        }
        const unsigned long long o = f.tile_len[t];
        copy_out(f.out + o, s_text, base);
        __syncthreads();
    }
}

// Binary pairs of a SLOTS chunk.
template <typename Id>
__global__ void __launch_bounds__(kFmtThreads) pairs_from_slots_kernel(const FmtArgs f)
{
    const Id *S = reinterpret_cast<const Id *>(f.edges);
    Id *out = reinterpret_cast<Id *>(f.out);
    const uint64_t n = f.rows * f.d;
    const uint64_t g0 = f.row0 * f.d;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n;
         x += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t r = x / f.d;
        out[2 * x] = (Id)(f.u_first + f.row0 + r);
        out[2 * x + 1] = S[g0 + x];
    }
}

int sm_count()
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms;
}

// Host copy of the seed edges' closed form (pa_device.cuh seed_edge_of).
void host_seed_edge(uint64_t e, uint32_t d, uint32_t mode, uint64_t &src, uint64_t &dst)
{
    if (mode == PA_SEED_CLIQUE) {
        uint64_t v = 1, base = 0;
        while (base + v <= e) { base += v; ++v; }
        src = v;
        dst = e - base;
    } else {
        src = d;
        dst = e;
    }
}

template <typename Id, bool Slots>
int launch_text(const FmtArgs &f, uint32_t smem, cudaStream_t s)
{
    const uint32_t grid = (uint32_t)std::min<uint64_t>(f.n_tiles, (uint64_t)sm_count() * 8);
    text_len_kernel<Id, Slots><<<grid, kFmtThreads, 0, s>>>(f);
    tile_scan_kernel<<<1, 1024, 0, s>>>(f.tile_len, f.n_tiles, f.total);
    auto wk = text_write_kernel<Id, Slots>;
    cudaError_t e = cudaFuncSetAttribute(wk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_cuda_error(e);
    wk<<<grid, kFmtThreads, smem, s>>>(f);
    e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

int launch_text_any(uint32_t id_bytes, bool slots, const FmtArgs &f, uint32_t smem, cudaStream_t s)
{
    if (id_bytes == 8)
        return slots ? launch_text<int64_t, true>(f, smem, s) : launch_text<int64_t, false>(f, smem, s);
    return slots ? launch_text<int32_t, true>(f, smem, s) : launch_text<int32_t, false>(f, smem, s);
}

// The writer thread: sinks finished copies in order.
struct Writer {
    pa_sink_fn sink;
    void *ctx;
    void *buf[2] = {nullptr, nullptr};
    cudaEvent_t copied[2] = {nullptr, nullptr};
    std::mutex mu;
    std::condition_variable cv;
    std::deque<std::pair<int, uint64_t>> jobs;   // (buffer, bytes)
    bool busy[2] = {false, false};
    bool done = false;
    int status = PA_OK;
    cudaError_t cuda = cudaSuccess;

    void run()
    {
        for (;;) {
            std::pair<int, uint64_t> job;
            bool failed;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return !jobs.empty() || done; });
                if (jobs.empty()) return;
                job = jobs.front();
                jobs.pop_front();
                failed = status != PA_OK;
            }
            const cudaError_t e = cudaEventSynchronize(copied[job.first]);
            int rc = PA_OK;
            if (e != cudaSuccess) rc = PA_ERR_CUDA;
            else if (!failed && job.second && sink(ctx, buf[job.first], job.second) != 0)
                rc = PA_ERR_IO;
            std::lock_guard<std::mutex> lk(mu);
            if (e != cudaSuccess && cuda == cudaSuccess) cuda = e;
            if (rc != PA_OK && status == PA_OK) status = rc;
            busy[job.first] = false;
            cv.notify_all();
        }
    }
};

// Staging memory kept between calls.  Pinning a few hundred MB of host memory
// and freeing it again (which waits for the device) cost ~0.3 s per call, a
// sixth of a 2^30-node text write; the buffers grow to the largest request and
// stay until pa_stream_trim.  One call at a time uses the cached set; a
// concurrent call allocates its own.
struct Staging {
    int device = -1;
    void *host[2] = {nullptr, nullptr};
    uint64_t host_bytes = 0;
    void *dev[2] = {nullptr, nullptr};
    uint64_t dev_bytes = 0;
    void *meta = nullptr;
    uint64_t meta_bytes = 0;
    unsigned long long *h_total = nullptr;

    void free_all()
    {
        for (int i = 0; i < 2; ++i) {
            if (host[i]) cudaFreeHost(host[i]);
            if (dev[i]) cudaFree(dev[i]);
            host[i] = dev[i] = nullptr;
        }
        if (meta) cudaFree(meta);
        if (h_total) cudaFreeHost(h_total);
        meta = nullptr;
        h_total = nullptr;
        host_bytes = dev_bytes = meta_bytes = 0;
    }
};

std::mutex g_stage_mu;
Staging g_stage;
bool g_stage_busy = false;

// Take the cached set (or an empty one) and grow it to the sizes asked.
cudaError_t stage_acquire(Staging &S, bool &cached, uint64_t host_bytes, uint64_t dev_bytes,
                          uint64_t meta_bytes)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return e;
    {
        std::lock_guard<std::mutex> lk(g_stage_mu);
        cached = !g_stage_busy;
        if (cached) {
            g_stage_busy = true;
            if (g_stage.device == device) S = g_stage;
            else g_stage.free_all();   // cached for another device: let it go
            g_stage = Staging();
        }
    }
    if (S.device != device) S = Staging();   // nothing cached for this device
    S.device = device;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        if (S.host_bytes < host_bytes) {
            if (S.host[i]) cudaFreeHost(S.host[i]);
            S.host[i] = nullptr;
            e = cudaMallocHost(&S.host[i], host_bytes);
        }
        if (e == cudaSuccess && S.dev_bytes < dev_bytes) {
            if (S.dev[i]) cudaFree(S.dev[i]);
            S.dev[i] = nullptr;
            e = cudaMalloc(&S.dev[i], dev_bytes);
        }
    }
    if (e == cudaSuccess) {
        S.host_bytes = std::max(S.host_bytes, host_bytes);
        S.dev_bytes = std::max(S.dev_bytes, dev_bytes);
    }
    if (e == cudaSuccess && S.meta_bytes < meta_bytes) {
        if (S.meta) cudaFree(S.meta);
        S.meta = nullptr;
        e = cudaMalloc(&S.meta, meta_bytes);
        if (e == cudaSuccess) S.meta_bytes = meta_bytes;
    }
    if (e == cudaSuccess && !S.h_total)
        e = cudaMallocHost(reinterpret_cast<void **>(&S.h_total), 2 * sizeof(unsigned long long));
    return e;
}

void stage_release(Staging &S, bool cached, bool keep)
{
    if (cached && keep) {
        std::lock_guard<std::mutex> lk(g_stage_mu);
        g_stage = S;
        g_stage_busy = false;
        return;
    }
    S.free_all();
    if (cached) {
        std::lock_guard<std::mutex> lk(g_stage_mu);
        g_stage_busy = false;
    }
}

}  // namespace

int stream_edges(const pa_params *prm, const GenPlan &p, const void *d_edges, int format,
                 uint64_t chunk_edges, pa_sink_fn sink, void *ctx, cudaStream_t s,
                 uint64_t *bytes_out)
{
    const uint32_t d = prm->d;
    const uint64_t rows = prm->n - p.u_first;
    const bool text = format == PA_FORMAT_TEXT;
    const uint64_t pair_bytes = 2ull * p.id_bytes;
    uint64_t written = 0;

    // seed edges, on the host
    {
        std::string head;
        std::vector<unsigned char> bin;
        for (uint64_t e = 0; e < p.seed_edges; ++e) {
            uint64_t a, b;
            host_seed_edge(e, d, prm->seed_mode, a, b);
            if (text) {
                head += std::to_string(a);
                head += ' ';
                head += std::to_string(b);
                head += '\n';
            } else if (p.id_bytes == 8) {
                const int64_t v[2] = {(int64_t)a, (int64_t)b};
                bin.insert(bin.end(), (const unsigned char *)v, (const unsigned char *)v + 16);
            } else {
                const int32_t v[2] = {(int32_t)a, (int32_t)b};
                bin.insert(bin.end(), (const unsigned char *)v, (const unsigned char *)v + 8);
            }
        }
        const void *data = text ? (const void *)head.data() : (const void *)bin.data();
        const uint64_t nb = text ? head.size() : bin.size();
        if (nb && sink(ctx, data, nb) != 0) return PA_ERR_IO;
        written += nb;
    }
    if (rows == 0) {
        if (bytes_out) *bytes_out = written;
        return PA_OK;
    }

    // chunk geometry: whole tiles of tile_rows rows
    const uint32_t tile_rows = kTileEdges / d;
    if (chunk_edges == 0) chunk_edges = kChunkEdgesAuto;
    uint64_t chunk_rows = std::max<uint64_t>(1, chunk_edges / d);
    chunk_rows = (chunk_rows + tile_rows - 1) / tile_rows * tile_rows;
    chunk_rows = std::min(chunk_rows, rows);
    const uint64_t n_chunks = (rows + chunk_rows - 1) / chunk_rows;
    const uint32_t max_line = 2 * dec_digits(prm->n - 1) + 2;
    const uint64_t chunk_cap = text ? chunk_rows * d * max_line : chunk_rows * d * pair_bytes;
    const uint64_t tiles_cap = (chunk_rows + tile_rows - 1) / tile_rows;
    const uint32_t smem = tile_rows * d * max_line + 32;   // + slack read by copy_out
    const bool direct = !text && !p.slots;   // PAIRS binary: copy the edge list itself

    Writer W;
    W.sink = sink;
    W.ctx = ctx;
    Staging St;
    bool cached = false;
    cudaError_t e = stage_acquire(St, cached, chunk_cap, direct ? 0 : chunk_cap,
                                  text ? 2 * (tiles_cap + 1) * sizeof(unsigned long long) : 0);
    unsigned char *stage[2] = {(unsigned char *)St.dev[0], (unsigned char *)St.dev[1]};
    unsigned long long *meta = (unsigned long long *)St.meta;   // 2 x (tile counts + 1 total)
    unsigned long long *h_total = St.h_total;
    W.buf[0] = St.host[0];
    W.buf[1] = St.host[1];
    cudaEvent_t formatted[2] = {nullptr, nullptr};
    cudaStream_t cs = nullptr;
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&W.copied[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&formatted[i], cudaEventDisableTiming);
    }

    std::thread writer;
    int rc = PA_OK;
    if (e == cudaSuccess) writer = std::thread([&W] { W.run(); });
    for (uint64_t c = 0; c < n_chunks && e == cudaSuccess && rc == PA_OK; ++c) {
        const int b = (int)(c & 1);
        const uint64_t r0 = c * chunk_rows;
        const uint64_t rc_rows = std::min(chunk_rows, rows - r0);
        FmtArgs f;
        f.edges = d_edges;
        f.out = stage[b];
        f.tile_len = meta ? meta + b * (tiles_cap + 1) : nullptr;
        f.total = meta ? meta + b * (tiles_cap + 1) + tiles_cap : nullptr;
        f.row0 = r0;
        f.rows = rc_rows;
        f.u_first = p.u_first;
        f.seed_edges = p.slots ? 0 : p.seed_edges;
        f.d = d;
        f.tile_rows = tile_rows;
        f.n_tiles = (rc_rows + tile_rows - 1) / tile_rows;
        uint64_t nbytes = rc_rows * d * pair_bytes;
        const void *from = stage[b];
        if (!direct) {
            // the staging buffer of chunk c - 2 must have been copied out
            if (c >= 2) e = cudaStreamWaitEvent(s, W.copied[b], 0);
            if (e != cudaSuccess) break;
            if (text) {
                rc = launch_text_any(p.id_bytes, p.slots, f, smem, s);
                if (rc != PA_OK) break;
                e = cudaMemcpyAsync(h_total + b, f.total, sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, s);
            } else {
                const uint32_t grid = (uint32_t)std::min<uint64_t>((rc_rows * d + 255) / 256,
                                                                   (uint64_t)sm_count() * 16);
                if (p.id_bytes == 8) pairs_from_slots_kernel<int64_t><<<grid, 256, 0, s>>>(f);
                else pairs_from_slots_kernel<int32_t><<<grid, 256, 0, s>>>(f);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaEventRecord(formatted[b], s);
            if (e == cudaSuccess && text) {
                e = cudaEventSynchronize(formatted[b]);
                nbytes = h_total[b];
            }
            if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, formatted[b], 0);
        } else {
            from = (const unsigned char *)d_edges + (p.seed_edges + r0 * d) * pair_bytes;
            if (c == 0) {   // the edge list was written on the caller's stream
                e = cudaEventRecord(formatted[0], s);
                if (e == cudaSuccess) e = cudaStreamWaitEvent(cs, formatted[0], 0);
            }
        }
        if (e != cudaSuccess) break;
        {
            // the pinned buffer of chunk c - 2 must have been sunk
            std::unique_lock<std::mutex> lk(W.mu);
            W.cv.wait(lk, [&] { return !W.busy[b]; });
            if (W.status != PA_OK) break;
            W.busy[b] = true;
        }
        e = cudaMemcpyAsync(W.buf[b], from, nbytes, cudaMemcpyDeviceToHost, cs);
        if (e == cudaSuccess) e = cudaEventRecord(W.copied[b], cs);
        {
            std::lock_guard<std::mutex> lk(W.mu);
            if (e == cudaSuccess) W.jobs.emplace_back(b, nbytes);
            else W.busy[b] = false;
        }
        W.cv.notify_all();
        written += nbytes;
    }
    if (writer.joinable()) {
        {
            std::lock_guard<std::mutex> lk(W.mu);
            W.done = true;
        }
        W.cv.notify_all();
        writer.join();
    }
    if (cs) {
        const cudaError_t e2 = cudaStreamSynchronize(cs);
        if (e == cudaSuccess) e = e2;
        cudaStreamDestroy(cs);
    }
    const cudaError_t e3 = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = e3;
    if (e == cudaSuccess) e = W.cuda;
    for (int i = 0; i < 2; ++i) {
        if (W.copied[i]) cudaEventDestroy(W.copied[i]);
        if (formatted[i]) cudaEventDestroy(formatted[i]);
    }
    stage_release(St, cached, e == cudaSuccess);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (rc == PA_OK) rc = W.status;
    if (rc == PA_OK && bytes_out) *bytes_out = written;
    return rc;
}

namespace {

int file_sink(void *ctx, const void *data, uint64_t bytes)
{
    return std::fwrite(data, 1, bytes, (FILE *)ctx) == bytes ? 0 : 1;
}

}  // namespace
}  // namespace pa

using namespace pa;

extern "C" {

int pa_stream_edges(const pa_params *prm, const void *d_edges, int format, uint64_t chunk_edges,
                    pa_sink_fn sink, void *ctx, void *stream, uint64_t *bytes_out)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (prm->d > kTileEdges) return PA_ERR_NOT_SUPPORTED;   // a tile holds one row at least
    if (!sink || (format != PA_FORMAT_TEXT && format != PA_FORMAT_BINARY)) return PA_ERR_INVALID;
    if (!d_edges && prm->n > p.u_first) return PA_ERR_INVALID;
    return stream_edges(prm, p, d_edges, format, chunk_edges, sink, ctx, (cudaStream_t)stream,
                        bytes_out);
}

int pa_stream_trim(void)
{
    std::lock_guard<std::mutex> lk(g_stage_mu);
    if (g_stage_busy) return PA_ERR_BUSY;
    g_stage.free_all();
    g_stage = Staging();
    return PA_OK;
}

int pa_write_edges(const pa_params *prm, const void *d_edges, const char *path, int format,
                   void *stream)
{
    GenPlan p;
    int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!path || (format != PA_FORMAT_TEXT && format != PA_FORMAT_BINARY)) return PA_ERR_INVALID;
    if (!d_edges && prm->n > p.u_first) return PA_ERR_INVALID;
    FILE *f = std::fopen(path, "wb");
    if (!f) return PA_ERR_IO;
    rc = stream_edges(prm, p, d_edges, format, 0, file_sink, f, (cudaStream_t)stream, nullptr);
    if (std::fclose(f) != 0 && rc == PA_OK) rc = PA_ERR_IO;
    return rc;
}

int pa_generate_to_file(const pa_params *prm, const char *path, int format, pa_stats *stats,
                        uint64_t *bytes_out)
{
    GenPlan p;
    int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!path || (format != PA_FORMAT_TEXT && format != PA_FORMAT_BINARY)) return PA_ERR_INVALID;
    FILE *f = std::fopen(path, "wb");   // fail before generating, not after
    if (!f) return PA_ERR_IO;
    void *edges = nullptr, *scratch = nullptr;
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&edges, p.edges_bytes ? p.edges_bytes : 16);
    if (e == cudaSuccess) e = cudaMalloc(&scratch, p.scratch_bytes);
    if (e == cudaSuccess) {
        rc = launch_generate(prm, p, edges, scratch, s, 0);
        pa_stats st;
        if (rc == PA_OK) rc = pa_generate_finish(scratch, &st, s);
        if (rc == PA_OK && stats) *stats = st;
        if (rc == PA_OK) rc = stream_edges(prm, p, edges, format, 0, file_sink, f, s, bytes_out);
    }
    if (std::fclose(f) != 0 && rc == PA_OK) rc = PA_ERR_IO;
    if (edges) cudaFree(edges);
    if (scratch) cudaFree(scratch);
    if (s) cudaStreamDestroy(s);
    if (e != cudaSuccess) return set_cuda_error(e);
    return rc;
}

}  // extern "C"
