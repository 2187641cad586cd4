// pa_post.cu -- passes over a generated edge list: row canonicalisation and
// undirected degrees (the device side of src/PA/cuPPA/cuPPA.cu:103-165, which
// copies the whole graph to the host and counts there).
#include "pa_device.cuh"
#include "pa_internal.h"
#include "pa_wide.h"

namespace pa {
namespace {

constexpr uint32_t kFull = 0xffffffffu;

// Sort each generated node's d pairs by dst.  A group of d lanes holds one row;
// lane i's rank is the number of smaller values in its group (values in a row
// are distinct), and it stores its pair at that rank.  All loads of a warp
// iteration happen before its stores, so in == out is safe.
template <typename Id>
__global__ void canon_kernel(const Id *in, Id *out, uint64_t n, uint32_t d, uint64_t seed_edges)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t G = 32u / d;
    const uint32_t g = lane / d, i = lane - g * d;
    const bool used = lane < G * d;
    const uint64_t rows = n - (d + 1);
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);

    // seed edges are already canonical
    if (in != out)
        for (uint64_t e = w0 * 32 + lane; e < seed_edges; e += warps * 32) {
            out[2 * e] = in[2 * e];
            out[2 * e + 1] = in[2 * e + 1];
        }

    for (uint64_t r0 = w0 * G; r0 < rows; r0 += warps * G) {
        const uint64_t row = r0 + g;
        const bool act = used && row < rows;
        const uint64_t e = seed_edges + row * d + i;
        Id src = 0, dst = 0;
        if (act) {
            src = in[2 * e];
            dst = in[2 * e + 1];
        }
        uint32_t rank = 0;
        for (uint32_t j = 0; j < d; ++j) {
            const Id o = __shfl_sync(kFull, dst, g * d + j);
            rank += (o < dst) ? 1u : 0u;
        }
        __syncwarp();
        if (act) {
            const uint64_t eo = seed_edges + row * d + rank;
            out[2 * eo] = src;
            out[2 * eo + 1] = dst;
        }
    }
}

// Undirected degree: +1 on both endpoints of every pair.  Equal endpoints in a
// warp are combined with __match_any_sync before the atomic (hub nodes take
// most increments when p is small).
template <typename Id>
__global__ void degree_kernel(const Id *E, uint64_t n_edges, uint64_t n, unsigned long long *deg)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t base = (uint64_t)blockIdx.x * blockDim.x; base < n_edges; base += stride) {
        const uint64_t e = base + threadIdx.x;
        unsigned long long s = e < n_edges ? (unsigned long long)E[2 * e] : ~0ull;
        unsigned long long t = e < n_edges ? (unsigned long long)E[2 * e + 1] : ~0ull;
        const bool act = s < n && t < n;   // ids are used as addresses: never trust them
        if (!act) s = t = ~0ull - lane;    // unique keys, never a leader for a real id
        const uint32_t ms = __match_any_sync(kFull, s);
        const uint32_t mt = __match_any_sync(kFull, t);
        if (act && (__ffs(ms) - 1) == (int)lane) atomicAdd(deg + s, (unsigned long long)__popc(ms));
        if (act && (__ffs(mt) - 1) == (int)lane) atomicAdd(deg + t, (unsigned long long)__popc(mt));
    }
}

// The same over a SLOTS graph: a group of d lanes takes one row (node
// u_first + row, targets S[row*d ..]); the seed edges come from their closed form.
template <typename Id>
__global__ void degree_slots_kernel(const Id *S, uint64_t rows, uint32_t d, uint64_t u_first,
                                    uint32_t seed_mode, uint64_t seed_edges, uint64_t n,
                                    unsigned long long *deg)
{
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t G = 32u / d;
    const uint32_t g = lane / d;
    const bool used = lane < G * d;
    const uint64_t warps = (uint64_t)gridDim.x * (blockDim.x >> 5);
    const uint64_t w0 = (uint64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (w0 == 0)
        for (uint64_t e = lane; e < seed_edges; e += 32) {
            uint64_t s, t;
            seed_edge_of(e, d, seed_mode, s, t);
            atomicAdd(deg + s, 1ull);
            atomicAdd(deg + t, 1ull);
        }
    for (uint64_t r0 = w0 * G; r0 < rows; r0 += warps * G) {
        const uint64_t row = r0 + g;
        const bool in = used && row < rows;
        unsigned long long t = in ? (unsigned long long)S[row * d + (lane - g * d)] : ~0ull;
        const bool act = in && t < n;       // ids are used as addresses: never trust them
        if (!act) t = ~0ull - lane;
        const uint32_t mt = __match_any_sync(kFull, t);
        if (act && (__ffs(mt) - 1) == (int)lane) atomicAdd(deg + t, (unsigned long long)__popc(mt));
        // the row's own node: d increments, from its first lane
        if (in && lane == g * d) atomicAdd(deg + u_first + row, (unsigned long long)d);
    }
}

// MurmurHash3's 64-bit finalizer (Appleby, public domain): a bijective mix.
__device__ __forceinline__ uint64_t fmix64(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xFF51AFD7ED558CCDull;
    k ^= k >> 33;
    k *= 0xC4CEB9FE1A85EC53ull;
    k ^= k >> 33;
    return k;
}

// Digest term of id x at position pos (the position is mixed in first, so two
// elements that trade places change the digest).
__device__ __forceinline__ uint64_t digest_term(uint64_t pos, uint64_t x)
{
    return fmix64(fmix64(pos * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull) ^ x);
}

// Sum and xor of the digest terms of x[0..count), positions from `base`.  A
// thread takes 16-byte vectors (two int64 or four int32 ids) with streaming
// loads when x is 16-byte aligned; a warp and then the block reduce, and one
// thread per block adds to acc (sum) and xors into acc + 1.
template <typename Id>
__global__ void __launch_bounds__(256) digest_kernel(const Id *x, uint64_t count, uint64_t base,
                                                     bool vec, unsigned long long *acc)
{
    constexpr uint32_t V = 16 / sizeof(Id);
    uint64_t sum = 0, xr = 0;
    const uint64_t tid = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t nvec = vec ? count / V : 0;
    const uint4 *xv = reinterpret_cast<const uint4 *>(x);
    for (uint64_t i = tid; i < nvec; i += stride) {
        const uint4 w = __ldcs(xv + i);
        Id vals[V];
        memcpy(vals, &w, sizeof(w));
#pragma unroll
        for (uint32_t j = 0; j < V; ++j) {
            const uint64_t h = digest_term(base + i * V + j, (uint64_t)(int64_t)vals[j]);
            sum += h;
            xr ^= h;
        }
    }
    for (uint64_t i = nvec * V + tid; i < count; i += stride) {
        const uint64_t h = digest_term(base + i, (uint64_t)(int64_t)x[i]);
        sum += h;
        xr ^= h;
    }
    for (int off = 16; off > 0; off >>= 1) {
        sum += __shfl_xor_sync(kFull, sum, off);
        xr ^= __shfl_xor_sync(kFull, xr, off);
    }
    __shared__ uint64_t ssum[8], sxr[8];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0) {
        ssum[warp] = sum;
        sxr[warp] = xr;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t w = 1; w < (blockDim.x >> 5); ++w) {
            sum += ssum[w];
            xr ^= sxr[w];
        }
        atomicAdd(acc, (unsigned long long)sum);
        atomicXor(acc + 1, (unsigned long long)xr);
    }
}

// The same for d > 32: one thread per slot (slot j of row j / d); the row's
// node gets its d increments from the thread of the row's first slot.
template <typename Id>
__global__ void degree_slots_any_kernel(const Id *S, uint64_t rows, uint32_t d, uint64_t u_first,
                                        uint32_t seed_mode, uint64_t seed_edges, uint64_t n,
                                        unsigned long long *deg)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (uint64_t e = t0; e < seed_edges; e += stride) {
        uint64_t s, t;
        seed_edge_of(e, d, seed_mode, s, t);
        atomicAdd(deg + s, 1ull);
        atomicAdd(deg + t, 1ull);
    }
    for (uint64_t j = t0; j < rows * d; j += stride) {
        const unsigned long long t = (unsigned long long)S[j];
        if (t < n) atomicAdd(deg + t, 1ull);   // ids are used as addresses: never trust them
        if (j % d == 0) atomicAdd(deg + u_first + j / d, (unsigned long long)d);
    }
}

int grid_for(uint64_t work_items, uint32_t threads)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint64_t want = (work_items + threads - 1) / threads;
    const uint64_t cap = (uint64_t)sms * 8;
    if (want > cap) want = cap;
    return (int)(want ? want : 1);
}

}  // namespace
}  // namespace pa

using namespace pa;

extern "C" {

int pa_canonicalize(const pa_params *prm, const void *d_edges, void *d_out, void *stream)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !d_out) return PA_ERR_INVALID;
    if (p.slots) return PA_ERR_NOT_SUPPORTED;
    const uint64_t rows = prm->n - p.u_first;
    const uint32_t threads = 256;
    const int grid = grid_for(rows * prm->d, threads);
    cudaStream_t s = (cudaStream_t)stream;
    if (p.wide) return gen::canon_wide(p.id_bytes, d_edges, d_out, prm->n, prm->d, p.seed_edges, s);
    if (p.id_bytes == 8)
        canon_kernel<int64_t><<<grid, threads, 0, s>>>((const int64_t *)d_edges, (int64_t *)d_out,
                                                       prm->n, prm->d, p.seed_edges);
    else
        canon_kernel<int32_t><<<grid, threads, 0, s>>>((const int32_t *)d_edges, (int32_t *)d_out,
                                                       prm->n, prm->d, p.seed_edges);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

int pa_degrees(const pa_params *prm, const void *d_edges, int64_t *d_deg, void *stream)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !d_deg) return PA_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(d_deg, 0, prm->n * sizeof(int64_t), s);
    if (e != cudaSuccess) return set_cuda_error(e);
    const uint32_t threads = 256;
    const int grid = grid_for(p.n_edges, threads);
    if (p.slots && p.wide) {
        const uint64_t rows = prm->n - p.u_first;
        if (p.id_bytes == 8)
            degree_slots_any_kernel<int64_t><<<grid, threads, 0, s>>>(
                (const int64_t *)d_edges, rows, prm->d, p.u_first, prm->seed_mode, p.seed_edges,
                prm->n, (unsigned long long *)d_deg);
        else
            degree_slots_any_kernel<int32_t><<<grid, threads, 0, s>>>(
                (const int32_t *)d_edges, rows, prm->d, p.u_first, prm->seed_mode, p.seed_edges,
                prm->n, (unsigned long long *)d_deg);
    } else if (p.slots) {
        const uint64_t rows = prm->n - p.u_first;
        if (p.id_bytes == 8)
            degree_slots_kernel<int64_t><<<grid, threads, 0, s>>>(
                (const int64_t *)d_edges, rows, prm->d, p.u_first, prm->seed_mode, p.seed_edges,
                prm->n, (unsigned long long *)d_deg);
        else
            degree_slots_kernel<int32_t><<<grid, threads, 0, s>>>(
                (const int32_t *)d_edges, rows, prm->d, p.u_first, prm->seed_mode, p.seed_edges,
                prm->n, (unsigned long long *)d_deg);
    } else if (p.n_edges) {
        if (p.id_bytes == 8)
            degree_kernel<int64_t><<<grid, threads, 0, s>>>((const int64_t *)d_edges, p.n_edges,
                                                            prm->n, (unsigned long long *)d_deg);
        else
            degree_kernel<int32_t><<<grid, threads, 0, s>>>((const int32_t *)d_edges, p.n_edges,
                                                            prm->n, (unsigned long long *)d_deg);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

int pa_digest(const void *d_ids, uint64_t count, uint32_t id_bits, uint64_t index_base,
              uint64_t *d_acc, void *stream)
{
    if (!d_acc || (id_bits != 32 && id_bits != 64) || (count && !d_ids)) return PA_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(d_acc) & 7u) return PA_ERR_INVALID;
    if (!count) return PA_OK;
    const uint32_t threads = 256;
    const bool vec = (reinterpret_cast<uintptr_t>(d_ids) & 15u) == 0;
    // Up to eight blocks of 256 threads per SM (grid_for): enough 16-byte loads
    // in flight to stream at HBM speed; the grid never exceeds the work.
    const int grid = grid_for(count / (vec ? 16u / (id_bits / 8u) : 1u) + 1, threads);
    cudaStream_t s = (cudaStream_t)stream;
    if (id_bits == 64)
        digest_kernel<int64_t><<<grid, threads, 0, s>>>((const int64_t *)d_ids, count, index_base,
                                                        vec, (unsigned long long *)d_acc);
    else
        digest_kernel<int32_t><<<grid, threads, 0, s>>>((const int32_t *)d_ids, count, index_base,
                                                        vec, (unsigned long long *)d_acc);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

}  // extern "C"
