// pa_io.cu -- file outputs of a generated graph.
//
//  * pa_write_edges: the edge list as text, one "u v" line per edge -- the format
//    of PAHelper::writeGraphToDisk (src/PA/SPA/PAHelper.hpp:163-177) -- or as raw
//    little-endian id pairs.  The device buffer is streamed to the file through
//    two pinned staging buffers, so copy and formatting overlap.  With the
//    reference's seed graph (PA_SEED_STAR_REF) the PAIRS order is exactly the
//    reference's row order: node M's star row, then rows M+1..N-1 in slot order.
//  * pa_write_degree_distribution: the "Degree,Count" CSV of
//    cuPPA::printDegreeDistribution (src/PA/cuPPA/cuPPA.cu:103-165), degree-0
//    nodes omitted as there.  Degrees and their histogram are computed on the
//    device: per-CTA shared-memory bins for degrees below 4096, global bins up to
//    2^20, and a list for the (few) nodes above; only the histogram crosses to
//    the host, not the graph.
#include <algorithm>
#include <cstdio>
#include <map>
#include <vector>

#include "pa_internal.h"

namespace pa {
namespace {

constexpr uint32_t kSmemBins = 4096;
constexpr uint64_t kGlobalBins = 1ull << 20;

__global__ void degree_hist_kernel(const int64_t *deg, uint64_t n, unsigned long long *hist,
                                   unsigned long long *big, unsigned long long *big_count,
                                   uint64_t big_cap)
{
    __shared__ unsigned int s_bins[kSmemBins];
    for (uint32_t i = threadIdx.x; i < kSmemBins; i += blockDim.x) s_bins[i] = 0;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t x = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += stride) {
        const int64_t k = deg[x];
        if (k <= 0) continue;
        if ((uint64_t)k < kSmemBins) {
            atomicAdd(&s_bins[k], 1u);
        } else if ((uint64_t)k < kGlobalBins) {
            atomicAdd(hist + k, 1ull);
        } else {
            const unsigned long long slot = atomicAdd(big_count, 1ull);
            if (slot < big_cap) big[slot] = (unsigned long long)k;
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kSmemBins; i += blockDim.x)
        if (s_bins[i]) atomicAdd(hist + i, (unsigned long long)s_bins[i]);
}

int grid_for(uint64_t items)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (items + 255) / 256;
    return (int)std::max<uint64_t>(1, std::min<uint64_t>(want, (uint64_t)sms * 4));
}

// Decimal digits of v into p (no terminator); returns the end.
inline char *put_u64(char *p, uint64_t v)
{
    char tmp[24];
    int k = 0;
    do {
        tmp[k++] = (char)('0' + v % 10);
        v /= 10;
    } while (v);
    while (k) *p++ = tmp[--k];
    return p;
}

}  // namespace
}  // namespace pa

using namespace pa;

extern "C" {

int pa_write_edges(const pa_params *prm, const void *d_edges, const char *path, int format,
                   void *stream)
{
    GenPlan p;
    int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !path || (format != PA_FORMAT_TEXT && format != PA_FORMAT_BINARY))
        return PA_ERR_INVALID;
    FILE *f = std::fopen(path, "wb");
    if (!f) return PA_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t pair_bytes = 2ull * p.id_bytes;
    const uint64_t chunk_pairs = 1ull << 22;   // 4M pairs per staging buffer
    void *stage[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        e = cudaMallocHost(&stage[i], chunk_pairs * pair_bytes);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming);
    }
    std::vector<char> text;
    if (format == PA_FORMAT_TEXT) text.resize(chunk_pairs * 42);
    const uint64_t total = p.n_edges;
    const uint64_t chunks = (total + chunk_pairs - 1) / chunk_pairs;
    auto issue = [&](uint64_t c) {
        const uint64_t first = c * chunk_pairs;
        const uint64_t cnt = std::min(chunk_pairs, total - first);
        cudaError_t ee = cudaMemcpyAsync(stage[c & 1],
                                         (const unsigned char *)d_edges + first * pair_bytes,
                                         cnt * pair_bytes, cudaMemcpyDeviceToHost, s);
        if (ee == cudaSuccess) ee = cudaEventRecord(done[c & 1], s);
        return ee;
    };
    if (e == cudaSuccess && chunks) e = issue(0);
    for (uint64_t c = 0; c < chunks && e == cudaSuccess; ++c) {
        if (c + 1 < chunks) e = issue(c + 1);
        if (e == cudaSuccess) e = cudaEventSynchronize(done[c & 1]);
        if (e != cudaSuccess) break;
        const uint64_t first = c * chunk_pairs;
        const uint64_t cnt = std::min(chunk_pairs, total - first);
        size_t wrote, want;
        if (format == PA_FORMAT_BINARY) {
            want = cnt * pair_bytes;
            wrote = std::fwrite(stage[c & 1], 1, want, f);
        } else {
            char *q = text.data();
            for (uint64_t i = 0; i < cnt; ++i) {
                uint64_t u, v;
                if (p.id_bytes == 8) {
                    const int64_t *pp = (const int64_t *)stage[c & 1] + 2 * i;
                    u = (uint64_t)pp[0];
                    v = (uint64_t)pp[1];
                } else {
                    const int32_t *pp = (const int32_t *)stage[c & 1] + 2 * i;
                    u = (uint32_t)pp[0];
                    v = (uint32_t)pp[1];
                }
                q = put_u64(q, u);
                *q++ = ' ';
                q = put_u64(q, v);
                *q++ = '\n';
            }
            want = (size_t)(q - text.data());
            wrote = std::fwrite(text.data(), 1, want, f);
        }
        if (wrote != want) {
            rc = PA_ERR_INVALID;
            break;
        }
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    for (int i = 0; i < 2; ++i) {
        if (done[i]) cudaEventDestroy(done[i]);
        if (stage[i]) cudaFreeHost(stage[i]);
    }
    if (std::fclose(f) != 0 && rc == PA_OK) rc = PA_ERR_INVALID;
    if (e != cudaSuccess) return set_cuda_error(e);
    return rc;
}

int pa_write_degree_distribution(const pa_params *prm, const void *d_edges, const char *path,
                                 void *stream)
{
    GenPlan p;
    int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !path) return PA_ERR_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const uint64_t n = prm->n;
    const uint64_t big_cap = 2 * p.n_edges / kGlobalBins + 1024;   // nodes of degree >= 2^20
    int64_t *deg = nullptr;
    unsigned long long *hist = nullptr;   // kGlobalBins bins, then big_count, then the big list
    cudaError_t e = cudaMallocAsync(&deg, n * sizeof(int64_t), s);
    if (e == cudaSuccess)
        e = cudaMallocAsync(&hist, (kGlobalBins + 1 + big_cap) * sizeof(unsigned long long), s);
    if (e == cudaSuccess)
        e = cudaMemsetAsync(hist, 0, (kGlobalBins + 1) * sizeof(unsigned long long), s);
    if (e == cudaSuccess) {
        rc = pa_degrees(prm, d_edges, deg, stream);
        if (rc == PA_OK) {
            degree_hist_kernel<<<grid_for(n), 256, 0, s>>>(deg, n, hist, hist + kGlobalBins + 1,
                                                            hist + kGlobalBins, big_cap);
            e = cudaGetLastError();
        }
    }
    std::vector<unsigned long long> h(kGlobalBins + 1);
    std::vector<unsigned long long> big;
    if (e == cudaSuccess && rc == PA_OK) {
        e = cudaMemcpyAsync(h.data(), hist, h.size() * sizeof(unsigned long long),
                            cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        const uint64_t nb = std::min<uint64_t>(h[kGlobalBins], big_cap);
        if (e == cudaSuccess && h[kGlobalBins] > big_cap) rc = PA_ERR_CAPACITY;
        if (e == cudaSuccess && nb) {
            big.resize(nb);
            e = cudaMemcpyAsync(big.data(), hist + kGlobalBins + 1, nb * sizeof(unsigned long long),
                                cudaMemcpyDeviceToHost, s);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        }
    }
    if (deg) cudaFreeAsync(deg, s);
    if (hist) cudaFreeAsync(hist, s);
    cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (rc != PA_OK) return rc;
    std::map<uint64_t, uint64_t> hub;
    for (unsigned long long k : big) ++hub[k];
    FILE *f = std::fopen(path, "wb");
    if (!f) return PA_ERR_INVALID;
    std::fprintf(f, "Degree,Count\n");
    for (uint64_t k = 1; k < kGlobalBins; ++k)
        if (h[k]) std::fprintf(f, "%llu,%llu\n", (unsigned long long)k, (unsigned long long)h[k]);
    for (const auto &kv : hub)
        std::fprintf(f, "%llu,%llu\n", (unsigned long long)kv.first, (unsigned long long)kv.second);
    return std::fclose(f) == 0 ? PA_OK : PA_ERR_INVALID;
}

}  // extern "C"
