// pa_io.cu -- file outputs of a generated graph.
//
//  (pa_write_edges, the edge-list writer, is in pa_stream.cu.)
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

}  // namespace
}  // namespace pa

using namespace pa;

extern "C" {

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
    if (!f) return PA_ERR_IO;
    std::fprintf(f, "Degree,Count\n");
    for (uint64_t k = 1; k < kGlobalBins; ++k)
        if (h[k]) std::fprintf(f, "%llu,%llu\n", (unsigned long long)k, (unsigned long long)h[k]);
    for (const auto &kv : hub)
        std::fprintf(f, "%llu,%llu\n", (unsigned long long)kv.first, (unsigned long long)kv.second);
    return std::fclose(f) == 0 ? PA_OK : PA_ERR_IO;
}

}  // extern "C"
