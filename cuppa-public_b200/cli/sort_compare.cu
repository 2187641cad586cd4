// sort_compare -- measurement probe, not part of the library: times the CSR
// build of one generated graph (pa_build_csr) and, on the same graph, CUB's
// DeviceRadixSort::SortKeys of the (destination << 32 | source) items the CSR
// build sorts, over the same key bits.  It shows how the build's own sort
// compares with a library radix sort on this part.
//
//   sort_compare n d p [id_bits=64] [reps=4]
//
// Prints one line per repetition and a summary line of minima.
#include <cub/device/device_radix_sort.cuh>

#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include "cuppa_pa.h"

#define CK(x)                                                                              \
    do {                                                                                   \
        cudaError_t e_ = (x);                                                              \
        if (e_ != cudaSuccess) {                                                           \
            fprintf(stderr, "%s:%d %s\n", __FILE__, __LINE__, cudaGetErrorString(e_));     \
            return 1;                                                                      \
        }                                                                                  \
    } while (0)
#define PK(x)                                                                              \
    do {                                                                                   \
        int r_ = (x);                                                                      \
        if (r_ != PA_OK) {                                                                 \
            fprintf(stderr, "%s:%d %s\n", __FILE__, __LINE__, pa_strerror(r_));            \
            return 1;                                                                      \
        }                                                                                  \
    } while (0)

template <typename Id>
__global__ void make_items(const Id *E, uint64_t m, unsigned long long *items)
{
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += stride)
        items[i] = ((unsigned long long)(uint64_t)E[2 * i + 1] << 32) | (uint64_t)E[2 * i];
}

static int run(uint64_t n, uint32_t d, double p, uint32_t id_bits, int reps)
{
    pa_params prm;
    PK(pa_params_init(&prm));
    prm.n = n;
    prm.d = d;
    prm.p = p;
    prm.seed = 7;
    prm.id_bits = id_bits;
    prm.seed_mode = PA_SEED_CLIQUE;
    uint64_t eb = 0, sb = 0;
    PK(pa_edges_bytes(&prm, &eb));
    PK(pa_scratch_bytes(&prm, &sb));
    const uint64_t m = pa_edge_count(&prm);
    void *E = nullptr, *S = nullptr;
    CK(cudaMalloc(&E, eb));
    CK(cudaMalloc(&S, sb));
    PK(pa_generate(&prm, E, eb, S, sb, nullptr));
    CK(cudaDeviceSynchronize());
    CK(cudaFree(S));

    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // the CSR build
    uint64_t rb = 0, cb = 0, csb = 0;
    PK(pa_csr_bytes(&prm, &rb, &cb, &csb));
    void *R = nullptr, *C = nullptr, *CS = nullptr;
    CK(cudaMalloc(&R, rb));
    CK(cudaMalloc(&C, cb));
    CK(cudaMalloc(&CS, csb));
    float best_csr = 1e30f;
    for (int r = 0; r <= reps; ++r) {
        CK(cudaEventRecord(e0));
        PK(pa_build_csr(&prm, E, (int64_t *)R, C, CS, csb, nullptr));
        CK(cudaEventRecord(e1));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (r > 0 && ms < best_csr) best_csr = ms;
        printf("pa_build_csr rep %d: %.2f ms\n", r, ms);
    }
    CK(cudaFree(R));
    CK(cudaFree(C));
    CK(cudaFree(CS));

    // CUB on the same items and key bits (keys < n need bits(n) bits, as in
    // the CSR build)
    int bits = 1;
    while (bits < 32 && (n >> bits) != 0) ++bits;
    unsigned long long *A = nullptr, *B = nullptr;
    CK(cudaMalloc(&A, 8 * m));
    CK(cudaMalloc(&B, 8 * m));
    cub::DoubleBuffer<unsigned long long> db(A, B);
    void *tmp = nullptr;
    size_t tb = 0;
    CK(cub::DeviceRadixSort::SortKeys(tmp, tb, db, (int64_t)m, 32, 32 + bits));
    CK(cudaMalloc(&tmp, tb));
    float best_cub = 1e30f;
    for (int r = 0; r <= reps; ++r) {
        if (id_bits == 64)
            make_items<int64_t><<<148 * 8, 512>>>((const int64_t *)E, m, db.Current());
        else
            make_items<int32_t><<<148 * 8, 512>>>((const int32_t *)E, m, db.Current());
        CK(cudaGetLastError());
        CK(cudaEventRecord(e0));
        CK(cub::DeviceRadixSort::SortKeys(tmp, tb, db, (int64_t)m, 32, 32 + bits));
        CK(cudaEventRecord(e1));
        CK(cudaEventSynchronize(e1));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, e0, e1));
        if (r > 0 && ms < best_cub) best_cub = ms;
        printf("cub SortKeys rep %d: %.2f ms\n", r, ms);
    }
    printf("n=%llu d=%u p=%g id_bits=%u items=%llu key_bits=%d: pa_build_csr %.2f ms (whole "
           "CSR), cub SortKeys %.2f ms (sort only)\n",
           (unsigned long long)n, d, p, id_bits, (unsigned long long)m, bits, best_csr, best_cub);
    CK(cudaFree(tmp));
    CK(cudaFree(A));
    CK(cudaFree(B));
    CK(cudaFree(E));
    return 0;
}

int main(int argc, char **argv)
{
    if (argc < 4) {
        fprintf(stderr, "usage: %s n d p [id_bits=64] [reps=4]\n", argv[0]);
        return 2;
    }
    const uint64_t n = strtoull(argv[1], nullptr, 0);
    const uint32_t d = (uint32_t)atoi(argv[2]);
    const double p = atof(argv[3]);
    const uint32_t id_bits = argc > 4 ? (uint32_t)atoi(argv[4]) : 64u;
    const int reps = argc > 5 ? atoi(argv[5]) : 4;
    return run(n, d, p, id_bits, reps);
}
