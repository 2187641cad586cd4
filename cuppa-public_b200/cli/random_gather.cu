// random_gather -- rate and DRAM cost of random 8-byte global loads on this GPU.
//
// The generator's copy reads are 8-byte loads of slots at uniformly random
// positions of a buffer far larger than L2.  This probe measures what the
// hardware gives that access pattern, for several load flavours: the rate of
// random reads over a buffer of the given size (default 64 GB), and the rate of
// the coalesced 16-byte store stream the generator's edge writes use.
//
//   random_gather [buffer-GB]
//
// The DRAM bytes moved per random read are read with ncu's dram__bytes_read.sum
// on this binary (see the profile summary that cites it).
#include <cstdint>
#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

__device__ __forceinline__ uint64_t mix(uint64_t x)
{
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdULL;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ULL;
    x ^= x >> 33;
    return x;
}

template <int V>
__device__ __forceinline__ uint64_t ld(const uint64_t *p)
{
    uint64_t v;
    if (V == 0) v = *p;
    else if (V == 1) v = __ldg(p);
    else if (V == 2) asm volatile("ld.relaxed.gpu.global.u64 %0,[%1];" : "=l"(v) : "l"(p));
    else if (V == 3) v = __ldcg(p);
    else if (V == 4) asm volatile("ld.global.L2::64B.u64 %0,[%1];" : "=l"(v) : "l"(p));
    else asm volatile("ld.global.nc.L1::no_allocate.u64 %0,[%1];" : "=l"(v) : "l"(p));
    return v;
}

template <int V, int ILP>
__global__ void gather(const uint64_t *buf, uint64_t n, uint64_t reads, uint64_t *out)
{
    uint64_t acc = 0;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid * ILP; i < reads; i += T * ILP) {
        uint64_t v[ILP];
#pragma unroll
        for (int j = 0; j < ILP; j++) v[j] = ld<V>(buf + mix(i + j) % n);
#pragma unroll
        for (int j = 0; j < ILP; j++) acc += v[j];
    }
    if (acc == 0x1234567) out[0] = acc;
}

__global__ void fill(uint64_t *buf, uint64_t n)
{
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += T) buf[i] = i;
}

__global__ void stream_store(uint4 *buf, uint64_t n16)
{
    const uint64_t T = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n16; i += T)
        buf[i] = make_uint4((uint32_t)i, 0, (uint32_t)i, 0);
}

template <int V, int ILP>
float run(const uint64_t *buf, uint64_t n, uint64_t reads, uint64_t *out, int sms)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    gather<V, ILP><<<sms * 8, 256>>>(buf, n, reads, out);
    cudaDeviceSynchronize();
    cudaEventRecord(a);
    gather<V, ILP><<<sms * 8, 256>>>(buf, n, reads, out);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms;
    cudaEventElapsedTime(&ms, a, b);
    return ms;
}

int main(int argc, char **argv)
{
    const double gb = argc > 1 ? std::atof(argv[1]) : 64.0;
    const uint64_t n = (uint64_t)(gb * 1e9 / 8);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    uint64_t *buf, *out;
    if (cudaMalloc(&buf, n * 8) != cudaSuccess || cudaMalloc(&out, 8) != cudaSuccess) {
        std::printf("allocation of %.1f GB failed\n", gb);
        return 1;
    }
    fill<<<sms * 8, 256>>>(buf, n);
    cudaDeviceSynchronize();
    const uint64_t reads = 1ull << 30;
    const char *names[] = {"weak", "ldg.nc", "relaxed.gpu", "cg", "L2::64B", "nc.no_allocate"};
    float t[6];
    t[0] = run<0, 4>(buf, n, reads, out, sms);
    t[1] = run<1, 4>(buf, n, reads, out, sms);
    t[2] = run<2, 4>(buf, n, reads, out, sms);
    t[3] = run<3, 4>(buf, n, reads, out, sms);
    t[4] = run<4, 4>(buf, n, reads, out, sms);
    t[5] = run<5, 4>(buf, n, reads, out, sms);
    for (int i = 0; i < 6; i++)
        std::printf("buffer %.1f GB  random 8-byte loads (%s): %.2f ms, %.2f G reads/s\n", gb, names[i],
                    t[i], reads / t[i] / 1e6);
    const uint64_t n16 = n * 8 / 16;
    stream_store<<<sms * 8, 256>>>((uint4 *)buf, n16);
    cudaDeviceSynchronize();
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a);
    stream_store<<<sms * 8, 256>>>((uint4 *)buf, n16);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms;
    cudaEventElapsedTime(&ms, a, b);
    std::printf("buffer %.1f GB  coalesced 16-byte stores: %.2f ms, %.1f GB/s\n", gb, ms, n * 8 / ms / 1e6);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : 1;
}
