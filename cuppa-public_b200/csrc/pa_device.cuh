// pa_device.cuh -- device helpers shared by the generator kernels:
// Philox4x32-10, the seed-graph closed forms, and the memory-model primitives
// (acquire/release loads and stores at GPU scope) that publish finished tiles.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pa {

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).  The key is warp-uniform
// (the generation seed), so the compiler keeps the round keys in uniform
// registers; each round is two 32x32->64 multiplies and two 3-input XORs.
// ---------------------------------------------------------------------------
constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;

__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1)
{
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)kPhiloxM0 * c.x;
        const uint64_t p1 = (uint64_t)kPhiloxM1 * c.z;
        c = make_uint4((uint32_t)(p1 >> 32) ^ c.y ^ k0, (uint32_t)p1,
                       (uint32_t)(p0 >> 32) ^ c.w ^ k1, (uint32_t)p0);
        k0 += kPhiloxW0;
        k1 += kPhiloxW1;
    }
    return c;
}

// One draw of the copy model for slot i of node u at retry r:
//   v      = floor(x * u / 2^64), x = w1:w0     (uniform earlier node)
//   direct = w2 < pth                           (pth = floor(p * 2^32), 2^32 for p = 1)
//   k      = floor(w3 * d / 2^32)               (uniform slot of v)
struct Draw {
    uint64_t v;
    uint32_t k;
    bool direct;
};

__device__ __forceinline__ Draw draw_slot(uint64_t u, uint32_t i, uint32_t r, uint32_t key0,
                                          uint32_t key1, uint64_t pth, uint32_t d)
{
    const uint4 w = philox4x32_10(make_uint4((uint32_t)u, (uint32_t)(u >> 32), i, r), key0, key1);
    Draw out;
    out.v = __umul64hi(((uint64_t)w.y << 32) | w.x, u);
    out.k = __umulhi(w.w, d);
    out.direct = (uint64_t)w.z < pth;
    return out;
}

// One draw of the BA model (endpoint R = floor(x * 2du / 2^64), split as
// v = floor(x*u / 2^64), q = floor(2d * (x*u mod 2^64) / 2^64)):
//   direct = q odd, k = q / 2.
__device__ __forceinline__ Draw draw_slot_ba(uint64_t u, uint32_t i, uint32_t r, uint32_t key0,
                                             uint32_t key1, uint32_t d)
{
    const uint4 w = philox4x32_10(make_uint4((uint32_t)u, (uint32_t)(u >> 32), i, r), key0, key1);
    const uint64_t x = ((uint64_t)w.y << 32) | w.x;
    const uint32_t q = (uint32_t)__umul64hi(x * u, 2ull * d);
    Draw out;
    out.v = __umul64hi(x, u);
    out.k = q >> 1;
    out.direct = q & 1u;
    return out;
}

// e-th canonical seed edge (e < seed edge count): CLIQUE (1) rows v = 1..d hold
// (v, 0..v-1); STAR_REF (0) is node d -> 0..d-1.
__device__ __forceinline__ void seed_edge_of(uint64_t e, uint32_t d, uint32_t mode, uint64_t &src,
                                             uint64_t &dst)
{
    if (mode == 1) {
        // row v starts at v(v-1)/2: v = floor((1 + sqrt(1 + 8e)) / 2), with the
        // rounding of the square root corrected in integers
        uint64_t v = (uint64_t)((1.0 + sqrt(1.0 + 8.0 * (double)e)) * 0.5);
        if (v < 1) v = 1;
        while (v > 1 && v * (v - 1) / 2 > e) --v;
        while ((v + 1) * v / 2 <= e) ++v;
        src = v;
        dst = e - v * (v - 1) / 2;
    } else {
        src = d;
        dst = e;
    }
}

// Slot k of seed node v (v <= d): STAR_REF (0) or CLIQUE (1).
__device__ __forceinline__ uint64_t seed_slot(uint64_t v, uint32_t k, uint32_t d, uint32_t mode)
{
    if (mode == 1) return k < v ? (uint64_t)k : (uint64_t)k + 1;
    return v < d ? v : (uint64_t)k;
}

// ---------------------------------------------------------------------------
// Memory-model primitives (PTX ISA: ld/st .acquire/.release/.relaxed, .gpu scope)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u32(uint32_t *p, uint32_t v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void red_max_release_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("red.release.gpu.global.max.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint32_t atom_add_acq_rel_u32(uint32_t *p, uint32_t v)
{
    uint32_t old;
    asm volatile("atom.acq_rel.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ uint32_t atom_add_relaxed_u32(uint32_t *p, uint32_t v)
{
    uint32_t old;
    asm volatile("atom.relaxed.gpu.global.add.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}

__device__ __forceinline__ void red_add_relaxed_u32(uint32_t *p, uint32_t v)
{
    asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed_u32(uint32_t *p, uint32_t v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ void fence_sc_gpu() { asm volatile("fence.sc.gpu;" ::: "memory"); }
__device__ __forceinline__ void fence_acq_rel_gpu() { asm volatile("fence.acq_rel.gpu;" ::: "memory"); }

__device__ __forceinline__ uint4 ld_relaxed_v4_u32(const uint32_t *p)
{
    uint4 v;
    asm volatile("ld.relaxed.gpu.global.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p)
                 : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

// Copy-target reads: strong (L2-coherent) loads.  L1 is not coherent across SMs,
// and a line holding a finished slot may also hold a neighbour that was still
// being written when the line was cached, so these reads never use L1.
__device__ __forceinline__ uint64_t ld_slot(const int64_t *p)
{
    uint64_t v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t ld_slot(const int32_t *p)
{
    uint32_t v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t lanemask_lt()
{
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

// 128-bit / 64-bit edge stores.
__device__ __forceinline__ void st_pair(int64_t *p, uint64_t a, uint64_t b)
{
    asm volatile("st.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}

__device__ __forceinline__ void st_pair(int32_t *p, uint64_t a, uint64_t b)
{
    asm volatile("st.global.v2.u32 [%0], {%1, %2};" ::"l"(p), "r"((uint32_t)a), "r"((uint32_t)b)
                 : "memory");
}

// gpu-scope relaxed pair stores: the start kernel's readers poll the second
// field of a pair while its writer may still be running.
__device__ __forceinline__ void st_relaxed_pair(int64_t *p, uint64_t a, uint64_t b)
{
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b)
                 : "memory");
}

__device__ __forceinline__ void st_relaxed_pair(int32_t *p, uint64_t a, uint64_t b)
{
    asm volatile("st.relaxed.gpu.global.v2.u32 [%0], {%1, %2};" ::"l"(p), "r"((uint32_t)a),
                 "r"((uint32_t)b)
                 : "memory");
}

// gpu-scope relaxed store of one id (the SLOTS layout's counterpart).
__device__ __forceinline__ void st_relaxed_id(int64_t *p, uint64_t v)
{
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed_id(int32_t *p, uint64_t v)
{
    asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"((uint32_t)v) : "memory");
}

__device__ __forceinline__ void st_pair2(int32_t *p, uint64_t a, uint64_t b, uint64_t c, uint64_t d)
{
    asm volatile("st.global.v4.u32 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"((uint32_t)a),
                 "r"((uint32_t)b), "r"((uint32_t)c), "r"((uint32_t)d)
                 : "memory");
}

}  // namespace pa
