// pa_generate_noalloc.cu -- generation with library-resident scratch.
//
// pa_generate() needs a scratch buffer from its caller, and pa_graph_create()
// allocates one.  Some callers can do neither: a host that hands the library a
// pre-carved output buffer from its own memory pool and forbids any further
// device allocation; a request loop on a latency-critical path, where
// cudaMalloc/cudaFree would stall it (cudaFree, in particular, synchronizes the
// device and so blocks every stream in the process); or a caller that has no
// allocator at hand at all.  For them this file keeps the scratch in a
// fixed-size __device__ array that is part of the library image, so
// pa_generate_noalloc() allocates nothing: the caller passes only the
// parameters and the edge buffer.
//
// Costs and limits, stated once:
//  * the array (PA_NOALLOC_SCRATCH_BYTES, 16 MiB) is held on every GPU that
//    loads this library, from the module load until the process exits;
//  * one generation's scratch must fit in it (about 4 bytes per tile of
//    32/d * 2 nodes, plus 35 KiB: roughly n <= 65 million nodes at d = 4 and
//    n <= 8 million at d = 32); larger requests are rejected with
//    PA_ERR_CAPACITY before any GPU work;
//  * every call on a device shares the one array.  Calls whose GPU work
//    overlaps (different streams, or different host threads) race on it and
//    produce undefined results; issue them on one stream or serialize them;
//  * the device address of the array is looked up with cudaGetSymbolAddress
//    on the first call in each CUDA context (with that context's device
//    current) and cached under the context's ID.  A context created anew --
//    after cudaDeviceReset, or after the primary context was released and
//    retained again -- has a new ID, so its first call looks the address up
//    again instead of reusing one from a context that no longer exists;
//  * each call clears the part of the array it uses before launching, so the
//    contents a previous call left behind never leak into the result.
#include <cuda.h>

#include <mutex>

#include "pa_internal.h"

namespace pa {
namespace {

static_assert(PA_NOALLOC_SCRATCH_BYTES % 256 == 0, "scratch size is a multiple of 256");

// The library-resident generation scratch (control block, tile flags,
// superblock counts and progress trace of one generation).
static __device__ __align__(256) unsigned char g_noalloc_scratch[PA_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 128;
std::mutex g_mu;
unsigned long long g_ctx_id[kMaxDevices] = {};   // context the cached address belongs to
void *g_addr[kMaxDevices] = {};

// Driver entry points for the context identity, fetched through the runtime so
// the library needs no link against libcuda.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_get_current = nullptr;
CtxGetIdFn g_ctx_get_id = nullptr;

// ID of the calling thread's current CUDA context, 0 when none is current.
// Context IDs are unique for the life of the process, unlike context handles,
// which the driver may hand out again after a context is destroyed.
int current_context_id(unsigned long long *id)
{
    *id = 0;
    if (!g_ctx_get_current || !g_ctx_get_id) {
        void *f0 = nullptr, *f1 = nullptr;
        cudaDriverEntryPointQueryResult q0, q1;
        cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0);
        if (e != cudaSuccess) return set_cuda_error(e);
        e = cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1);
        if (e != cudaSuccess) return set_cuda_error(e);
        if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return PA_ERR_NOT_SUPPORTED;
        g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(f0);
        g_ctx_get_id = reinterpret_cast<CtxGetIdFn>(f1);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_get_current(&ctx) != CUDA_SUCCESS) return PA_ERR_CUDA;
    if (!ctx) return PA_OK;
    if (g_ctx_get_id(ctx, id) != CUDA_SUCCESS) return PA_ERR_CUDA;
    return PA_OK;
}

// Device address of g_noalloc_scratch in the current context: looked up with
// cudaGetSymbolAddress on the first call in each context and cached under the
// context's ID.
int noalloc_scratch(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (dev < 0 || dev >= kMaxDevices) return PA_ERR_NOT_SUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    unsigned long long ctx = 0;
    int st = current_context_id(&ctx);
    if (st != PA_OK) return st;
    if (ctx == 0 || ctx != g_ctx_id[dev] || !g_addr[dev]) {
        void *p = nullptr;
        // The lookup makes the device's primary context current if none was.
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return set_cuda_error(e);
        st = current_context_id(&ctx);
        if (st != PA_OK) return st;
        g_ctx_id[dev] = ctx;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return PA_OK;
}

}  // namespace
}  // namespace pa

using namespace pa;

extern "C" int pa_generate_noalloc(const pa_params *prm, void *d_edges, uint64_t edges_bytes,
                                   pa_stats *stats, void *stream)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || (reinterpret_cast<uintptr_t>(d_edges) & 15u)) return PA_ERR_INVALID;
    if (edges_bytes < p.edges_bytes) return PA_ERR_CAPACITY;
    if (p.scratch_bytes > PA_NOALLOC_SCRATCH_BYTES) return PA_ERR_CAPACITY;

    void *scratch = nullptr;
    int st = noalloc_scratch(&scratch);
    if (st != PA_OK) return st;
    st = launch_generate(prm, p, d_edges, scratch, (cudaStream_t)stream, 0);
    if (st != PA_OK) return st;
    // Wait for this generation and read its status and counters back.
    return pa_generate_finish(scratch, stats, stream);
}
