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
//    on the first call on each device (with that device current) and cached.
//    Make that first call before any stream capture begins;
//  * each call clears the part of the array it uses before launching, so the
//    contents a previous call left behind never leak into the result.
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
void *g_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device (set-up on first use).
int noalloc_scratch(void **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (dev < 0 || dev >= kMaxDevices) return PA_ERR_NOT_SUPPORTED;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return set_cuda_error(e);
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
