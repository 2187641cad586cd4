// pa_api.cu -- the extern "C" surface: parameter checks, sizes, generation entry
// points, the library-owned graph handle and error strings.
//
// Error convention (replacing checkCudaErrors/exit of the reference,
// src/Common/CommonHelper.cuh:148-157 and src/main.cu:38-44): every entry point
// returns a pa_status; CUDA failures are reported as PA_ERR_CUDA with the
// cudaError_t kept per thread for pa_last_cuda_error().  Nothing here prints,
// exits or resets the device.
#include <cmath>
#include <cstring>

#include "pa_internal.h"
#include "pa_wide.h"

namespace pa {

static thread_local int g_last_cuda_error = 0;

int set_cuda_error(cudaError_t e)
{
    g_last_cuda_error = (int)e;
    if (e == cudaErrorMemoryAllocation) return PA_ERR_OOM;
    return PA_ERR_CUDA;
}

static uint64_t p_threshold(double p)
{
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 1ull << 32;
    uint64_t t = (uint64_t)(p * 4294967296.0);  // exact scaling, floor
    return t > (1ull << 32) ? (1ull << 32) : t;
}

uint64_t start_split(uint64_t n, uint64_t u_first, uint64_t sb_nodes, uint64_t want)
{
    // The start kernel runs 32-bit node arithmetic: keep it well below 2^32.
    if (want > (1ull << 31)) want = 1ull << 31;
    const uint64_t avail = n > u_first ? n - u_first : 0;
    const uint64_t span = (want + sb_nodes - 1) / sb_nodes * sb_nodes;
    return u_first + (span < avail ? span : avail);
}

int make_plan(const pa_params *prm, GenPlan *plan)
{
    const int rc = pa_params_check(prm);
    if (rc != PA_OK) return rc;
    GenPlan p{};
    p.id_bytes = prm->id_bits / 8;
    p.wide = prm->d > 32;
    // d > 32: one node per warp (pa_wide.cu); the tile geometry below is unused
    p.groups = p.wide ? 1u : 32u / prm->d;
    p.passes = prm->tile_passes ? prm->tile_passes : 2u;
    p.tile_nodes = p.groups * p.passes;
    p.u_first = (uint64_t)prm->d + 1;
    const uint64_t n_gen = prm->n - p.u_first;
    p.n_tiles = p.wide ? 0 : (n_gen + p.tile_nodes - 1) / p.tile_nodes;
    p.seed_edges = pa_seed_edge_count(prm->d, prm->seed_mode);
    p.n_edges = p.seed_edges + n_gen * prm->d;
    p.pth = p_threshold(prm->p);
    p.model = prm->model;
    p.slots = prm->layout == PA_LAYOUT_SLOTS;
    p.edges_bytes = p.slots ? n_gen * prm->d * p.id_bytes : p.n_edges * 2ull * p.id_bytes;
    p.n_sb = (p.n_tiles + kSbTiles - 1) / kSbTiles;
    p.sb_offset = kCtlBytes + ((p.n_tiles * 4ull + 255ull) & ~255ull);
    p.trace_offset = p.sb_offset + ((p.n_sb * 4ull + 255ull) & ~255ull);
    p.start_offset = p.trace_offset + (uint64_t)kTraceMax * 16ull;
    p.spin_limit_ns = prm->spin_limit_ns ? prm->spin_limit_ns : 2000000000ull;
    const uint64_t want = prm->start_nodes == PA_START_NONE ? 0
                          : prm->start_nodes ? prm->start_nodes
                                             : kStartNodesAuto;
    p.u_split = p.wide ? prm->n
                       : start_split(prm->n, p.u_first, (uint64_t)kSbTiles * p.tile_nodes, want);
    const uint64_t st_nodes = (uint64_t)kStartPasses * p.groups;
    p.start_tiles = p.wide ? 0 : (p.u_split - p.u_first + st_nodes - 1) / st_nodes;
    p.scratch_bytes = p.start_offset + kStartAreaBytes;
    p.claim_tiles = prm->claim_tiles ? prm->claim_tiles : kClaimTilesAuto;
    *plan = p;
    return PA_OK;
}

}  // namespace pa

using namespace pa;

extern "C" {

int pa_abi_version(void) { return PA_ABI_VERSION; }

int pa_last_cuda_error(void) { return g_last_cuda_error; }

const char *pa_strerror(int status)
{
    switch (status) {
    case PA_OK: return "ok";
    case PA_ERR_INVALID: return "invalid argument";
    case PA_ERR_OOM: return "device out of memory";
    case PA_ERR_SPIN_TIMEOUT: return "device wait exceeded its limit";
    case PA_ERR_CUDA: return "CUDA runtime error";
    case PA_ERR_CAPACITY: return "buffer too small";
    case PA_ERR_NOT_SUPPORTED: return "not supported";
    case PA_ERR_BUSY: return "busy: admission refused";
    case PA_ERR_NOT_FOUND: return "unknown ticket";
    case PA_ERR_IO: return "file or sink error";
    default: return "unknown status";
    }
}

int pa_params_init(pa_params *out)
{
    if (!out) return PA_ERR_INVALID;
    std::memset(out, 0, sizeof(*out));
    // Reference runner defaults (src/main.cu:130-142): n1 = 1000, x1 = 4, alpha = 0.5.
    out->n = 1000;
    out->d = 4;
    out->id_bits = 32;
    out->p = 0.5;
    out->seed = 42;
    out->seed_mode = PA_SEED_CLIQUE;
    out->layout = PA_LAYOUT_PAIRS;
    return PA_OK;
}

int pa_params_check(const pa_params *prm)
{
    if (!prm) return PA_ERR_INVALID;
    if (prm->d == 0) return PA_ERR_INVALID;
    // d up to the reference's int16 EdgeIndexType (src/Common/DataTypes.h:11-28);
    // d > 32 runs the wide kernel (pa_wide.cu), whose node ids are 31-bit
    if (prm->d > gen::kWideMaxD) return PA_ERR_NOT_SUPPORTED;
    if (prm->d > 32 && prm->n > (1ull << 31)) return PA_ERR_NOT_SUPPORTED;
    if (prm->id_bits != 32 && prm->id_bits != 64) return PA_ERR_INVALID;
    if (prm->n < (uint64_t)prm->d + 1) return PA_ERR_INVALID;
    if (prm->id_bits == 32 && prm->n > 0x7fffffffull) return PA_ERR_INVALID;
    if (prm->n > (1ull << 40)) return PA_ERR_INVALID;
    if (!(prm->p >= 0.0 && prm->p <= 1.0)) return PA_ERR_INVALID;
    if (prm->seed_mode != PA_SEED_STAR_REF && prm->seed_mode != PA_SEED_CLIQUE) return PA_ERR_INVALID;
    if (prm->layout != PA_LAYOUT_PAIRS && prm->layout != PA_LAYOUT_SLOTS) return PA_ERR_NOT_SUPPORTED;
    if (prm->layout == PA_LAYOUT_SLOTS && prm->d <= 32 &&
        (prm->start_nodes != 0 || prm->n - prm->d - 1 > kStartNodesAuto))
        return PA_ERR_NOT_SUPPORTED;
    if (prm->tile_passes != 0 && prm->tile_passes != 1 && prm->tile_passes != 2 &&
        prm->tile_passes != 4 && prm->tile_passes != 8)
        return PA_ERR_INVALID;
    if (prm->threads != 0 && prm->threads != 256) return PA_ERR_NOT_SUPPORTED;
    if ((prm->flags & ~(PA_FLAG_TEST_WITHHOLD_FIRST_TILE | PA_FLAG_PREFILLED)) != 0)
        return PA_ERR_INVALID;
    if (prm->claim_tiles > 64) return PA_ERR_INVALID;
    if (prm->model != PA_MODEL_COPY && prm->model != PA_MODEL_BA) return PA_ERR_INVALID;
    if (prm->model == PA_MODEL_BA && prm->seed_mode != PA_SEED_STAR_REF) return PA_ERR_INVALID;
    return PA_OK;
}

uint64_t pa_seed_edge_count(uint32_t d, uint32_t seed_mode)
{
    return seed_mode == PA_SEED_CLIQUE ? (uint64_t)d * (d + 1) / 2 : (uint64_t)d;
}

uint64_t pa_edge_count(const pa_params *prm)
{
    GenPlan p;
    return make_plan(prm, &p) == PA_OK ? p.n_edges : 0;
}

int pa_edges_bytes(const pa_params *prm, uint64_t *bytes)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!bytes) return PA_ERR_INVALID;
    *bytes = p.edges_bytes;
    return PA_OK;
}

int pa_start_split(const pa_params *prm, uint64_t *u_split)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!u_split) return PA_ERR_INVALID;
    *u_split = p.u_split;
    return PA_OK;
}

int pa_scratch_bytes(const pa_params *prm, uint64_t *bytes)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!bytes) return PA_ERR_INVALID;
    *bytes = p.scratch_bytes;
    return PA_OK;
}

int pa_generate(const pa_params *prm, void *d_edges, uint64_t edges_bytes, void *d_scratch,
                uint64_t scratch_bytes, void *stream)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !d_scratch) return PA_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(d_edges) & 15u) || (reinterpret_cast<uintptr_t>(d_scratch) & 15u))
        return PA_ERR_INVALID;
    if (edges_bytes < p.edges_bytes || scratch_bytes < p.scratch_bytes) return PA_ERR_CAPACITY;
    return launch_generate(prm, p, d_edges, d_scratch, (cudaStream_t)stream, 0);
}

int pa_fill(const pa_params *prm, void *d_edges, uint64_t edges_bytes, void *stream)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || (reinterpret_cast<uintptr_t>(d_edges) & 15u)) return PA_ERR_INVALID;
    if (edges_bytes < p.edges_bytes) return PA_ERR_CAPACITY;
    return fill_prefill(prm, p, d_edges, (cudaStream_t)stream);
}

int pa_generate_timed(const pa_params *prm, void *d_edges, uint64_t edges_bytes, void *d_scratch,
                      uint64_t scratch_bytes, void *stream, void *const *events)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !d_scratch || !events) return PA_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(d_edges) & 15u) || (reinterpret_cast<uintptr_t>(d_scratch) & 15u))
        return PA_ERR_INVALID;
    if (edges_bytes < p.edges_bytes || scratch_bytes < p.scratch_bytes) return PA_ERR_CAPACITY;
    const cudaEvent_t ev[4] = {(cudaEvent_t)events[0], (cudaEvent_t)events[1],
                               (cudaEvent_t)events[2], (cudaEvent_t)events[3]};
    return launch_generate(prm, p, d_edges, d_scratch, (cudaStream_t)stream, 0, ev);
}

int pa_generate_finish(const void *d_scratch, pa_stats *out, void *stream)
{
    if (!d_scratch) return PA_ERR_INVALID;
    GenCtl ctl;
    cudaError_t e = cudaMemcpyAsync(&ctl, d_scratch, sizeof(ctl), cudaMemcpyDeviceToHost,
                                    (cudaStream_t)stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e != cudaSuccess) return set_cuda_error(e);
    if (out) {
        out->retries = ctl.retries;
        out->waits = ctl.waits;
        out->tiles = ctl.tiles;
        out->pending_reads = ctl.pending_reads;
        out->pending_polls = ctl.pending_polls;
        out->status = ctl.error;
        out->reserved = 0;
    }
    return (int)ctl.error;
}

int pa_generate_trace(const pa_params *prm, const void *d_scratch, uint64_t *out, uint32_t max_samples,
                      uint32_t *count, void *stream)
{
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_scratch || !count || (max_samples && !out)) return PA_ERR_INVALID;
    GenCtl ctl;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemcpyAsync(&ctl, d_scratch, sizeof(ctl), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_cuda_error(e);
    uint32_t n = ctl.trace_count < kTraceMax ? ctl.trace_count : kTraceMax;
    if (n > max_samples) n = max_samples;
    if (n) {
        e = cudaMemcpyAsync(out, (const unsigned char *)d_scratch + p.trace_offset, n * 16ull,
                            cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return set_cuda_error(e);
    }
    *count = n;
    return PA_OK;
}

int pa_graph_create(const pa_params *prm, pa_graph *g)
{
    if (!g) return PA_ERR_INVALID;
    std::memset(g, 0, sizeof(*g));
    GenPlan p;
    const int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    g->params = *prm;
    g->n_edges = p.n_edges;
    g->edges_bytes = p.edges_bytes;
    g->scratch_bytes = p.scratch_bytes;
    cudaError_t e = cudaMalloc(&g->edges, p.edges_bytes ? p.edges_bytes : 16);
    if (e == cudaSuccess) e = cudaMalloc(&g->scratch, p.scratch_bytes);
    if (e != cudaSuccess) {
        pa_graph_destroy(g);
        return set_cuda_error(e);
    }
    return PA_OK;
}

int pa_graph_generate(pa_graph *g, void *stream, pa_stats *stats)
{
    if (!g || !g->edges || !g->scratch) return PA_ERR_INVALID;
    const int rc = pa_generate(&g->params, g->edges, g->edges_bytes, g->scratch, g->scratch_bytes,
                               stream);
    if (rc != PA_OK) return rc;
    return pa_generate_finish(g->scratch, stats, stream);
}

int pa_graph_destroy(pa_graph *g)
{
    if (!g) return PA_ERR_INVALID;
    cudaError_t e1 = cudaSuccess, e2 = cudaSuccess;
    if (g->edges) e1 = cudaFree(g->edges);
    if (g->scratch) e2 = cudaFree(g->scratch);
    g->edges = nullptr;
    g->scratch = nullptr;
    if (e1 != cudaSuccess) return set_cuda_error(e1);
    if (e2 != cudaSuccess) return set_cuda_error(e2);
    return PA_OK;
}

}  // extern "C"
