// pa_plan.cu -- a generation captured once into a CUDA graph and replayed.
//
// A small graph (10^4..10^5 nodes) takes tens of microseconds on the GPU, the
// same order as issuing its scratch clear, sentinel fill and kernel launch one
// by one.  A plan records that sequence for fixed parameters and buffers with
// stream capture and replays it with one cudaGraphLaunch.  The replay writes
// exactly what pa_generate writes (the captured work is pa_generate's).
#include <new>

#include "pa_internal.h"

struct pa_plan {
    pa_params prm;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    void *scratch = nullptr;
};

using namespace pa;

extern "C" {

int pa_plan_create(const pa_params *prm, void *d_edges, uint64_t edges_bytes, void *d_scratch,
                   uint64_t scratch_bytes, pa_plan **out)
{
    if (!out) return PA_ERR_INVALID;
    *out = nullptr;
    GenPlan p;
    int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (!d_edges || !d_scratch) return PA_ERR_INVALID;
    if ((reinterpret_cast<uintptr_t>(d_edges) & 15u) || (reinterpret_cast<uintptr_t>(d_scratch) & 15u))
        return PA_ERR_INVALID;
    if (edges_bytes < p.edges_bytes || scratch_bytes < p.scratch_bytes) return PA_ERR_CAPACITY;
    pa_plan *P = new (std::nothrow) pa_plan();
    if (!P) return PA_ERR_OOM;
    P->prm = *prm;
    P->scratch = d_scratch;
    cudaStream_t s = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        rc = launch_generate(prm, p, d_edges, d_scratch, s, 0);
        const cudaError_t e2 = cudaStreamEndCapture(s, &P->graph);
        if (rc == PA_OK && e2 != cudaSuccess) e = e2;
    }
    if (e == cudaSuccess && rc == PA_OK) e = cudaGraphInstantiate(&P->exec, P->graph, 0);
    if (s) cudaStreamDestroy(s);
    if (e != cudaSuccess || rc != PA_OK) {
        if (P->exec) cudaGraphExecDestroy(P->exec);
        if (P->graph) cudaGraphDestroy(P->graph);
        delete P;
        return rc != PA_OK ? rc : set_cuda_error(e);
    }
    *out = P;
    return PA_OK;
}

int pa_plan_launch(pa_plan *P, void *stream)
{
    if (!P) return PA_ERR_INVALID;
    const cudaError_t e = cudaGraphLaunch(P->exec, (cudaStream_t)stream);
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

int pa_plan_destroy(pa_plan *P)
{
    if (!P) return PA_ERR_INVALID;
    if (P->exec) cudaGraphExecDestroy(P->exec);
    if (P->graph) cudaGraphDestroy(P->graph);
    delete P;
    return PA_OK;
}

}  // extern "C"
