// pa_server.cu -- the request server: continuous batching of generation
// requests under a device-memory budget.
//
// One control thread per server owns a non-blocking CUDA stream and a CUDA
// memory pool on the server's device.  Client threads only touch host state
// (under the server mutex): submit queues a request with the admission queue
// (pa_sched.cpp), poll/wait read its state, release hands its buffer back.
// The control thread loops:
//   1. completions: batches finish in stream order; for each whose event has
//      fired, read the device status it copied back, mark its requests done and
//      return their generation scratch to the budget;
//   2. frees: buffers of released (or TTL-expired) results are freed on the
//      stream and their budget returned;
//   3. admission: while fewer than max_inflight batches are on the GPU, admit
//      what fits the budget and launch it as one batch per id width (the
//      fill / start / tail launches of pa_batch.cu) -- requests that arrived
//      while the previous batch ran make up the next, and consecutive batches'
//      launches follow each other on the stream without a host round trip;
//   4. sleep briefly (20 us with work in flight, else until woken).
// Memory per request: its edge buffer plus the generation scratch of its own
// plan, which bounds its share of the batch scratch; with CSR outputs also its
// rowptr, col and CSR scratch.  The CSR of every request of a batch is queued
// on the stream right after the batch; the CSR scratch (and the edge buffer,
// when pairs are not kept) is freed in stream order behind it and its budget
// returned when the batch completes.  Requests too large for the batch
// kernels' 32-bit node arithmetic run as single generations.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstddef>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

#include "pa_batch.h"

namespace pa {
namespace {

enum ReqState { RQ_QUEUED, RQ_RUNNING, RQ_DONE };

struct Request {
    pa_params prm{};
    uint64_t n_edges = 0, edges_bytes = 0, scratch_reserve = 0;
    uint64_t rowptr_bytes = 0, col_bytes = 0, csr_scratch = 0;   // 0 without CSR outputs
    void *edges = nullptr;
    int64_t *rowptr = nullptr;
    void *col = nullptr;
    int32_t status = PA_OK;
    uint32_t batch_size = 0;
    uint64_t t_submit = 0, t_start = 0, t_done = 0;
    ReqState state = RQ_QUEUED;
    bool batchable = true;
};

struct Pinned {
    unsigned char *p = nullptr;
    uint64_t cap = 0;
};

struct Launch {
    std::vector<uint64_t> tickets;
    void *scratch = nullptr;
    Pinned buf;            // image; then the generation status word at status_off and
    uint64_t status_off = 0;   // one CSR status word per request after it
    cudaEvent_t done = nullptr;
};

uint64_t scratch_reserve(const pa_params &prm, bool batchable)
{
    pa_params q = prm;
    if (batchable) q.tile_passes = 1;   // the batch launches' tile shape
    GenPlan p;
    return make_plan(&q, &p) == PA_OK ? p.scratch_bytes : 0;
}

}  // namespace
}  // namespace pa

using namespace pa;

struct pa_server {
    pa_server_config cfg{};
    int device = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    pa_sched *sched = nullptr;
    std::unordered_map<uint64_t, Request> reqs;
    // work for the control thread: free the buffer (if any), then return the
    // ticket's whole budget (if the ticket is not 0)
    std::vector<std::pair<uint64_t, void *>> to_free;
    std::deque<std::pair<uint64_t, uint64_t>> done_order;  // t_done, ticket (TTL)
    uint64_t next_ticket = 1;
    std::chrono::steady_clock::time_point t0;
    pa_server_stats st{};
    // control thread only
    cudaStream_t stream = nullptr;
    cudaMemPool_t pool = nullptr;
    std::deque<Launch> inflight;
    std::vector<Pinned> pinned_free;

    uint64_t now() const
    {
        return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                   std::chrono::steady_clock::now() - t0)
            .count();
    }
};

namespace {

Pinned get_pinned(pa_server *S, uint64_t bytes)
{
    for (size_t i = 0; i < S->pinned_free.size(); ++i)
        if (S->pinned_free[i].cap >= bytes) {
            Pinned b = S->pinned_free[i];
            S->pinned_free.erase(S->pinned_free.begin() + (ptrdiff_t)i);
            return b;
        }
    Pinned b;
    b.cap = std::max<uint64_t>(bytes, 1ull << 20);
    if (cudaMallocHost(&b.p, b.cap) != cudaSuccess) b = Pinned{};
    return b;
}

// Queue a request's buffers for freeing and its budget for return (lock held).
void drop_buffers(pa_server *S, uint64_t tk, Request &r)
{
    for (void *b : {r.edges, (void *)r.rowptr, r.col})
        if (b) S->to_free.emplace_back(0, b);
    S->to_free.emplace_back(tk, nullptr);
    r.edges = nullptr;
    r.rowptr = nullptr;
    r.col = nullptr;
}

// Mark tickets done with `status` (lock held).  Failed requests give all their
// memory back at once; finished ones give back their scratch share.
void complete(pa_server *S, const std::vector<uint64_t> &tickets, int status, uint32_t batch_size,
              const uint32_t *csr_status = nullptr)
{
    const uint64_t t = S->now();
    const bool keep_pairs = (S->cfg.outputs & PA_OUT_PAIRS) != 0;
    for (size_t q = 0; q < tickets.size(); ++q) {
        const uint64_t tk = tickets[q];
        auto it = S->reqs.find(tk);
        if (it == S->reqs.end()) continue;
        Request &r = it->second;
        int st = status;
        if (st == PA_OK && csr_status) st = (int)csr_status[q];
        r.state = RQ_DONE;
        r.status = st;
        r.batch_size = batch_size;
        r.t_done = t;
        if (st == PA_OK) {
            ++S->st.completed;
            S->st.edges_done += r.n_edges;
            // the generation and CSR scratch, and the pairs when not kept, are
            // already freed on the stream
            uint64_t give = r.scratch_reserve + r.csr_scratch;
            if (r.col_bytes && !keep_pairs) give += r.edges_bytes;
            pa_sched_release(S->sched, tk, give);
        } else {
            ++S->st.failed;
            drop_buffers(S, tk, r);
        }
        S->done_order.emplace_back(t, tk);
    }
    S->cv_done.notify_all();
}

// What the control thread needs of an admitted request (copied under the lock).
struct Job {
    uint64_t ticket;
    pa_params prm;
    uint64_t edges_bytes, rowptr_bytes, col_bytes, csr_scratch;
};

// A pool allocation; when the pool's free blocks are too fragmented, its unused
// memory goes back to the device (after the stream drains) and the allocation
// is tried once more.  The budget bounds what is held, not the fragmentation.
cudaError_t pool_alloc(pa_server *S, void **p, uint64_t bytes)
{
    cudaError_t e = cudaMallocFromPoolAsync(p, std::max<uint64_t>(bytes, 16), S->pool, S->stream);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        cudaStreamSynchronize(S->stream);
        cudaMemPoolTrimTo(S->pool, 0);
        e = cudaMallocFromPoolAsync(p, std::max<uint64_t>(bytes, 16), S->pool, S->stream);
    }
    return e;
}

// Launch one group of admitted requests (same id width, all batchable) as a
// batch, or one request alone; then, with CSR outputs, every request's CSR.
// Called without the lock.
void launch_group(pa_server *S, const std::vector<Job> &jobs, bool batch)
{
    const uint32_t k = (uint32_t)jobs.size();
    const bool csr = (S->cfg.outputs & PA_OUT_CSR) != 0;
    const bool keep_pairs = (S->cfg.outputs & PA_OUT_PAIRS) != 0;
    std::vector<void *> edges(k, nullptr), rowptr(k, nullptr), col(k, nullptr), cscr(k, nullptr);
    std::vector<pa_params> prms(k);
    std::vector<uint64_t> ebytes(k);
    Launch L;
    for (uint32_t i = 0; i < k; ++i) {
        L.tickets.push_back(jobs[i].ticket);
        prms[i] = jobs[i].prm;
        ebytes[i] = jobs[i].edges_bytes;
    }
    int rc = PA_OK;
    cudaError_t e = cudaSuccess;
    for (uint32_t i = 0; i < k && e == cudaSuccess; ++i) {
        e = pool_alloc(S, &edges[i], ebytes[i]);
        if (csr && e == cudaSuccess) e = pool_alloc(S, &rowptr[i], jobs[i].rowptr_bytes);
        if (csr && e == cudaSuccess) e = pool_alloc(S, &col[i], jobs[i].col_bytes);
    }
    if (e != cudaSuccess) rc = set_cuda_error(e);
    BatchJob J;
    uint64_t scratch_bytes = 0, image_bytes = 0;
    if (rc == PA_OK) {
        if (batch) {
            rc = batch_prepare(prms.data(), k, J);
            scratch_bytes = J.scratch_bytes;
            image_bytes = J.image_bytes;
        } else {
            rc = pa_scratch_bytes(&prms[0], &scratch_bytes);
        }
    }
    if (rc == PA_OK) {
        e = pool_alloc(S, &L.scratch, scratch_bytes);
        if (e != cudaSuccess) rc = set_cuda_error(e);
    }
    if (rc == PA_OK) {
        L.status_off = (image_bytes + 15) & ~15ull;
        L.buf = get_pinned(S, L.status_off + 4ull * (k + 1));
        if (!L.buf.p) rc = PA_ERR_OOM;
    }
    if (rc == PA_OK && batch) {
        rc = batch_bind(J, prms.data(), edges.data(), ebytes.data(), L.scratch, L.buf.p);
        if (rc == PA_OK) rc = batch_enqueue(J, L.scratch, L.buf.p, S->stream);
    } else if (rc == PA_OK) {
        rc = pa_generate(&prms[0], edges[0], ebytes[0], L.scratch, scratch_bytes, S->stream);
    }
    if (rc == PA_OK) {
        e = cudaMemcpyAsync(L.buf.p + L.status_off,
                            (const unsigned char *)L.scratch + offsetof(GenCtl, error),
                            sizeof(uint32_t), cudaMemcpyDeviceToHost, S->stream);
        if (e != cudaSuccess) rc = set_cuda_error(e);
    }
    // CSR of every request, in the same stream; its scratch (and the pairs when
    // they are not kept) is freed in stream order behind it
    uint32_t *csr_status = reinterpret_cast<uint32_t *>(L.buf.p + L.status_off) + 1;
    for (uint32_t i = 0; i < k && rc == PA_OK; ++i) {
        if (!csr) {
            csr_status[i] = PA_OK;
            continue;
        }
        e = pool_alloc(S, &cscr[i], jobs[i].csr_scratch);
        if (e != cudaSuccess) {
            rc = set_cuda_error(e);
            break;
        }
        uint64_t err_off = 0;
        rc = csr_enqueue(&prms[i], edges[i], (int64_t *)rowptr[i], col[i], cscr[i], jobs[i].csr_scratch,
                         S->stream, &err_off);
        if (rc != PA_OK) break;
        e = cudaMemcpyAsync(csr_status + i, (const unsigned char *)cscr[i] + err_off, 4,
                            cudaMemcpyDeviceToHost, S->stream);
        if (e == cudaSuccess) e = cudaFreeAsync(cscr[i], S->stream);
        cscr[i] = nullptr;
        if (e == cudaSuccess && !keep_pairs) {
            e = cudaFreeAsync(edges[i], S->stream);
            edges[i] = nullptr;
        }
        if (e != cudaSuccess) rc = set_cuda_error(e);
    }
    if (rc == PA_OK) {
        e = cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(L.done, S->stream);
        if (e != cudaSuccess) rc = set_cuda_error(e);
    }
    if (rc != PA_OK) {
        // Whatever part of the group was queued may still read the pinned image:
        // let the stream drain before the buffers are reused or freed.
        cudaStreamSynchronize(S->stream);
        if (L.scratch) cudaFreeAsync(L.scratch, S->stream);
        for (void *b : cscr)
            if (b) cudaFreeAsync(b, S->stream);
        if (L.done) cudaEventDestroy(L.done);
    }
    std::lock_guard<std::mutex> lk(S->mu);
    for (uint32_t i = 0; i < k; ++i) {
        auto it = S->reqs.find(jobs[i].ticket);
        if (it == S->reqs.end()) continue;
        it->second.edges = edges[i];
        it->second.rowptr = (int64_t *)rowptr[i];
        it->second.col = col[i];
    }
    ++S->st.batches;
    if (rc == PA_OK) {
        S->inflight.push_back(L);
        return;
    }
    if (L.buf.p) S->pinned_free.push_back(L.buf);
    complete(S, L.tickets, rc, k);
}

void control_loop(pa_server *S)
{
    cudaSetDevice(S->device);
    const uint32_t max_batch = S->cfg.max_batch ? S->cfg.max_batch : 4096u;
    const uint32_t max_inflight = S->cfg.max_inflight ? S->cfg.max_inflight : 2u;
    std::vector<uint64_t> adm(max_batch);
    for (;;) {
        bool progressed = false;
        // 1. completions, in stream order
        while (!S->inflight.empty()) {
            Launch &L = S->inflight.front();
            const cudaError_t q = cudaEventQuery(L.done);
            if (q == cudaErrorNotReady) break;
            int status = PA_OK;
            if (q != cudaSuccess) {
                status = set_cuda_error(q);
            } else {
                uint32_t dev_status = 0;
                std::memcpy(&dev_status, L.buf.p + L.status_off, sizeof(dev_status));
                status = (int)dev_status;
            }
            cudaFreeAsync(L.scratch, S->stream);
            cudaEventDestroy(L.done);
            {
                std::lock_guard<std::mutex> lk(S->mu);
                S->pinned_free.push_back(L.buf);
                complete(S, L.tickets, status, (uint32_t)L.tickets.size(),
                         reinterpret_cast<const uint32_t *>(L.buf.p + L.status_off) + 1);
            }
            S->inflight.pop_front();
            progressed = true;
        }
        // 2. released and expired buffers
        std::vector<std::pair<uint64_t, void *>> frees;
        bool stopping;
        {
            std::lock_guard<std::mutex> lk(S->mu);
            if (S->cfg.ttl_ns) {
                const uint64_t t = S->now();
                while (!S->done_order.empty() && S->done_order.front().first + S->cfg.ttl_ns <= t) {
                    const uint64_t tk = S->done_order.front().second;
                    S->done_order.pop_front();
                    auto it = S->reqs.find(tk);
                    if (it == S->reqs.end() || it->second.state != RQ_DONE) continue;
                    drop_buffers(S, tk, it->second);
                    S->reqs.erase(it);
                    ++S->st.expired;
                }
            } else {
                S->done_order.clear();
            }
            frees.swap(S->to_free);
            stopping = S->stop;
        }
        for (auto &f : frees) {
            if (f.second) cudaFreeAsync(f.second, S->stream);
            if (f.first) pa_sched_release(S->sched, f.first, UINT64_MAX);
            progressed = true;
        }
        if (stopping && S->inflight.empty()) break;
        // 3. admission
        if (!stopping && S->inflight.size() < max_inflight) {
            std::vector<Job> j32, j64, solo;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                const uint64_t t = S->now();
                const uint32_t n = pa_sched_admit(S->sched, t, adm.data(), max_batch);
                for (uint32_t i = 0; i < n; ++i) {
                    Request &r = S->reqs[adm[i]];
                    r.state = RQ_RUNNING;
                    r.t_start = t;
                    const Job jb{adm[i], r.prm, r.edges_bytes, r.rowptr_bytes, r.col_bytes,
                                 r.csr_scratch};
                    if (!r.batchable) solo.push_back(jb);
                    else if (r.prm.id_bits == 64) j64.push_back(jb);
                    else j32.push_back(jb);
                }
            }
            if (!j32.empty()) launch_group(S, j32, true);
            if (!j64.empty()) launch_group(S, j64, true);
            for (const Job &jb : solo) launch_group(S, {jb}, false);
            if (!j32.empty() || !j64.empty() || !solo.empty()) progressed = true;
        }
        // 4. sleep
        if (!progressed) {
            std::unique_lock<std::mutex> lk(S->mu);
            if (S->inflight.empty())
                S->cv_work.wait_for(lk, std::chrono::milliseconds(2));
            else
                S->cv_work.wait_for(lk, std::chrono::microseconds(20));
        }
    }
    // shutdown: every launch has completed; free what is still held
    {
        std::lock_guard<std::mutex> lk(S->mu);
        for (auto &kv : S->reqs)
            for (void *b : {kv.second.edges, (void *)kv.second.rowptr, kv.second.col})
                if (b) cudaFreeAsync(b, S->stream);
        S->reqs.clear();
        for (auto &f : S->to_free)
            if (f.second) cudaFreeAsync(f.second, S->stream);
        S->to_free.clear();
        S->cv_done.notify_all();
    }
    cudaStreamSynchronize(S->stream);
}

}  // namespace

extern "C" {

int pa_server_config_init(pa_server_config *cfg)
{
    if (!cfg) return PA_ERR_INVALID;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->device = -1;
    return PA_OK;
}

int pa_server_create(const pa_server_config *cfg, pa_server **out)
{
    if (!cfg || !out) return PA_ERR_INVALID;
    *out = nullptr;
    if (cfg->reserved0 != 0 || (cfg->outputs & ~(uint32_t)(PA_OUT_PAIRS | PA_OUT_CSR)) != 0)
        return PA_ERR_INVALID;
    pa_server *S = new (std::nothrow) pa_server();
    if (!S) return PA_ERR_OOM;
    S->cfg = *cfg;
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    S->device = cfg->device >= 0 ? cfg->device : prev;
    if (e == cudaSuccess) e = cudaSetDevice(S->device);
    size_t free_b = 0, total_b = 0;
    if (e == cudaSuccess) e = cudaMemGetInfo(&free_b, &total_b);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&S->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        cudaMemPoolProps props;
        std::memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = S->device;
        e = cudaMemPoolCreate(&S->pool, &props);
    }
    if (e == cudaSuccess) {
        uint64_t keep = UINT64_MAX;   // freed blocks stay with the pool for reuse
        e = cudaMemPoolSetAttribute(S->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        if (S->pool) cudaMemPoolDestroy(S->pool);
        if (S->stream) cudaStreamDestroy(S->stream);
        delete S;
        return set_cuda_error(e);
    }
    if (S->cfg.budget_bytes == 0) S->cfg.budget_bytes = (uint64_t)free_b / 4 * 3;
    if (S->cfg.aging_ns == 0) S->cfg.aging_ns = 100000000ull;
    if (S->cfg.outputs == 0) S->cfg.outputs = PA_OUT_PAIRS;
    S->sched = pa_sched_create(S->cfg.budget_bytes, S->cfg.aging_ns, S->cfg.max_queue);
    if (!S->sched) {
        cudaMemPoolDestroy(S->pool);
        cudaStreamDestroy(S->stream);
        delete S;
        return PA_ERR_OOM;
    }
    S->st.budget_bytes = S->cfg.budget_bytes;
    S->t0 = std::chrono::steady_clock::now();
    S->worker = std::thread(control_loop, S);
    *out = S;
    return PA_OK;
}

int pa_server_submit(pa_server *S, const pa_params *prm, uint64_t *ticket)
{
    if (!S || !prm || !ticket) return PA_ERR_INVALID;
    GenPlan p;
    int rc = make_plan(prm, &p);
    if (rc != PA_OK) return rc;
    if (prm->flags != 0) return PA_ERR_INVALID;
    if (p.slots) return PA_ERR_NOT_SUPPORTED;
    Request r;
    r.prm = *prm;
    r.n_edges = p.n_edges;
    r.edges_bytes = p.edges_bytes;
    r.batchable = prm->n + 64 + 32 < (1ull << 32);
    r.scratch_reserve = scratch_reserve(*prm, r.batchable);
    if (S->cfg.outputs & PA_OUT_CSR) {
        rc = pa_csr_bytes(prm, &r.rowptr_bytes, &r.col_bytes, &r.csr_scratch);
        if (rc != PA_OK) return rc;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return PA_ERR_INVALID;
    r.t_submit = S->now();
    const uint64_t tk = S->next_ticket++;
    rc = pa_sched_submit(S->sched, tk,
                         r.edges_bytes + r.scratch_reserve + r.rowptr_bytes + r.col_bytes +
                             r.csr_scratch,
                         r.t_submit);
    if (rc != PA_OK) return rc;
    S->reqs.emplace(tk, r);
    ++S->st.submitted;
    *ticket = tk;
    S->cv_work.notify_one();
    return PA_OK;
}

static void fill_result(const Request &r, pa_result *out)
{
    if (!out) return;
    out->edges = r.edges;
    out->n_edges = r.n_edges;
    out->edges_bytes = r.edges_bytes;
    out->status = r.status;
    out->batch_size = r.batch_size;
    out->t_submit_ns = r.t_submit;
    out->t_start_ns = r.t_start;
    out->t_done_ns = r.t_done;
    out->rowptr = r.rowptr;
    out->col = r.col;
    out->col_bytes = r.col ? r.col_bytes : 0;
}

int pa_server_poll(pa_server *S, uint64_t ticket, pa_result *out)
{
    if (!S) return PA_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return PA_ERR_NOT_FOUND;
    if (it->second.state != RQ_DONE) return PA_ERR_BUSY;
    fill_result(it->second, out);
    return PA_OK;
}

int pa_server_wait(pa_server *S, uint64_t ticket, uint64_t timeout_ns, pa_result *out)
{
    if (!S) return PA_ERR_INVALID;
    std::unique_lock<std::mutex> lk(S->mu);
    const auto deadline = std::chrono::steady_clock::now() + std::chrono::nanoseconds(timeout_ns);
    for (;;) {
        auto it = S->reqs.find(ticket);
        if (it == S->reqs.end()) return PA_ERR_NOT_FOUND;
        if (it->second.state == RQ_DONE) {
            fill_result(it->second, out);
            return PA_OK;
        }
        if (timeout_ns == 0) {
            S->cv_done.wait_for(lk, std::chrono::milliseconds(50));
        } else {
            if (std::chrono::steady_clock::now() >= deadline) return PA_ERR_BUSY;
            S->cv_done.wait_until(lk, deadline);
        }
    }
}

int pa_server_release(pa_server *S, uint64_t ticket)
{
    if (!S) return PA_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return PA_ERR_NOT_FOUND;
    Request &r = it->second;
    if (r.state == RQ_RUNNING) return PA_ERR_BUSY;
    if (r.state == RQ_QUEUED)
        pa_sched_release(S->sched, ticket, UINT64_MAX);   // withdrawn before admission
    else
        drop_buffers(S, ticket, r);
    S->reqs.erase(it);
    ++S->st.released;
    S->cv_work.notify_one();
    return PA_OK;
}

int pa_server_stats_get(pa_server *S, pa_server_stats *out)
{
    if (!S || !out) return PA_ERR_INVALID;
    std::lock_guard<std::mutex> lk(S->mu);
    *out = S->st;
    out->queued = pa_sched_queued(S->sched);
    uint64_t running = 0;
    for (const auto &kv : S->reqs)
        if (kv.second.state == RQ_RUNNING) ++running;
    out->running = running;
    out->bytes_in_use = pa_sched_in_use(S->sched);
    return PA_OK;
}

int pa_server_destroy(pa_server *S)
{
    if (!S) return PA_ERR_INVALID;
    {
        std::lock_guard<std::mutex> lk(S->mu);
        S->stop = true;
        S->cv_work.notify_all();
    }
    if (S->worker.joinable()) S->worker.join();
    for (auto &b : S->pinned_free) cudaFreeHost(b.p);
    cudaMemPoolDestroy(S->pool);
    cudaStreamDestroy(S->stream);
    pa_sched_destroy(S->sched);
    delete S;
    return PA_OK;
}

}  // extern "C"
