// pa_server.cu -- the request server: continuous batching of generation
// requests under a device-memory budget.
//
// One control thread per server owns the server's CUDA streams and memory
// pools on its device.  Client threads only touch host state (under the server
// mutex): submit queues a request with the admission queue (pa_sched.cpp),
// poll/wait read its state, release hands its buffer back.
//
// Two lanes share the budget.  Requests of at most express_edges edges go to
// the express lane, the rest to the bulk lane.  Each lane has one stream (the
// express lane's at the device's highest stream priority), on which up to
// max_inflight of its launches queue in order, and a memory pool of its own, so
// that an allocation never waits for memory freed behind the other lane's
// work.  Kernels are not preempted, but the block scheduler hands SMs that free
// up to waiting blocks of higher-priority streams first: a small request that
// arrives while a large batch runs starts at the batch's next kernel boundary
// (a start kernel's tail, or between its CSR kernels) instead of after the
// whole batch.
//
// The control thread loops, never waiting on the GPU:
//   1. completions: for each in-flight launch whose event has fired, read the
//      device status it copied back, mark its requests done and return their
//      generation scratch to the budget; retired launches (an error after part
//      of a launch was queued) give their staging buffers back the same way;
//   2. frees: buffers of released (or TTL-expired) results are freed on the
//      stream that made them and their budget returned;
//   3. admission: for each lane with room in flight, admit what fits the budget
//      and launch it as one batch per id width (the fill / start / tail launches
//      of pa_batch.cu) -- requests that arrived while earlier batches ran make
//      up the next; a group whose allocations fail (a fragmented pool) waits,
//      admitted, for the next completion and is retried;
//   4. sleep briefly (20 us with work in flight, else until woken).
// Memory per request: its edge buffer plus the generation scratch of its own
// plan, which bounds its share of the batch scratch; with CSR outputs also its
// rowptr, col and CSR scratch.  The CSR of every request of a batch is queued
// on the batch's stream right after it; the CSR scratch (and the edge buffer,
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
    uint32_t lane = 0;                 // kBulk or kExpress
    cudaStream_t stream = nullptr;     // the stream that made (and frees) its buffers
};

constexpr uint32_t kBulk = 0, kExpress = 1, kLanes = 2;
constexpr uint64_t kExpressEdgesAuto = 1ull << 22;

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
    cudaStream_t stream = nullptr;
};

// Staging of a launch that failed after part of it was queued: returned to the
// pools once the work queued before the failure has run.
struct Retired {
    cudaEvent_t done = nullptr;
    cudaStream_t stream = nullptr;
    Pinned buf;
    std::vector<void *> device;   // freed on `stream` when `done` fires
};

// What the control thread needs of an admitted request (copied under the lock).
struct Job {
    uint64_t ticket;
    pa_params prm;
    uint64_t edges_bytes, rowptr_bytes, col_bytes, csr_scratch;
};

struct LaneState {
    std::vector<cudaStream_t> streams;             // one stream: launches queue in order
    cudaMemPool_t pool = nullptr;                  // the lane's own device memory
    std::vector<Launch> inflight;                  // each on one of `streams`
    std::deque<std::pair<std::vector<Job>, bool>> deferred;   // groups (batch?) waiting to
                                                               // be retried after a completion
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
    uint64_t express_edges = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    pa_sched *sched = nullptr;
    std::unordered_map<uint64_t, Request> reqs;
    // work for the control thread: free the buffer (if any) on the stream, then
    // return the ticket's whole budget (if the ticket is not 0)
    struct Free {
        uint64_t ticket;
        void *ptr;
        cudaStream_t stream;
    };
    std::vector<Free> to_free;
    std::deque<std::pair<uint64_t, uint64_t>> done_order;  // t_done, ticket (TTL)
    uint64_t next_ticket = 1;
    std::chrono::steady_clock::time_point t0;
    pa_server_stats st{};
    // control thread only
    LaneState lanes[kLanes];
    std::vector<Retired> retired;
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
// Buffers are freed in order on the stream that made them (the lane's stream,
// whose pool owns them).
void drop_buffers(pa_server *S, uint64_t tk, Request &r)
{
    for (void *b : {r.edges, (void *)r.rowptr, r.col})
        if (b) S->to_free.push_back({0, b, r.stream});
    S->to_free.push_back({tk, nullptr, nullptr});
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

// A pool allocation, stream-ordered on s.  When the pool's free blocks are too
// fragmented, its memory that is free and no longer in use goes back to the
// device and the allocation is tried once more; the caller retries later
// (after a completion) if that fails too.  Nothing here waits for the GPU.
cudaError_t pool_alloc(cudaMemPool_t pool, void **p, uint64_t bytes, cudaStream_t s)
{
    cudaError_t e = cudaMallocFromPoolAsync(p, std::max<uint64_t>(bytes, 16), pool, s);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        cudaMemPoolTrimTo(pool, 0);
        e = cudaMallocFromPoolAsync(p, std::max<uint64_t>(bytes, 16), pool, s);
        if (e != cudaSuccess) (void)cudaGetLastError();
    }
    return e;
}

// The lane's stream with the fewest launches in flight.
cudaStream_t pick_stream(const LaneState &L)
{
    cudaStream_t best = L.streams[0];
    size_t best_n = SIZE_MAX;
    for (cudaStream_t s : L.streams) {
        size_t c = 0;
        for (const Launch &x : L.inflight) c += x.stream == s;
        if (c < best_n) {
            best_n = c;
            best = s;
        }
    }
    return best;
}

// Launch one group of admitted requests (same id width, all batchable) as a
// batch, or one request alone, on the lane's least busy stream; then, with CSR
// outputs, every request's CSR.  Called without the lock.  When an allocation
// fails before anything is queued and may_defer is set, the partial
// allocations are freed and false is returned: the caller keeps the group
// (admitted, its budget held) and retries after a completion.
bool launch_group(pa_server *S, const std::vector<Job> &jobs, bool batch, uint32_t lane,
                  bool may_defer)
{
    LaneState &LS = S->lanes[lane];
    const cudaStream_t st = pick_stream(LS);
    const uint32_t k = (uint32_t)jobs.size();
    const bool csr = (S->cfg.outputs & PA_OUT_CSR) != 0;
    const bool keep_pairs = (S->cfg.outputs & PA_OUT_PAIRS) != 0;
    std::vector<void *> edges(k, nullptr), rowptr(k, nullptr), col(k, nullptr), cscr(k, nullptr);
    std::vector<pa_params> prms(k);
    std::vector<uint64_t> ebytes(k);
    Launch L;
    L.stream = st;
    for (uint32_t i = 0; i < k; ++i) {
        L.tickets.push_back(jobs[i].ticket);
        prms[i] = jobs[i].prm;
        ebytes[i] = jobs[i].edges_bytes;
    }
    int rc = PA_OK;
    cudaError_t e = cudaSuccess;
    for (uint32_t i = 0; i < k && e == cudaSuccess; ++i) {
        e = pool_alloc(LS.pool, &edges[i], ebytes[i], st);
        if (csr && e == cudaSuccess) e = pool_alloc(LS.pool, &rowptr[i], jobs[i].rowptr_bytes, st);
        if (csr && e == cudaSuccess) e = pool_alloc(LS.pool, &col[i], jobs[i].col_bytes, st);
    }
    BatchJob J;
    uint64_t scratch_bytes = 0, image_bytes = 0;
    if (e == cudaSuccess) {
        if (batch) {
            rc = batch_prepare(prms.data(), k, J);
            scratch_bytes = J.scratch_bytes;
            image_bytes = J.image_bytes;
        } else {
            rc = pa_scratch_bytes(&prms[0], &scratch_bytes);
        }
        if (rc == PA_OK) e = pool_alloc(LS.pool, &L.scratch, scratch_bytes, st);
    }
    if (e != cudaSuccess && may_defer) {
        // nothing queued yet: give the memory back (stream-ordered) and wait
        for (uint32_t i = 0; i < k; ++i)
            for (void *b : {edges[i], rowptr[i], col[i]})
                if (b) cudaFreeAsync(b, st);
        if (L.scratch) cudaFreeAsync(L.scratch, st);
        return false;
    }
    if (e != cudaSuccess && rc == PA_OK) rc = set_cuda_error(e);
    if (rc == PA_OK) {
        L.status_off = (image_bytes + 15) & ~15ull;
        L.buf = get_pinned(S, L.status_off + 4ull * (k + 1));
        if (!L.buf.p) rc = PA_ERR_OOM;
    }
    bool queued = false;   // work that reads the pinned image or the scratch is queued
    if (rc == PA_OK && batch) {
        rc = batch_bind(J, prms.data(), edges.data(), ebytes.data(), L.scratch, L.buf.p);
        queued = true;
        if (rc == PA_OK) rc = batch_enqueue(J, L.scratch, L.buf.p, st);
    } else if (rc == PA_OK) {
        queued = true;
        rc = pa_generate(&prms[0], edges[0], ebytes[0], L.scratch, scratch_bytes, st);
    }
    if (rc == PA_OK) {
        e = cudaMemcpyAsync(L.buf.p + L.status_off,
                            (const unsigned char *)L.scratch + offsetof(GenCtl, error),
                            sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
        if (e != cudaSuccess) rc = set_cuda_error(e);
    }
    // CSR of every request, in the same stream; its scratch (and the pairs when
    // they are not kept) is freed in stream order behind it
    uint32_t *csr_status = L.buf.p ? reinterpret_cast<uint32_t *>(L.buf.p + L.status_off) + 1
                                   : nullptr;
    for (uint32_t i = 0; i < k && rc == PA_OK; ++i) {
        if (!csr) {
            csr_status[i] = PA_OK;
            continue;
        }
        e = pool_alloc(LS.pool, &cscr[i], jobs[i].csr_scratch, st);
        if (e != cudaSuccess) {
            rc = set_cuda_error(e);
            break;
        }
        uint64_t err_off = 0;
        rc = csr_enqueue(&prms[i], edges[i], (int64_t *)rowptr[i], col[i], cscr[i],
                         jobs[i].csr_scratch, st, &err_off);
        if (rc != PA_OK) break;
        e = cudaMemcpyAsync(csr_status + i, (const unsigned char *)cscr[i] + err_off, 4,
                            cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaFreeAsync(cscr[i], st);
        cscr[i] = nullptr;
        if (e == cudaSuccess && !keep_pairs) {
            e = cudaFreeAsync(edges[i], st);
            edges[i] = nullptr;
        }
        if (e != cudaSuccess) rc = set_cuda_error(e);
    }
    if (rc == PA_OK) {
        e = cudaEventCreateWithFlags(&L.done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(L.done, st);
        if (e != cudaSuccess) rc = set_cuda_error(e);
    }
    if (rc != PA_OK) {
        // The staging may still be read by what was queued before the failure:
        // it is given back when an event behind that work fires.
        if (L.done) {
            cudaEventDestroy(L.done);
            L.done = nullptr;
        }
        Retired R;
        R.stream = st;
        R.buf = L.buf;
        if (L.scratch) R.device.push_back(L.scratch);
        for (void *b : cscr)
            if (b) R.device.push_back(b);
        bool parked = false;
        if (queued && cudaEventCreateWithFlags(&R.done, cudaEventDisableTiming) == cudaSuccess) {
            if (cudaEventRecord(R.done, st) == cudaSuccess) {
                S->retired.push_back(R);
                parked = true;
            } else {
                cudaEventDestroy(R.done);
            }
        }
        if (!parked) {
            // nothing queued (or no event to wait on): the stream orders the frees
            if (queued) cudaStreamSynchronize(st);   // last resort: no event could be made
            for (void *b : R.device) cudaFreeAsync(b, st);
            if (R.buf.p) {
                std::lock_guard<std::mutex> lk(S->mu);
                S->pinned_free.push_back(R.buf);
            }
        }
        L.buf = Pinned{};
    }
    std::lock_guard<std::mutex> lk(S->mu);
    for (uint32_t i = 0; i < k; ++i) {
        auto it = S->reqs.find(jobs[i].ticket);
        if (it == S->reqs.end()) continue;
        it->second.edges = edges[i];
        it->second.rowptr = (int64_t *)rowptr[i];
        it->second.col = col[i];
        it->second.stream = st;
    }
    ++S->st.batches;
    if (rc == PA_OK) {
        LS.inflight.push_back(L);
        return true;
    }
    complete(S, L.tickets, rc, k);
    return true;
}

// Admitted requests of one lane as launch groups: one batch per id width, and
// requests too large for the batch kernels alone.  Lock held.
std::vector<std::pair<std::vector<Job>, bool>> make_groups(pa_server *S, const uint64_t *tickets,
                                                           uint32_t n, uint64_t t)
{
    std::vector<Job> j32, j64;
    std::vector<std::pair<std::vector<Job>, bool>> out;
    for (uint32_t i = 0; i < n; ++i) {
        Request &r = S->reqs[tickets[i]];
        r.state = RQ_RUNNING;
        r.t_start = t;
        const Job jb{tickets[i], r.prm, r.edges_bytes, r.rowptr_bytes, r.col_bytes, r.csr_scratch};
        if (!r.batchable) out.push_back({{jb}, false});
        else if (r.prm.id_bits == 64) j64.push_back(jb);
        else j32.push_back(jb);
    }
    if (!j64.empty()) out.insert(out.begin(), {j64, true});
    if (!j32.empty()) out.insert(out.begin(), {j32, true});
    return out;
}

bool anything_in_flight(const pa_server *S)
{
    for (const LaneState &L : S->lanes)
        if (!L.inflight.empty()) return true;
    return !S->retired.empty();
}

void control_loop(pa_server *S)
{
    cudaSetDevice(S->device);
    const uint32_t max_batch = S->cfg.max_batch ? S->cfg.max_batch : 4096u;
    const uint32_t max_inflight = S->cfg.max_inflight ? S->cfg.max_inflight : 4u;
    std::vector<uint64_t> adm(max_batch);
    for (;;) {
        bool progressed = false, freed = false;
        // 1. completions (each stream runs its launches in order; streams in any order)
        for (LaneState &LS : S->lanes) {
            for (size_t i = 0; i < LS.inflight.size();) {
                Launch &L = LS.inflight[i];
                const cudaError_t q = cudaEventQuery(L.done);
                if (q == cudaErrorNotReady) {
                    ++i;
                    continue;
                }
                int status = PA_OK;
                if (q != cudaSuccess) {
                    status = set_cuda_error(q);
                } else {
                    uint32_t dev_status = 0;
                    std::memcpy(&dev_status, L.buf.p + L.status_off, sizeof(dev_status));
                    status = (int)dev_status;
                }
                cudaFreeAsync(L.scratch, L.stream);
                cudaEventDestroy(L.done);
                {
                    std::lock_guard<std::mutex> lk(S->mu);
                    S->pinned_free.push_back(L.buf);
                    complete(S, L.tickets, status, (uint32_t)L.tickets.size(),
                             reinterpret_cast<const uint32_t *>(L.buf.p + L.status_off) + 1);
                }
                LS.inflight.erase(LS.inflight.begin() + (ptrdiff_t)i);
                progressed = freed = true;
            }
        }
        for (size_t i = 0; i < S->retired.size();) {
            Retired &R = S->retired[i];
            if (cudaEventQuery(R.done) == cudaErrorNotReady) {
                ++i;
                continue;
            }
            for (void *b : R.device) cudaFreeAsync(b, R.stream);
            cudaEventDestroy(R.done);
            if (R.buf.p) {
                std::lock_guard<std::mutex> lk(S->mu);
                S->pinned_free.push_back(R.buf);
            }
            S->retired.erase(S->retired.begin() + (ptrdiff_t)i);
            progressed = freed = true;
        }
        // 2. released and expired buffers
        std::vector<pa_server::Free> frees;
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
            if (f.ptr) cudaFreeAsync(f.ptr, f.stream ? f.stream : S->lanes[kBulk].streams[0]);
            if (f.ticket) pa_sched_release(S->sched, f.ticket, UINT64_MAX);
            progressed = freed = true;
        }
        // 3. groups whose allocations failed: retried once memory has come back,
        // failed when nothing is left in flight to give any back
        for (uint32_t lane = 0; lane < kLanes; ++lane) {
            LaneState &LS = S->lanes[lane];
            while (!LS.deferred.empty() && LS.inflight.size() < max_inflight) {
                auto &g = LS.deferred.front();
                if (stopping) {
                    std::vector<uint64_t> tks;
                    for (const Job &jb : g.first) tks.push_back(jb.ticket);
                    std::lock_guard<std::mutex> lk(S->mu);
                    complete(S, tks, PA_ERR_OOM, (uint32_t)tks.size());
                } else {
                    const bool busy = anything_in_flight(S);
                    if (busy && !freed) break;
                    if (!launch_group(S, g.first, g.second, lane, busy)) break;
                }
                LS.deferred.pop_front();
                progressed = true;
            }
        }
        if (stopping && !anything_in_flight(S) && S->lanes[kBulk].deferred.empty() &&
            S->lanes[kExpress].deferred.empty())
            break;
        // 4. admission, lane by lane
        for (uint32_t lane = 0; lane < kLanes && !stopping; ++lane) {
            LaneState &LS = S->lanes[lane];
            if (LS.inflight.size() >= max_inflight || !LS.deferred.empty()) continue;
            std::vector<std::pair<std::vector<Job>, bool>> groups;
            {
                std::lock_guard<std::mutex> lk(S->mu);
                const uint64_t t = S->now();
                const uint32_t n = pa_sched_admit_lanes(S->sched, t, adm.data(), max_batch, 1u << lane);
                groups = make_groups(S, adm.data(), n, t);
            }
            for (auto &g : groups) {
                if (!LS.deferred.empty() || !launch_group(S, g.first, g.second, lane, true))
                    LS.deferred.push_back(g);
                progressed = true;
            }
        }
        // 5. sleep
        if (!progressed) {
            std::unique_lock<std::mutex> lk(S->mu);
            if (!anything_in_flight(S))
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
                if (b) cudaFreeAsync(b, kv.second.stream ? kv.second.stream
                                                         : S->lanes[kBulk].streams[0]);
        S->reqs.clear();
        for (auto &f : S->to_free)
            if (f.ptr) cudaFreeAsync(f.ptr, f.stream ? f.stream : S->lanes[kBulk].streams[0]);
        S->to_free.clear();
        S->cv_done.notify_all();
    }
    for (const LaneState &LS : S->lanes)
        for (cudaStream_t s : LS.streams) cudaStreamSynchronize(s);
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
    if ((cfg->outputs & ~(uint32_t)(PA_OUT_PAIRS | PA_OUT_CSR)) != 0) return PA_ERR_INVALID;
    pa_server *S = new (std::nothrow) pa_server();
    if (!S) return PA_ERR_OOM;
    S->cfg = *cfg;
    S->express_edges = cfg->express_edges ? cfg->express_edges : kExpressEdgesAuto;
    int prev = 0;
    cudaError_t e = cudaGetDevice(&prev);
    S->device = cfg->device >= 0 ? cfg->device : prev;
    if (e == cudaSuccess) e = cudaSetDevice(S->device);
    size_t free_b = 0, total_b = 0;
    if (e == cudaSuccess) e = cudaMemGetInfo(&free_b, &total_b);
    int least = 0, greatest = 0;
    if (e == cudaSuccess) e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    for (uint32_t lane = 0; lane < kLanes && e == cudaSuccess; ++lane) {
        LaneState &LS = S->lanes[lane];
        cudaStream_t s = nullptr;
        e = cudaStreamCreateWithPriority(&s, cudaStreamNonBlocking,
                                         lane == kExpress ? greatest : least);
        if (e == cudaSuccess) LS.streams.push_back(s);
        if (e == cudaSuccess) {
            cudaMemPoolProps props;
            std::memset(&props, 0, sizeof(props));
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = S->device;
            e = cudaMemPoolCreate(&LS.pool, &props);
        }
        if (e == cudaSuccess) {
            uint64_t keep = UINT64_MAX;   // freed blocks stay with the pool for reuse
            e = cudaMemPoolSetAttribute(LS.pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    auto destroy_lanes = [&] {
        for (LaneState &LS : S->lanes) {
            for (cudaStream_t s : LS.streams) cudaStreamDestroy(s);
            if (LS.pool) cudaMemPoolDestroy(LS.pool);
        }
    };
    cudaSetDevice(prev);
    if (e != cudaSuccess) {
        destroy_lanes();
        delete S;
        return set_cuda_error(e);
    }
    if (S->cfg.budget_bytes == 0) S->cfg.budget_bytes = (uint64_t)free_b / 4 * 3;
    if (S->cfg.aging_ns == 0) S->cfg.aging_ns = 100000000ull;
    if (S->cfg.outputs == 0) S->cfg.outputs = PA_OUT_PAIRS;
    S->sched = pa_sched_create(S->cfg.budget_bytes, S->cfg.aging_ns, S->cfg.max_queue);
    if (!S->sched) {
        destroy_lanes();
        delete S;
        return PA_ERR_OOM;
    }
    // Map each lane's share of the budget into its pool now (allocated once and
    // freed; the pool keeps freed memory), so that serving does not grow the
    // pools -- a driver mapping on the control thread -- while requests wait.
    // The express lane's requests are small: an eighth of the budget.
    if (S->cfg.budget_bytes) {
        cudaSetDevice(S->device);
        for (uint32_t lane = 0; lane < kLanes; ++lane) {
            LaneState &LS = S->lanes[lane];
            const uint64_t share = lane == kExpress ? S->cfg.budget_bytes / 8
                                                    : S->cfg.budget_bytes - S->cfg.budget_bytes / 8;
            void *p = nullptr;
            if (cudaMallocFromPoolAsync(&p, share, LS.pool, LS.streams[0]) == cudaSuccess)
                cudaFreeAsync(p, LS.streams[0]);
            else
                (void)cudaGetLastError();   // best effort: the pool grows on demand instead
            cudaStreamSynchronize(LS.streams[0]);
        }
        cudaSetDevice(prev);
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
    if (p.slots || p.wide) return PA_ERR_NOT_SUPPORTED;
    Request r;
    r.prm = *prm;
    r.n_edges = p.n_edges;
    r.edges_bytes = p.edges_bytes;
    r.batchable = prm->n + 64 + 32 < (1ull << 32);
    r.scratch_reserve = scratch_reserve(*prm, r.batchable);
    r.lane = p.n_edges <= S->express_edges ? kExpress : kBulk;
    if (S->cfg.outputs & PA_OUT_CSR) {
        rc = pa_csr_bytes(prm, &r.rowptr_bytes, &r.col_bytes, &r.csr_scratch);
        if (rc != PA_OK) return rc;
    }
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->stop) return PA_ERR_INVALID;
    r.t_submit = S->now();
    const uint64_t tk = S->next_ticket++;
    rc = pa_sched_submit_lane(S->sched, tk,
                              r.edges_bytes + r.scratch_reserve + r.rowptr_bytes + r.col_bytes +
                                  r.csr_scratch,
                              r.t_submit, r.lane);
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
    for (LaneState &LS : S->lanes) {
        for (cudaStream_t s : LS.streams) cudaStreamDestroy(s);
        cudaMemPoolDestroy(LS.pool);
    }
    pa_sched_destroy(S->sched);
    delete S;
    return PA_OK;
}

}  // extern "C"
