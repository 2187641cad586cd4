// pa_sched.cpp -- admission queue of the request server (host logic only).
//
// Requests wait in arrival order.  An admission scan walks the queue from the
// front: a request whose bytes fit the free budget is admitted; one that does
// not is passed over, so small requests keep the GPU busy behind a large one --
// unless the passed-over request has already waited aging_ns, in which case
// the scan stops there and the budget that frees up goes to it first.  Budget
// comes back when a request (or part of it, e.g. its generation scratch once
// the batch has run) is released.
//
// The request server tags each request with a lane (bulk or express) and
// admits per lane: a scan for some lanes skips the others' requests, and an
// aged request stops admission of its own lane only.
#include <cstdint>
#include <deque>
#include <mutex>
#include <new>
#include <unordered_map>

#include "cuppa_pa.h"

struct pa_sched {
    struct Item {
        uint64_t ticket, bytes, t_submit;
        uint32_t lane;
    };
    std::deque<Item> queue;
    std::unordered_map<uint64_t, uint64_t> held;   // admitted ticket -> bytes still held
    uint64_t budget = 0, in_use = 0, aging = 0;
    uint32_t max_queue = 0;
    mutable std::mutex mu;
};

extern "C" {

int pa_sched_submit_lane(pa_sched *q, uint64_t ticket, uint64_t bytes, uint64_t now_ns,
                         uint32_t lane)
{
    if (!q || lane >= 32) return PA_ERR_INVALID;
    std::lock_guard<std::mutex> lk(q->mu);
    if (bytes > q->budget) return PA_ERR_CAPACITY;
    if (q->max_queue && q->queue.size() >= q->max_queue) return PA_ERR_BUSY;
    if (q->held.count(ticket)) return PA_ERR_INVALID;
    for (const auto &it : q->queue)
        if (it.ticket == ticket) return PA_ERR_INVALID;
    q->queue.push_back({ticket, bytes, now_ns, lane});
    return PA_OK;
}

uint32_t pa_sched_admit_lanes(pa_sched *q, uint64_t now_ns, uint64_t *out, uint32_t cap,
                              uint32_t lane_mask)
{
    if (!q || !out || cap == 0) return 0;
    std::lock_guard<std::mutex> lk(q->mu);
    uint32_t n = 0;
    uint32_t open = lane_mask;   // lanes still admitting in this scan
    for (auto it = q->queue.begin(); it != q->queue.end() && n < cap && open;) {
        const uint32_t bit = 1u << it->lane;
        if (!(open & bit)) {
            ++it;
        } else if (it->bytes <= q->budget - q->in_use) {
            q->in_use += it->bytes;
            q->held[it->ticket] = it->bytes;
            out[n++] = it->ticket;
            it = q->queue.erase(it);
        } else if (now_ns - it->t_submit >= q->aging) {
            open &= ~bit;   // an aged request keeps its turn in its lane
            ++it;
        } else {
            ++it;
        }
    }
    return n;
}

pa_sched *pa_sched_create(uint64_t budget_bytes, uint64_t aging_ns, uint32_t max_queue)
{
    pa_sched *q = new (std::nothrow) pa_sched();
    if (!q) return nullptr;
    q->budget = budget_bytes;
    q->aging = aging_ns;
    q->max_queue = max_queue;
    return q;
}

void pa_sched_destroy(pa_sched *q) { delete q; }

int pa_sched_submit(pa_sched *q, uint64_t ticket, uint64_t bytes, uint64_t now_ns)
{
    return pa_sched_submit_lane(q, ticket, bytes, now_ns, 0);
}

uint32_t pa_sched_admit(pa_sched *q, uint64_t now_ns, uint64_t *out, uint32_t cap)
{
    return pa_sched_admit_lanes(q, now_ns, out, cap, ~0u);
}

int pa_sched_release(pa_sched *q, uint64_t ticket, uint64_t bytes)
{
    if (!q) return PA_ERR_INVALID;
    std::lock_guard<std::mutex> lk(q->mu);
    auto it = q->held.find(ticket);
    if (it == q->held.end()) {
        // a request still queued is simply withdrawn
        for (auto jt = q->queue.begin(); jt != q->queue.end(); ++jt)
            if (jt->ticket == ticket) {
                if (bytes != UINT64_MAX) return PA_ERR_INVALID;
                q->queue.erase(jt);
                return PA_OK;
            }
        return PA_ERR_NOT_FOUND;
    }
    const uint64_t give = bytes == UINT64_MAX || bytes > it->second ? it->second : bytes;
    it->second -= give;
    q->in_use -= give;
    if (bytes == UINT64_MAX) q->held.erase(it);
    return PA_OK;
}

uint64_t pa_sched_in_use(const pa_sched *q)
{
    if (!q) return 0;
    std::lock_guard<std::mutex> lk(q->mu);
    return q->in_use;
}

uint64_t pa_sched_queued(const pa_sched *q)
{
    if (!q) return 0;
    std::lock_guard<std::mutex> lk(q->mu);
    return q->queue.size();
}

}  // extern "C"
