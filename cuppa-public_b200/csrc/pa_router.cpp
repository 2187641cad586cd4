// pa_router.cpp -- requests spread over several GPUs (host logic only).
//
// One graph never spans GPUs: every copy read may land on any earlier node, so
// a graph stays on the GPU that generates it, and more GPUs serve more graphs.
// The router owns one request server per device (pa_server_*, each with its own
// control thread, memory pool and admission queue) and places each request on
// the server whose routed, unreleased bytes would be the smallest fraction of
// its budget.  Tickets carry the server index in their low byte; results, waits
// and releases go to that server.  No data crosses between GPUs, so there is no
// collective; NVLink is not involved.
//
// pa_batch_partition is the batch counterpart: instances are dealt to k parts
// largest first, each to the part with the fewest edge bytes so far (LPT), so
// one process per GPU can each run pa_batch_generate on its own part.
#include <algorithm>
#include <cstdint>
#include <mutex>
#include <new>
#include <numeric>
#include <unordered_map>
#include <vector>

#include "cuppa_pa.h"

namespace {

constexpr uint32_t kMaxServers = 255;

// Bytes a request holds on its server while admitted or unreleased: its edge
// list, plus the CSR arrays when the server keeps CSR.
uint64_t request_bytes(const pa_params *prm, uint32_t outputs)
{
    uint64_t eb = 0;
    if (pa_edges_bytes(prm, &eb) != PA_OK) return 0;
    uint64_t total = (outputs & PA_OUT_PAIRS) || outputs == 0 ? eb : 0;
    if (outputs & PA_OUT_CSR) {
        uint64_t rb = 0, cb = 0, sb = 0;
        if (pa_csr_bytes(prm, &rb, &cb, &sb) == PA_OK) total += rb + cb;
    }
    return total ? total : 1;
}

}  // namespace

struct pa_router {
    std::vector<pa_server *> servers;
    std::vector<int32_t> devices;
    std::vector<uint64_t> budget;
    std::vector<uint64_t> load;                       // routed, unreleased bytes
    std::unordered_map<uint64_t, uint64_t> held;      // router ticket -> bytes
    uint32_t outputs = PA_OUT_PAIRS;
    std::mutex mu;
};

extern "C" {

uint32_t pa_route_pick(const uint64_t *load_bytes, const uint64_t *budget_bytes, uint32_t n,
                       uint64_t request_bytes)
{
    if (!load_bytes || !budget_bytes || n == 0) return 0;
    uint32_t best = 0;
    for (uint32_t i = 1; i < n; ++i) {
        // (load_i + req) / budget_i < (load_b + req) / budget_b, without rounding
        const unsigned __int128 lhs =
            (unsigned __int128)(load_bytes[i] + request_bytes) * budget_bytes[best];
        const unsigned __int128 rhs =
            (unsigned __int128)(load_bytes[best] + request_bytes) * budget_bytes[i];
        if (lhs < rhs) best = i;
    }
    return best;
}

int pa_batch_partition(const pa_params *prms, uint32_t count, uint32_t k, uint32_t *part_of)
{
    if ((!prms && count) || k == 0 || (!part_of && count)) return PA_ERR_INVALID;
    std::vector<uint64_t> w(count);
    for (uint32_t i = 0; i < count; ++i) {
        uint64_t eb = 0;
        const int rc = pa_edges_bytes(prms + i, &eb);
        if (rc != PA_OK) return rc;
        w[i] = eb;
    }
    std::vector<uint32_t> order(count);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(),
                     [&](uint32_t a, uint32_t b) { return w[a] > w[b]; });
    std::vector<uint64_t> sum(k, 0);
    for (uint32_t i : order) {
        const uint32_t p = (uint32_t)(std::min_element(sum.begin(), sum.end()) - sum.begin());
        part_of[i] = p;
        sum[p] += w[i];
    }
    return PA_OK;
}

int pa_router_create(const pa_server_config *cfg, const int32_t *devices, uint32_t n_devices,
                     pa_router **out)
{
    if (!cfg || !devices || !out || n_devices == 0 || n_devices > kMaxServers)
        return PA_ERR_INVALID;
    *out = nullptr;
    pa_router *r = new (std::nothrow) pa_router();
    if (!r) return PA_ERR_OOM;
    r->outputs = cfg->outputs ? cfg->outputs : PA_OUT_PAIRS;
    for (uint32_t i = 0; i < n_devices; ++i) {
        pa_server_config c = *cfg;
        c.device = devices[i];
        pa_server *s = nullptr;
        int rc = pa_server_create(&c, &s);
        pa_server_stats st;
        if (rc == PA_OK) rc = pa_server_stats_get(s, &st);
        if (rc != PA_OK) {
            if (s) pa_server_destroy(s);
            for (pa_server *x : r->servers) pa_server_destroy(x);
            delete r;
            return rc;
        }
        r->servers.push_back(s);
        r->devices.push_back(devices[i]);
        r->budget.push_back(st.budget_bytes ? st.budget_bytes : 1);
        r->load.push_back(0);
    }
    *out = r;
    return PA_OK;
}

int pa_router_submit(pa_router *r, const pa_params *prm, uint64_t *ticket)
{
    if (!r || !prm || !ticket) return PA_ERR_INVALID;
    const uint64_t bytes = request_bytes(prm, r->outputs);
    uint32_t i;
    {
        std::lock_guard<std::mutex> lk(r->mu);
        i = pa_route_pick(r->load.data(), r->budget.data(), (uint32_t)r->servers.size(), bytes);
        r->load[i] += bytes;   // reserved before the submit, so concurrent submits spread
    }
    uint64_t t = 0;
    const int rc = pa_server_submit(r->servers[i], prm, &t);
    std::lock_guard<std::mutex> lk(r->mu);
    if (rc != PA_OK) {
        r->load[i] -= bytes;
        return rc;
    }
    *ticket = (t << 8) | i;
    r->held[*ticket] = bytes;
    return PA_OK;
}

// Drop a ticket's routed bytes (released, or gone from its server by TTL).
static void forget(pa_router *r, uint64_t ticket, uint32_t i)
{
    std::lock_guard<std::mutex> lk(r->mu);
    auto it = r->held.find(ticket);
    if (it != r->held.end()) {
        r->load[i] -= it->second;
        r->held.erase(it);
    }
}

static int split(pa_router *r, uint64_t ticket, uint32_t &i, uint64_t &t)
{
    if (!r) return PA_ERR_INVALID;
    i = (uint32_t)(ticket & 0xffu);
    t = ticket >> 8;
    return i < r->servers.size() ? PA_OK : PA_ERR_NOT_FOUND;
}

int pa_router_poll(pa_router *r, uint64_t ticket, pa_result *out)
{
    uint32_t i;
    uint64_t t;
    int rc = split(r, ticket, i, t);
    if (rc != PA_OK) return rc;
    rc = pa_server_poll(r->servers[i], t, out);
    if (rc == PA_ERR_NOT_FOUND) forget(r, ticket, i);
    return rc;
}

int pa_router_wait(pa_router *r, uint64_t ticket, uint64_t timeout_ns, pa_result *out)
{
    uint32_t i;
    uint64_t t;
    int rc = split(r, ticket, i, t);
    if (rc != PA_OK) return rc;
    rc = pa_server_wait(r->servers[i], t, timeout_ns, out);
    if (rc == PA_ERR_NOT_FOUND) forget(r, ticket, i);
    return rc;
}

int pa_router_release(pa_router *r, uint64_t ticket)
{
    uint32_t i;
    uint64_t t;
    int rc = split(r, ticket, i, t);
    if (rc != PA_OK) return rc;
    rc = pa_server_release(r->servers[i], t);
    if (rc == PA_OK || rc == PA_ERR_NOT_FOUND) forget(r, ticket, i);
    return rc;
}

int pa_router_device_of(pa_router *r, uint64_t ticket, int32_t *device)
{
    uint32_t i;
    uint64_t t;
    const int rc = split(r, ticket, i, t);
    if (rc != PA_OK) return rc;
    if (!device) return PA_ERR_INVALID;
    *device = r->devices[i];
    return PA_OK;
}

int pa_router_stats_get(pa_router *r, uint32_t index, pa_server_stats *out)
{
    if (!r || !out || index > r->servers.size()) return PA_ERR_INVALID;
    if (index < r->servers.size()) return pa_server_stats_get(r->servers[index], out);
    pa_server_stats sum{};
    for (pa_server *s : r->servers) {
        pa_server_stats st;
        const int rc = pa_server_stats_get(s, &st);
        if (rc != PA_OK) return rc;
        sum.submitted += st.submitted;
        sum.completed += st.completed;
        sum.released += st.released;
        sum.expired += st.expired;
        sum.failed += st.failed;
        sum.batches += st.batches;
        sum.queued += st.queued;
        sum.running += st.running;
        sum.bytes_in_use += st.bytes_in_use;
        sum.budget_bytes += st.budget_bytes;
        sum.edges_done += st.edges_done;
    }
    *out = sum;
    return PA_OK;
}

uint32_t pa_router_size(const pa_router *r) { return r ? (uint32_t)r->servers.size() : 0; }

int pa_router_destroy(pa_router *r)
{
    if (!r) return PA_ERR_INVALID;
    int rc = PA_OK;
    for (pa_server *s : r->servers) {
        const int x = pa_server_destroy(s);
        if (x != PA_OK && rc == PA_OK) rc = x;
    }
    delete r;
    return rc;
}

}  // extern "C"
