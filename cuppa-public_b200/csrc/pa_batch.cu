// pa_batch.cu -- many independent graphs in shared launches.
//
// Instances of uneven size (n, d, p, seed, seed graph) share launches instead of
// one launch each, so the dependency chains at the start of every graph run
// side by side and the launch and tail costs are paid once.  No reference
// counterpart (the reference generates one graph per process run,
// src/main.cu:105-116).
//
//  * One fill launch sets the start region of every instance to all-ones.
//  * One start-kernel launch (pa_start.cu) generates every instance's start
//    region, with slot-granular waits, the warp passes of all instances in
//    level order (pa_gen_core.cuh).
//  * One tail launch of the batch kernel below generates the rest of the
//    instances that are larger than their start region, tiles in level order.
//    Everything below an instance's start_end is complete when it starts, so
//    only copy reads at or above it check the completion count of the source's
//    superblock (64 tiles; the counts of a whole batch are L2-resident) and, if
//    that is not complete, poll the source tile's flag.
//  * A warp keeps its current instance's arguments in shared memory; the slot
//    code is the single-graph kernel's (pa_gen_core.cuh).
#include <algorithm>
#include <cstring>
#include <vector>

#include "pa_gen_core.cuh"

namespace pa {
namespace gen {

std::vector<uint64_t> level_bounds(uint64_t u_first, uint64_t lo, uint64_t n_end,
                                   uint64_t unit_nodes)
{
    auto units = [&](uint64_t node) { return (node - u_first + unit_nodes - 1) / unit_nodes; };
    const uint64_t n_units = units(n_end);
    std::vector<uint64_t> out{units(lo)};
    uint64_t B = lo;
    while (out.back() < n_units) {
        B += std::max<uint64_t>(kLevelMinNodes, B >> kLevelShift);
        out.push_back(std::min(units(std::min(B, n_end)), n_units));
    }
    return out;
}

}  // namespace gen

namespace {

using namespace gen;

struct BatchArgs {
    const GenArgs *inst;                    // per-instance arguments (device)
    LevelTables tab;
    uint32_t count;
    unsigned long long t_begin, t_end;      // global tiles of this launch
    unsigned long long *ticket;             // this launch's claim counter
    GenCtl *ctl;                            // shared status and counters
};

template <typename Id, int P>
__global__ void __launch_bounds__(kThreads, kMinBlocks) batch_kernel(const BatchArgs b)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ GenArgs s_args[kThreads / 32];
    const uint32_t warp = threadIdx.x >> 5;
    Id *tilebuf = reinterpret_cast<Id *>(smem_raw) + warp * (32u * P);
    GenArgs &a = s_args[warp];

    Lane L;
    L.lane = threadIdx.x & 31u;
    L.lt = lanemask_lt();
    L.le = L.lt | (1u << L.lane);
    uint32_t cur = 0xffffffffu;
    uint32_t water_node = 0;

    uint32_t n_retry = 0, n_wait = 0, n_done = 0, n_pend = 0, n_poll = 0;
    bool ok = true;
    while (ok) {
        unsigned long long chunk = 0;
        if (L.lane == 0) chunk = atomicAdd(b.ticket, 1ull);
        chunk = __shfl_sync(kFull, chunk, 0);
        const unsigned long long T0 = b.t_begin + chunk * kClaimTiles;
        if (T0 >= b.t_end) break;
        for (uint32_t c = 0; c < kClaimTiles && ok; ++c) {
            const unsigned long long T = T0 + c;
            if (T >= b.t_end) break;
            uint32_t i;
            uint64_t t;
            map_unit(b.tab, b.count, T, i, t);
            if (i != cur) {
                // copy the instance's arguments into this warp's shared slot
                __syncwarp();
                const uint32_t *src = reinterpret_cast<const uint32_t *>(b.inst + i);
                uint32_t *dst = reinterpret_cast<uint32_t *>(&a);
                for (uint32_t w = L.lane; w < sizeof(GenArgs) / 4; w += 32) dst[w] = __ldg(src + w);
                __syncwarp();
                cur = i;
                L.g = L.lane / a.d;
                L.slot = L.lane - L.g * a.d;
                L.used = L.lane < a.groups * a.d;
                L.gmask = L.used ? (a.d == 32 ? kFull : (((1u << a.d) - 1u) << (L.g * a.d))) : 0u;
                // everything below the instance's start region end is complete
                water_node = (uint32_t)a.start_end;
            }
            Id *E = reinterpret_cast<Id *>(a.edges);
            Slot<uint32_t> S[P];
            uint32_t wn = water_node;
            stage1<Id, uint32_t, P, true>(S, t, a, E, L, wn, n_pend);
            ok = stage2<Id, uint32_t, P, true>(S, t, a, E, tilebuf, L, wn, n_retry, n_wait,
                                               n_pend, n_poll);
            if (ok) ++n_done;
        }
    }

#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n_retry += __shfl_down_sync(kFull, n_retry, o);
        n_pend += __shfl_down_sync(kFull, n_pend, o);
        n_poll += __shfl_down_sync(kFull, n_poll, o);
    }
    if (L.lane == 0) {
        if (n_pend) atomicAdd(&b.ctl->pending_reads, (unsigned long long)n_pend);
        if (n_poll) atomicAdd(&b.ctl->pending_polls, (unsigned long long)n_poll);
        if (n_retry) atomicAdd(&b.ctl->retries, (unsigned long long)n_retry);
        if (n_wait) atomicAdd(&b.ctl->waits, (unsigned long long)n_wait);
        if (n_done) atomicAdd(&b.ctl->tiles, (unsigned long long)n_done);
    }
}

template <typename Id, int P>
int launch_batch(const BatchArgs &b, cudaStream_t s)
{
    auto kern = batch_kernel<Id, P>;
    const size_t smem = (size_t)(kThreads / 32) * 32 * P * sizeof(Id);
    int dev = 0, sms = 0, per_sm = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)kThreads, smem);
    if (e != cudaSuccess) return set_cuda_error(e);
    // no more warps than chunks to claim
    const unsigned long long chunks = (b.t_end - b.t_begin + kClaimTiles - 1) / kClaimTiles;
    unsigned long long blocks = (unsigned long long)sms * (per_sm > 0 ? per_sm : 1);
    const unsigned long long need = (chunks + kThreads / 32 - 1) / (kThreads / 32);
    if (need < blocks) blocks = need > 0 ? need : 1;
    kern<<<(unsigned)blocks, kThreads, smem, s>>>(b);
    e = cudaGetLastError();
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

}  // namespace

namespace gen {

int launch_tail(uint32_t id_bytes, uint32_t passes, const GenArgs *d_inst, const LevelTables &tabs,
                uint32_t count, unsigned long long t_begin, unsigned long long t_end,
                unsigned long long *d_ticket, GenCtl *ctl, cudaStream_t s)
{
    BatchArgs b;
    b.inst = d_inst;
    b.tab = tabs;
    b.count = count;
    b.t_begin = t_begin;
    b.t_end = t_end;
    b.ticket = d_ticket;
    b.ctl = ctl;
    if (t_end <= t_begin) return PA_OK;
    if (id_bytes == 8) {
        switch (passes) {
        case 1: return launch_batch<int64_t, 1>(b, s);
        case 2: return launch_batch<int64_t, 2>(b, s);
        case 4: return launch_batch<int64_t, 4>(b, s);
        }
    } else {
        switch (passes) {
        case 1: return launch_batch<int32_t, 1>(b, s);
        case 2: return launch_batch<int32_t, 2>(b, s);
        case 4: return launch_batch<int32_t, 4>(b, s);
        }
    }
    return PA_ERR_NOT_SUPPORTED;
}

}  // namespace gen

namespace {

// Level tables of one launch over a set of instances (host side).
struct HostLevels {
    uint32_t levels = 0;
    std::vector<unsigned long long> lvl, ibase, lstart;
    uint64_t lvl_off = 0, ibase_off = 0, lstart_off = 0;   // device copies in the scratch
};

// bounds[i]: unit bounds of instance i's levels (level_bounds).  Global order:
// level by level, instance by instance.
void build_levels(const std::vector<std::vector<uint64_t>> &bounds, HostLevels &H)
{
    const uint32_t count = (uint32_t)bounds.size();
    H.levels = 1;
    for (const auto &bd : bounds) H.levels = std::max<uint32_t>(H.levels, (uint32_t)bd.size() - 1);
    const uint32_t Lv = H.levels;
    H.lvl.assign(Lv + 1, 0);
    H.ibase.assign((uint64_t)Lv * (count + 1), 0);
    H.lstart.assign((uint64_t)Lv * count, 0);
    for (uint32_t l = 0; l < Lv; ++l) {
        unsigned long long acc = 0;
        for (uint32_t i = 0; i < count; ++i) {
            const auto &bd = bounds[i];
            const uint64_t lo = l < bd.size() ? bd[l] : bd.back();
            const uint64_t hi = l + 1 < bd.size() ? bd[l + 1] : bd.back();
            H.ibase[(uint64_t)l * (count + 1) + i] = acc;
            H.lstart[(uint64_t)l * count + i] = lo;
            acc += hi - lo;
        }
        H.ibase[(uint64_t)l * (count + 1) + count] = acc;
        H.lvl[l + 1] = H.lvl[l] + acc;
    }
}

// Scratch layout of a batch.
struct BatchLayout {
    uint64_t table_off, ticket_off, inst_off, total;
    std::vector<uint64_t> flags_off, sb_off;
    std::vector<GenPlan> plans;
    HostLevels start, tail;
    uint64_t max_start_pairs;
};

// One pass per tile by default: small tiles keep the dependency chains short.
uint32_t batch_passes(const pa_params *prms) { return prms[0].tile_passes ? prms[0].tile_passes : 1u; }

int batch_layout(const pa_params *prms, uint32_t count, BatchLayout &L)
{
    if (!prms || count == 0) return PA_ERR_INVALID;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    const uint32_t P = batch_passes(prms);
    L.plans.resize(count);
    L.flags_off.resize(count);
    L.sb_off.resize(count);
    L.max_start_pairs = 0;
    std::vector<std::vector<uint64_t>> sb(count), tb(count);
    for (uint32_t i = 0; i < count; ++i) {
        pa_params q = prms[i];
        q.tile_passes = P;   // one pass count per launch
        const int rc = make_plan(&q, &L.plans[i]);
        if (rc != PA_OK) return rc;
        const GenPlan &p = L.plans[i];
        if (prms[i].id_bits != prms[0].id_bits) return PA_ERR_INVALID;
        if (prms[i].n + p.tile_nodes + 32 >= (1ull << 32)) return PA_ERR_NOT_SUPPORTED;
        if (prms[i].flags != 0) return PA_ERR_INVALID;
        sb[i] = level_bounds(p.u_first, p.u_first, p.u_split, (uint64_t)kStartPasses * p.groups);
        tb[i] = level_bounds(p.u_first, p.u_split, prms[i].n, p.tile_nodes);
        L.max_start_pairs = std::max<uint64_t>(L.max_start_pairs, (p.u_split - p.u_first) * prms[i].d);
    }
    build_levels(sb, L.start);
    build_levels(tb, L.tail);
    if (L.start.levels > kMaxLevels || L.tail.levels > kMaxLevels) return PA_ERR_NOT_SUPPORTED;
    uint64_t o = kCtlBytes;
    L.table_off = o;
    o += al((uint64_t)count * sizeof(GenArgs));
    for (HostLevels *H : {&L.start, &L.tail}) {
        H->lvl_off = o;
        o += al(8ull * H->lvl.size());
        H->ibase_off = o;
        o += al(8ull * H->ibase.size());
        H->lstart_off = o;
        o += al(8ull * H->lstart.size());
    }
    L.ticket_off = o;
    o += 256;
    L.inst_off = o;
    for (uint32_t i = 0; i < count; ++i) {
        L.flags_off[i] = o;
        o += al(4 * L.plans[i].n_tiles);
        L.sb_off[i] = o;
        o += al(4 * L.plans[i].n_sb);
    }
    L.total = o;
    return PA_OK;
}

gen::LevelTables device_tables(const HostLevels &H, unsigned char *scr)
{
    gen::LevelTables t;
    t.lvl_base = reinterpret_cast<const unsigned long long *>(scr + H.lvl_off);
    t.inst_base = reinterpret_cast<const unsigned long long *>(scr + H.ibase_off);
    t.loc_start = reinterpret_cast<const unsigned long long *>(scr + H.lstart_off);
    t.levels = H.levels;
    return t;
}

}  // namespace
}  // namespace pa

using namespace pa;

extern "C" {

int pa_batch_scratch_bytes(const pa_params *prms, uint32_t count, uint64_t *bytes)
{
    if (!bytes) return PA_ERR_INVALID;
    BatchLayout L;
    const int rc = batch_layout(prms, count, L);
    if (rc != PA_OK) return rc;
    *bytes = L.total;
    return PA_OK;
}

int pa_batch_generate(const pa_params *prms, uint32_t count, void *const *d_edges,
                      const uint64_t *edges_bytes, void *d_scratch, uint64_t scratch_bytes,
                      void *stream)
{
    BatchLayout L;
    int rc = batch_layout(prms, count, L);
    if (rc != PA_OK) return rc;
    if (!d_edges || !edges_bytes || !d_scratch) return PA_ERR_INVALID;
    if (scratch_bytes < L.total) return PA_ERR_CAPACITY;
    if (reinterpret_cast<uintptr_t>(d_scratch) & 15u) return PA_ERR_INVALID;
    const uint32_t P = batch_passes(prms);
    if (P != 1 && P != 2 && P != 4) return PA_ERR_NOT_SUPPORTED;
    unsigned char *scr = (unsigned char *)d_scratch;
    std::vector<gen::GenArgs> table(count);
    for (uint32_t i = 0; i < count; ++i) {
        const GenPlan &p = L.plans[i];
        if (!d_edges[i] || (reinterpret_cast<uintptr_t>(d_edges[i]) & 15u)) return PA_ERR_INVALID;
        if (edges_bytes[i] < p.edges_bytes) return PA_ERR_CAPACITY;
        gen::GenArgs &a = table[i];
        std::memset(&a, 0, sizeof(a));
        a.edges = d_edges[i];
        a.ctl = reinterpret_cast<GenCtl *>(scr);
        a.reps = reinterpret_cast<GenRep *>(scr + kRepOffset);
        a.flags = reinterpret_cast<uint32_t *>(scr + L.flags_off[i]);
        a.sbcnt = reinterpret_cast<uint32_t *>(scr + L.sb_off[i]);
        a.n_sb = p.n_sb;
        a.sb_nodes = (uint64_t)kSbTiles * p.tile_nodes;
        a.n = prms[i].n;
        a.u_first = p.u_first;
        a.n_tiles = p.n_tiles;
        a.seed_edges = p.seed_edges;
        a.slot_off = (int64_t)p.seed_edges - (int64_t)(p.u_first * prms[i].d);
        a.pth = p.pth;
        a.spin_limit_ns = p.spin_limit_ns;
        a.key0 = (uint32_t)prms[i].seed;
        a.key1 = (uint32_t)(prms[i].seed >> 32);
        a.d = prms[i].d;
        a.groups = p.groups;
        a.tile_nodes = p.tile_nodes;
        a.seed_mode = prms[i].seed_mode;
        a.max_sleep_ns = 4096;   // many warps wait at once: keep their polls sparse
        a.window_shift = 63;
        a.min_window = 0;
        a.start_end = p.u_split;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(scr, 0, kCtlBytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(scr + L.ticket_off, 0, L.total - L.ticket_off, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr + L.table_off, table.data(), count * sizeof(gen::GenArgs),
                            cudaMemcpyHostToDevice, s);
    for (const HostLevels *H : {&L.start, &L.tail}) {
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(scr + H->lvl_off, H->lvl.data(), H->lvl.size() * 8ull,
                                cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(scr + H->ibase_off, H->ibase.data(), H->ibase.size() * 8ull,
                                cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(scr + H->lstart_off, H->lstart.data(), H->lstart.size() * 8ull,
                                cudaMemcpyHostToDevice, s);
    }
    // the host vectors are pageable: make sure the copies have read them
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_cuda_error(e);

    const gen::GenArgs *d_inst = reinterpret_cast<const gen::GenArgs *>(scr + L.table_off);
    unsigned long long *tickets = reinterpret_cast<unsigned long long *>(scr + L.ticket_off);
    GenCtl *ctl = reinterpret_cast<GenCtl *>(scr);
    const uint32_t id_bytes = prms[0].id_bits / 8;
    rc = gen::fill_start(id_bytes, d_inst, count, L.max_start_pairs, s);
    if (rc != PA_OK) return rc;
    gen::StartArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    sa.inst = d_inst;
    sa.tab = device_tables(L.start, scr);
    sa.count = count;
    sa.write_seeds = 1;
    sa.t_end = L.start.lvl[L.start.levels];
    sa.ticket = tickets;
    sa.ctl = ctl;
    if (count == 1) sa.one = table[0];
    rc = gen::launch_start(id_bytes, sa, 0, s);
    if (rc != PA_OK) return rc;
    return gen::launch_tail(id_bytes, P, d_inst, device_tables(L.tail, scr), count,
                            L.tail.lvl[0], L.tail.lvl[L.tail.levels], tickets + 1, ctl, s);
}

}  // extern "C"
