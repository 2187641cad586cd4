// pa_batch.cu -- many independent graphs, and the start of every graph, by
// level launches.
//
// The north star's batching: instances of uneven size (n, d, p, seed, seed
// graph) share launches instead of one launch each, so the long dependency
// chains at the start of every graph run side by side and the launch and tail
// costs are paid once.  No reference counterpart (the reference generates one
// graph per process run, src/main.cu:105-116).
//
//  * Levels (pa_gen_core.cuh): level l of a graph covers nodes
//    [B_l, B_{l+1}), B_{l+1} = B_l + max(4096, B_l / 8).  The tiles of all
//    instances form one index space ordered by level and, within a level, by
//    instance.  A warp claims four tiles at a time from the launch's ticket and
//    maps a tile to (level, instance, tile of the instance) by two binary
//    searches over prefix tables.
//  * Every level that starts below 2^21 nodes is its own launch.  The launch
//    boundary is a barrier: when level l starts, everything below it is
//    complete, so copy reads below B_l need no check at all and only the reads
//    into level l itself (about 1/9 of them) wait on tile flags.  The remaining
//    levels run as one launch, in which a copy read above the launch's start
//    checks the completion count of its source's superblock (64 tiles; the
//    counts of a whole batch are L2-resident) before it reads.
//  * Each instance's tiles are claimed in increasing order by running warps, so
//    every instance is deadlock-free exactly as in the single-graph kernel.
//  * A warp keeps its current instance's arguments in shared memory; the slot
//    code is the single-graph kernel's (pa_gen_core.cuh).
#include <algorithm>
#include <cstring>
#include <vector>

#include "pa_gen_core.cuh"

namespace pa {
namespace gen {

std::vector<uint64_t> level_bounds(uint64_t u_first, uint64_t n, uint64_t n_tiles,
                                   uint64_t tile_nodes)
{
    std::vector<uint64_t> out{0};
    uint64_t B = u_first;
    while (out.back() < n_tiles) {
        B += std::max<uint64_t>(kLevelMinNodes, B >> kLevelShift);
        const uint64_t nb = B >= n ? n : B;
        uint64_t t = (nb - u_first + tile_nodes - 1) / tile_nodes;
        if (t > n_tiles) t = n_tiles;
        out.push_back(t);
    }
    return out;
}

uint32_t split_levels(const std::vector<uint64_t> &bounds, uint64_t u_first, uint64_t tile_nodes)
{
    uint32_t l = 0;
    while (l + 1 < bounds.size() && u_first + bounds[l] * tile_nodes < kSplitNodes) ++l;
    return l;
}

}  // namespace gen

namespace {

using namespace gen;

struct BatchArgs {
    const GenArgs *inst;                    // per-instance arguments (device)
    LevelTables tab;
    uint32_t count;
    uint32_t l_begin;                       // first level of this launch
    unsigned long long t_begin, t_end;      // global tiles of this launch
    unsigned long long *ticket;             // this launch's claim counter
    GenCtl *ctl;                            // shared status and counters
};

// Largest index i in [0, len) with a[i] <= x (a ascending, a[0] <= x).
__device__ __forceinline__ uint32_t last_le(const unsigned long long *a, uint32_t len,
                                            unsigned long long x)
{
    uint32_t lo = 0, hi = len;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(a + mid) <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Global tile T -> (instance, tile of the instance).
__device__ __forceinline__ void map_tile(const BatchArgs &b, unsigned long long T, uint32_t &inst,
                                         uint64_t &t)
{
    const uint32_t l = last_le(b.tab.lvl_base, b.tab.levels, T);
    const unsigned long long r = T - __ldg(b.tab.lvl_base + l);
    const unsigned long long *ib = b.tab.inst_base + (uint64_t)l * (b.count + 1);
    inst = last_le(ib, b.count, r);
    t = __ldg(b.tab.loc_start + (uint64_t)l * b.count + inst) + (r - __ldg(ib + inst));
}

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

    // The launch that starts at level 0 writes every instance's seed edges
    // (closed forms; nothing reads them back).
    if (b.l_begin == 0) {
        const uint32_t gw = blockIdx.x * (kThreads / 32) + warp;
        const uint32_t nw = gridDim.x * (kThreads / 32);
        for (uint32_t i = gw; i < b.count; i += nw) {
            const GenArgs *ai = b.inst + i;
            Id *Ei = reinterpret_cast<Id *>(ai->edges);
            const uint32_t di = ai->d, mode = ai->seed_mode;
            const uint64_t se = ai->seed_edges;
            for (uint64_t e = L.lane; e < se; e += 32) {
                uint64_t s, u;
                seed_edge(e, di, mode, s, u);
                st_pair(Ei + 2 * e, s, u);
            }
        }
    }

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
            map_tile(b, T, i, t);
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
                // everything below this launch's first level is complete
                water_node = (uint32_t)(a.u_first +
                                        (uint64_t)__ldg(b.tab.loc_start +
                                                        (uint64_t)b.l_begin * b.count + i) *
                                            a.tile_nodes);
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

int launch_levels(uint32_t id_bytes, uint32_t passes, const GenArgs *d_inst, const LevelTables &tabs,
                  uint32_t count, uint32_t l_begin, unsigned long long t_begin,
                  unsigned long long t_end, unsigned long long *d_ticket, GenCtl *ctl,
                  cudaStream_t s)
{
    BatchArgs b;
    b.inst = d_inst;
    b.tab = tabs;
    b.count = count;
    b.l_begin = l_begin;
    b.t_begin = t_begin;
    b.t_end = t_end;
    b.ticket = d_ticket;
    b.ctl = ctl;
    if (t_end <= t_begin && l_begin != 0) return PA_OK;
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

// Scratch layout of a batch.
struct BatchLayout {
    uint64_t table_off, lvl_off, ibase_off, lstart_off, ticket_off, inst_off, total;
    uint32_t levels, split;
    std::vector<uint64_t> flags_off, sb_off;
    std::vector<GenPlan> plans;
    std::vector<std::vector<uint64_t>> bounds;   // per instance: tile index at each level start
};

// One pass per tile by default: small tiles keep the dependency chains at the
// start of each graph short.
uint32_t batch_passes(const pa_params *prms) { return prms[0].tile_passes ? prms[0].tile_passes : 1u; }

int batch_layout(const pa_params *prms, uint32_t count, BatchLayout &L)
{
    if (!prms || count == 0) return PA_ERR_INVALID;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    const uint32_t P = batch_passes(prms);
    L.plans.resize(count);
    L.flags_off.resize(count);
    L.sb_off.resize(count);
    L.bounds.resize(count);
    uint64_t o = kCtlBytes;
    L.table_off = o;
    o += al((uint64_t)count * sizeof(GenArgs));
    for (uint32_t i = 0; i < count; ++i) {
        pa_params q = prms[i];
        q.tile_passes = P;   // one pass count per launch
        const int rc = make_plan(&q, &L.plans[i]);
        if (rc != PA_OK) return rc;
        if (prms[i].id_bits != prms[0].id_bits) return PA_ERR_INVALID;
        if (prms[i].n + L.plans[i].tile_nodes + 32 >= (1ull << 32)) return PA_ERR_NOT_SUPPORTED;
        if (prms[i].flags != 0) return PA_ERR_INVALID;
        if (L.plans[i].n_tiles >= (1ull << 32)) return PA_ERR_NOT_SUPPORTED;
        L.bounds[i] = level_bounds(L.plans[i].u_first, prms[i].n, L.plans[i].n_tiles,
                                   L.plans[i].tile_nodes);
    }
    L.levels = 1;
    L.split = 0;
    for (uint32_t i = 0; i < count; ++i) {
        L.levels = std::max<uint32_t>(L.levels, (uint32_t)L.bounds[i].size() - 1);
        L.split = std::max<uint32_t>(
            L.split, split_levels(L.bounds[i], L.plans[i].u_first, L.plans[i].tile_nodes));
    }
    if (L.levels > kMaxLevels) return PA_ERR_NOT_SUPPORTED;
    L.lvl_off = o;
    o += al(8ull * (L.levels + 1));
    L.ibase_off = o;
    o += al(8ull * L.levels * (count + 1));
    L.lstart_off = o;
    o += al(4ull * L.levels * count);
    L.ticket_off = o;
    o += al(8ull * (kMaxLevels + 1));
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
    }
    // level tables: global order is level by level, instance by instance
    const uint32_t Lv = L.levels;
    std::vector<unsigned long long> lvl(Lv + 1, 0), ibase((uint64_t)Lv * (count + 1), 0);
    std::vector<unsigned int> lstart((uint64_t)Lv * count, 0);
    for (uint32_t l = 0; l < Lv; ++l) {
        unsigned long long acc = 0;
        for (uint32_t i = 0; i < count; ++i) {
            const auto &bd = L.bounds[i];
            const uint64_t lo = l < bd.size() ? bd[l] : bd.back();
            const uint64_t hi = l + 1 < bd.size() ? bd[l + 1] : bd.back();
            ibase[(uint64_t)l * (count + 1) + i] = acc;
            lstart[(uint64_t)l * count + i] = (unsigned int)lo;
            acc += hi - lo;
        }
        ibase[(uint64_t)l * (count + 1) + count] = acc;
        lvl[l + 1] = lvl[l] + acc;
    }
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(scr, 0, kCtlBytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(scr + L.ticket_off, 0, L.total - L.ticket_off, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr + L.table_off, table.data(), count * sizeof(gen::GenArgs),
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr + L.lvl_off, lvl.data(), lvl.size() * 8ull, cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr + L.ibase_off, ibase.data(), ibase.size() * 8ull,
                            cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr + L.lstart_off, lstart.data(), lstart.size() * 4ull,
                            cudaMemcpyHostToDevice, s);
    // the host vectors are pageable: make sure the copies have read them
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_cuda_error(e);

    gen::LevelTables tabs;
    tabs.lvl_base = reinterpret_cast<const unsigned long long *>(scr + L.lvl_off);
    tabs.inst_base = reinterpret_cast<const unsigned long long *>(scr + L.ibase_off);
    tabs.loc_start = reinterpret_cast<const unsigned int *>(scr + L.lstart_off);
    tabs.levels = Lv;
    const gen::GenArgs *d_inst = reinterpret_cast<const gen::GenArgs *>(scr + L.table_off);
    unsigned long long *tickets = reinterpret_cast<unsigned long long *>(scr + L.ticket_off);
    GenCtl *ctl = reinterpret_cast<GenCtl *>(scr);
    const uint32_t id_bytes = prms[0].id_bits / 8;
    // one launch per early level, then the rest in one launch
    const uint32_t split = std::min(L.split, Lv);
    for (uint32_t l = 0; l < split; ++l) {
        rc = gen::launch_levels(id_bytes, P, d_inst, tabs, count, l, lvl[l], lvl[l + 1], tickets + l,
                                ctl, s);
        if (rc != PA_OK) return rc;
    }
    if (split < Lv || split == 0)
        rc = gen::launch_levels(id_bytes, P, d_inst, tabs, count, split, lvl[split], lvl[Lv],
                                tickets + split, ctl, s);
    return rc;
}

}  // extern "C"
