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

#include "pa_batch.h"

// Resident start-kernel blocks per SM of a batch launch (a start_min_blocks
// variant: 4, 5 or 6).
#ifndef PA_BATCH_START_BLOCKS
#define PA_BATCH_START_BLOCKS gen::kStartMinBlocks
#endif

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
    uint32_t claim;                         // tiles per claim
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
        const unsigned long long T0 = b.t_begin + chunk * b.claim;
        if (T0 >= b.t_end) break;
        for (uint32_t c = 0; c < b.claim && ok; ++c) {
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
    const unsigned long long chunks = (b.t_end - b.t_begin + b.claim - 1) / b.claim;
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
                unsigned long long *d_ticket, GenCtl *ctl, uint32_t claim_tiles, cudaStream_t s)
{
    BatchArgs b;
    b.inst = d_inst;
    b.tab = tabs;
    b.count = count;
    b.t_begin = t_begin;
    b.t_end = t_end;
    b.ticket = d_ticket;
    b.ctl = ctl;
    b.claim = claim_tiles ? claim_tiles : 1u;
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

// bounds[i]: unit bounds of instance i's levels (level_bounds).  Global order:
// level by level, instance by instance.
void build_levels(const std::vector<std::vector<uint64_t>> &bounds, BatchLevels &H)
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

gen::LevelTables device_tables(const BatchLevels &H, unsigned char *scr)
{
    gen::LevelTables t;
    t.lvl_base = reinterpret_cast<const unsigned long long *>(scr + H.lvl_off);
    t.inst_base = reinterpret_cast<const unsigned long long *>(scr + H.ibase_off);
    t.loc_start = reinterpret_cast<const unsigned long long *>(scr + H.lstart_off);
    t.levels = H.levels;
    return t;
}

}  // namespace

int batch_prepare(const pa_params *prms, uint32_t count, BatchJob &J)
{
    if (!prms || count == 0) return PA_ERR_INVALID;
    auto al = [](uint64_t x) { return (x + 255) & ~255ull; };
    // one pass per tile by default: small tiles keep the dependency chains short
    const uint32_t P = prms[0].tile_passes ? prms[0].tile_passes : 1u;
    if (P != 1 && P != 2 && P != 4) return PA_ERR_NOT_SUPPORTED;
    J.count = count;
    J.passes = P;
    J.id_bytes = prms[0].id_bits / 8;
    J.claim_tiles = prms[0].claim_tiles ? prms[0].claim_tiles : kClaimTilesAuto;
    J.plans.assign(count, GenPlan{});
    J.max_start_pairs = 0;
    J.flags_off.assign(count, 0);
    J.sb_off.assign(count, 0);
    std::vector<std::vector<uint64_t>> sb(count), tb(count);
    for (uint32_t i = 0; i < count; ++i) {
        pa_params q = prms[i];
        q.tile_passes = P;   // one pass count per launch
        const int rc = make_plan(&q, &J.plans[i]);
        if (rc != PA_OK) return rc;
        const GenPlan &p = J.plans[i];
        if (p.slots || p.wide) return PA_ERR_NOT_SUPPORTED;
        if (prms[i].id_bits != prms[0].id_bits) return PA_ERR_INVALID;
        if (prms[i].n + p.tile_nodes + 32 >= (1ull << 32)) return PA_ERR_NOT_SUPPORTED;
        if (prms[i].flags != 0) return PA_ERR_INVALID;
        sb[i] = level_bounds(p.u_first, p.u_first, p.u_split, (uint64_t)kStartPasses * p.groups);
        tb[i] = level_bounds(p.u_first, p.u_split, prms[i].n, p.tile_nodes);
        J.max_start_pairs = std::max<uint64_t>(J.max_start_pairs, (p.u_split - p.u_first) * prms[i].d);
    }
    build_levels(sb, J.start);
    build_levels(tb, J.tail);
    if (J.start.levels > kMaxLevels || J.tail.levels > kMaxLevels) return PA_ERR_NOT_SUPPORTED;
    // scratch: control block | image (GenArgs table, level tables) | tickets, flags, counts
    uint64_t o = kCtlBytes;
    J.image_off = o;
    J.table_off = o;
    o += al((uint64_t)count * sizeof(gen::GenArgs));
    for (BatchLevels *H : {&J.start, &J.tail}) {
        H->lvl_off = o;
        o += al(8ull * H->lvl.size());
        H->ibase_off = o;
        o += al(8ull * H->ibase.size());
        H->lstart_off = o;
        o += al(8ull * H->lstart.size());
    }
    J.image_bytes = o - J.image_off;
    J.ticket_off = o;
    o += 128ull * (kStartCounters + 2);   // start counters, tail counter
    for (uint32_t i = 0; i < count; ++i) {
        J.flags_off[i] = o;
        o += al(4 * J.plans[i].n_tiles);
        J.sb_off[i] = o;
        o += al(4 * J.plans[i].n_sb);
    }
    J.scratch_bytes = o;
    return PA_OK;
}

int batch_bind(BatchJob &J, const pa_params *prms, void *const *d_edges, const uint64_t *edges_bytes,
               void *d_scratch, unsigned char *image)
{
    if (!d_edges || !edges_bytes || !d_scratch || !image) return PA_ERR_INVALID;
    if (reinterpret_cast<uintptr_t>(d_scratch) & 15u) return PA_ERR_INVALID;
    unsigned char *scr = (unsigned char *)d_scratch;
    gen::GenArgs *table = reinterpret_cast<gen::GenArgs *>(image + (J.table_off - J.image_off));
    for (uint32_t i = 0; i < J.count; ++i) {
        const GenPlan &p = J.plans[i];
        if (!d_edges[i] || (reinterpret_cast<uintptr_t>(d_edges[i]) & 15u)) return PA_ERR_INVALID;
        if (edges_bytes[i] < p.edges_bytes) return PA_ERR_CAPACITY;
        gen::GenArgs a;
        std::memset(&a, 0, sizeof(a));
        a.edges = d_edges[i];
        a.ctl = reinterpret_cast<GenCtl *>(scr);
        a.reps = reinterpret_cast<GenRep *>(scr + kRepOffset);
        a.flags = reinterpret_cast<uint32_t *>(scr + J.flags_off[i]);
        a.sbcnt = reinterpret_cast<uint32_t *>(scr + J.sb_off[i]);
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
        a.claim_tiles = J.claim_tiles;
        a.model = p.model;

        std::memcpy(table + i, &a, sizeof(a));
        if (i == 0) J.first = a;
    }
    for (const BatchLevels *H : {&J.start, &J.tail}) {
        std::memcpy(image + (H->lvl_off - J.image_off), H->lvl.data(), H->lvl.size() * 8ull);
        std::memcpy(image + (H->ibase_off - J.image_off), H->ibase.data(), H->ibase.size() * 8ull);
        std::memcpy(image + (H->lstart_off - J.image_off), H->lstart.data(), H->lstart.size() * 8ull);
    }
    return PA_OK;
}

int batch_enqueue(const BatchJob &J, void *d_scratch, const void *image, cudaStream_t s)
{
    unsigned char *scr = (unsigned char *)d_scratch;
    cudaError_t e = cudaMemsetAsync(scr, 0, kCtlBytes, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(scr + J.ticket_off, 0, J.scratch_bytes - J.ticket_off, s);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(scr + J.image_off, image, J.image_bytes, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return set_cuda_error(e);
    const gen::GenArgs *d_inst = reinterpret_cast<const gen::GenArgs *>(scr + J.table_off);
    // start-kernel counters: kStartCounters lines of 128 bytes; then the tail's
    unsigned long long *tickets = reinterpret_cast<unsigned long long *>(scr + J.ticket_off);
    unsigned long long *tail_ticket = tickets + 16 * kStartCounters;
    GenCtl *ctl = reinterpret_cast<GenCtl *>(scr);
    int rc = gen::fill_start(J.id_bytes, d_inst, J.count, J.max_start_pairs, s);
    if (rc != PA_OK) return rc;
    gen::StartArgs sa;
    std::memset(&sa, 0, sizeof(sa));
    sa.inst = d_inst;
    sa.tab = device_tables(J.start, scr);
    sa.count = J.count;
    sa.write_seeds = 1;
    sa.t_end = J.start.lvl[J.start.levels];
    sa.ticket = tickets;
    sa.ctl = ctl;
    if (J.count == 1) sa.one = J.first;
    rc = gen::launch_start(J.id_bytes, sa, 0, s, false, PA_BATCH_START_BLOCKS);
    if (rc != PA_OK) return rc;
    return gen::launch_tail(J.id_bytes, J.passes, d_inst, device_tables(J.tail, scr), J.count,
                            J.tail.lvl[0], J.tail.lvl[J.tail.levels], tail_ticket, ctl,
                            J.claim_tiles, s);
}

}  // namespace pa

using namespace pa;

extern "C" {

int pa_batch_scratch_bytes(const pa_params *prms, uint32_t count, uint64_t *bytes)
{
    if (!bytes) return PA_ERR_INVALID;
    BatchJob J;
    const int rc = batch_prepare(prms, count, J);
    if (rc != PA_OK) return rc;
    *bytes = J.scratch_bytes;
    return PA_OK;
}

int pa_batch_generate(const pa_params *prms, uint32_t count, void *const *d_edges,
                      const uint64_t *edges_bytes, void *d_scratch, uint64_t scratch_bytes,
                      void *stream)
{
    BatchJob J;
    int rc = batch_prepare(prms, count, J);
    if (rc != PA_OK) return rc;
    if (scratch_bytes < J.scratch_bytes) return PA_ERR_CAPACITY;
    std::vector<unsigned char> image(J.image_bytes);
    rc = batch_bind(J, prms, d_edges, edges_bytes, d_scratch, image.data());
    if (rc != PA_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    rc = batch_enqueue(J, d_scratch, image.data(), s);
    if (rc != PA_OK) return rc;
    // the image is pageable host memory: make sure the copy has read it
    const cudaError_t e = cudaStreamSynchronize(s);
    return e == cudaSuccess ? PA_OK : set_cuda_error(e);
}

}  // extern "C"
