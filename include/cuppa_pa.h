/*
 * cuppa_pa.h -- C ABI of the B200 copy-model preferential-attachment generator.
 *
 * Plain C, plain pointers and sizes; device buffers are CUDA device pointers and
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 * No call prints, exits, resets the device or frees memory it did not allocate.
 * Every call returns a pa_status (0 = PA_OK).
 *
 * Reference interfaces replaced (paths relative to the cuPPA-Public tree):
 *   class cuPPA(NodeType n, EdgeIndexType m, double p)     src/PA/cuPPA/cuPPA.cuh:84-105
 *     .generateGraph(conf)          src/PA/cuPPA/cuPPA_1.cu:9-254   -> pa_generate
 *     .generateGraphAdaptive(conf)  src/PA/cuPPA/cuPPA_2.cu:9-241   -> pa_generate
 *                                   (the persistent launch needs no stage tuning)
 *     .printDegreeDistribution      src/PA/cuPPA/cuPPA.cu:103-165   -> pa_degrees,
 *                                   pa_degree_distribution
 *   PAHelper::writeGraphToDisk      src/PA/SPA/PAHelper.hpp:163-177 -> pa_write_edges_text
 *   runner flags -n -x -a -b -t -s  src/main.cu:188-213             -> pa_params fields
 */
#ifndef CUPPA_PA_H_
#define CUPPA_PA_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PA_ABI_VERSION 1

typedef enum pa_status {
    PA_OK = 0,
    PA_ERR_INVALID = 1,       /* a parameter is out of range or a pointer is NULL      */
    PA_ERR_OOM = 2,           /* a device allocation made by the library failed        */
    PA_ERR_SPIN_TIMEOUT = 3,  /* a device-side wait hit its limit (pa_params.spin_limit_ns) */
    PA_ERR_CUDA = 4,          /* a CUDA runtime call failed; see pa_last_cuda_error()  */
    PA_ERR_CAPACITY = 5,      /* a caller buffer is smaller than the call needs         */
    PA_ERR_NOT_SUPPORTED = 6, /* valid request this build does not handle               */
    PA_ERR_BUSY = 7,          /* server: admission refused for now (retry later)        */
    PA_ERR_NOT_FOUND = 8,     /* server: unknown or already released ticket             */
    PA_ERR_IO = 9             /* a file could not be opened or written, or a sink failed */
} pa_status;

/* Seed graph on nodes 0..d.
 * STAR_REF: slots G[i][*] = i for i < d and G[d][j] = j -- the reference's seed
 *           (src/PA/SPA/SerialCopyModel3.cpp:38-49, src/PA/cuPPA/cuPPA_RRP.cu:57-73);
 *           its canonical edges are (d, j), j < d.
 * CLIQUE:   nodes 0..d form K_{d+1}; G[v][*] = v's neighbours ascending. */
enum { PA_SEED_STAR_REF = 0, PA_SEED_CLIQUE = 1 };

/* Edge layouts.
 * PAIRS: (src, dst) id pairs.  The first pa_seed_edge_count() pairs are the seed
 *        rows' canonical edges (src > dst, sorted); then node u = d+1..n-1 owns the
 *        d pairs at [S + (u-d-1)*d, S + (u-d)*d) in slot (generation) order.  Every
 *        pair is an edge with src > dst.  This is the reference's G[N][M] slot array
 *        (src/PA/cuPPA/cuPPA_1.cu:54) carried as an edge list. */
/* SLOTS: the targets alone -- node u = d+1..n-1 owns ids [(u-d-1)*d, (u-d)*d) in
 *        slot order, the seed rows are implied by seed_mode and not stored.  Half
 *        the bytes of PAIRS, so a graph twice as large stays resident; read it out
 *        with pa_write_edges / pa_stream_edges, which emit the PAIRS order.  The
 *        whole graph is generated by the start kernel, so n - d - 1 <= 2^31 and
 *        start_nodes must be 0 (auto); other entry points that take an edge list
 *        (CSR, canonicalize, batch, server) return PA_ERR_NOT_SUPPORTED. */
enum { PA_LAYOUT_PAIRS = 0, PA_LAYOUT_SLOTS = 1 };

/* pa_params.flags.  TEST_WITHHOLD_FIRST_TILE is for tests of the wait limit:
 * the generator never publishes its first tile, so every wait on that tile runs
 * into spin_limit_ns and the call reports PA_ERR_SPIN_TIMEOUT. */
#define PA_FLAG_TEST_WITHHOLD_FIRST_TILE 0x80000000u
/* PREFILLED: the caller has already set d_edges' generation region to
 * all-ones with pa_fill (on any stream, ordered before the generation), so the
 * generation skips its own fill. */
#define PA_FLAG_PREFILLED 0x1u
/* (with a start kernel, its first warp pass is withheld instead: the first
 *  nodes' slots are never written, with the same outcome) */

typedef struct pa_params {
    uint64_t n;             /* nodes                        (-n/--n1; cuPPA(n, ...))      */
    uint32_t d;             /* edges per new node, 1..32767 (-x/--x1; M; the reference's int16
                               EdgeIndexType, src/Common/DataTypes.h:11-28)               */
    uint32_t id_bits;       /* 32 or 64: width of each stored id                           */
    double p;               /* probability of a direct pick (-a/--alpha), 0 <= p <= 1      */
    uint64_t seed;          /* Philox key                                                 */
    uint32_t seed_mode;     /* PA_SEED_*                                                  */
    uint32_t layout;        /* PA_LAYOUT_*                                                */
    uint32_t blocks;        /* -b: CTAs of the persistent launch; 0 = one wave of the GPU */
    uint32_t threads;       /* -t: threads per CTA (multiple of 32, <= 1024); 0 = auto    */
    uint32_t tile_passes;   /* warp passes per claimed tile (1, 2, 4 or 8); 0 = auto      */
    uint32_t flags;         /* PA_FLAG_* (0 for normal use)                               */
    uint64_t spin_limit_ns; /* limit of any single device wait; 0 = 2 s                    */
    uint64_t start_nodes;   /* nodes after the seed generated by the start kernel (slot-
                               granular waits); rounded up to whole superblocks of the
                               persistent launch, at most 2^31.  0 = auto (as many as
                               that allows), PA_START_NONE = none                        */
    uint32_t claim_tiles;   /* tiles claimed per work-counter atomic (1..64); 0 = auto   */
    uint32_t model;         /* PA_MODEL_*: the attachment rule                            */
} pa_params;

/* pa_params.model.
 * PA_MODEL_COPY -- the copy model of -A cuppa / -A scm: each slot links to a
 *   uniform earlier node with probability p, else copies a uniform slot of it.
 * PA_MODEL_BA -- the repeated-nodes Barabasi-Albert model of -A sba
 *   (src/PA/SPA/SerialBA.cpp:68-186): each slot picks a uniform endpoint of all
 *   earlier edges, i.e. a node with probability proportional to its degree.
 *   Requires seed_mode PA_SEED_STAR_REF (the reference's initial graph); p is
 *   ignored.  The draw of slot i of node u at retry r: x = w1:w0 of
 *   Philox(ctr = (u_lo, u_hi, i, r)), R = floor(x * 2du / 2^64) indexes the
 *   endpoint list (2d^2 seed entries, then (target_j, w) per earlier node w),
 *   so v = floor(x * u / 2^64), q = R mod 2d: q odd -> v itself, q even ->
 *   v's slot q/2.  Same output layout, duplicate retries and slot order. */
#define PA_MODEL_COPY 0u
#define PA_MODEL_BA 1u

/* pa_params.start_nodes: no start kernel (the persistent launch does every node). */
#define PA_START_NONE UINT64_MAX

/* Statistics and device-side status of one generation. */
typedef struct pa_stats {
    uint64_t retries;       /* draws rejected as duplicates                               */
    uint64_t waits;         /* resolve iterations that waited on an unfinished tile       */
    uint64_t tiles;         /* tiles completed                                            */
    uint64_t pending_reads; /* copy reads whose source tile was not yet known complete    */
    uint64_t pending_polls; /* completion-flag polls that found the source tile unfinished */
    uint32_t status;        /* pa_status seen on the device (PA_OK or PA_ERR_SPIN_TIMEOUT) */
    uint32_t reserved;
} pa_stats;

/* ---- sizes -------------------------------------------------------------- */
/* Fills *out with defaults for every field; the caller then sets n, d, p, seed. */
int pa_params_init(pa_params *out);
/* Validate a parameter block (PA_OK or PA_ERR_INVALID / PA_ERR_NOT_SUPPORTED). */
int pa_params_check(const pa_params *prm);
uint64_t pa_seed_edge_count(uint32_t d, uint32_t seed_mode);
/* Number of edges (pairs) the generator writes. */
uint64_t pa_edge_count(const pa_params *prm);
/* Bytes of the edge buffer and of the scratch buffer pa_generate needs. */
int pa_edges_bytes(const pa_params *prm, uint64_t *bytes);
int pa_scratch_bytes(const pa_params *prm, uint64_t *bytes);

/* Nodes [d+1, *u_split) are generated by the start kernel (pa_params.start_nodes
 * rounded up to whole superblocks of the persistent launch, at most n); the
 * rest by the persistent launch. */
int pa_start_split(const pa_params *prm, uint64_t *u_split);

/* ---- generation ---------------------------------------------------------- */
/* Stream-ordered generation into caller memory.  d_scratch (pa_scratch_bytes)
 * is cleared by the call; it must not be shared by generations that overlap.
 * Host-side errors return at once; device-side status is read by pa_generate_finish. */
int pa_generate(const pa_params *prm, void *d_edges, uint64_t edges_bytes, void *d_scratch,
                uint64_t scratch_bytes, void *stream);
/* pa_generate with the phases timed: events[0..3] (cudaEvent_t, any may be
 * NULL) are recorded on `stream` before the first launch, before the start
 * kernel (after the scratch clear and the all-ones fill of its region), before
 * the persistent launch, and after the last launch.  The device side of the
 * per-stage timing table the reference writes (src/PA/cuPPA/cuPPA_1.cu:84-87,
 * 217-223). */
int pa_generate_timed(const pa_params *prm, void *d_edges, uint64_t edges_bytes, void *d_scratch,
                      uint64_t scratch_bytes, void *stream, void *const *events);
/* Set the generation region of d_edges -- every slot a generation writes and
 * reads back, the seed edges aside -- to all-ones, the "not yet written" mark
 * the generators wait on, for a later generation with PA_FLAG_PREFILLED.  The
 * fill runs on a small grid (one 128-thread block per SM), so it can run beside
 * a generation on another stream: a caller that generates graphs back to back
 * into two buffers fills the next buffer while the current one is generated.
 * Queued on `stream`.  No counterpart in the reference, whose per-batch fill
 * (src/PA/cuPPA/cuPPA_RRP.cu:78-102) sits inside its stage loop. */
int pa_fill(const pa_params *prm, void *d_edges, uint64_t edges_bytes, void *stream);
/* Wait for the stream, then copy the status and counters of the generation that
 * last used d_scratch.  Returns the device status. */
int pa_generate_finish(const void *d_scratch, pa_stats *out, void *stream);

/* Generation for callers that cannot allocate device memory (a host whose
 * memory pool forbids further allocations, or a latency-critical request loop
 * that must not stall in cudaMalloc/cudaFree).  No counterpart in the
 * reference.  The scratch lives in a PA_NOALLOC_SCRATCH_BYTES (16 MiB)
 * __device__ array inside this library, held on every GPU that loads it until
 * the process exits; the caller passes only the parameters and the edge
 * buffer.  Requests whose scratch exceeds the array (roughly n > 65 million
 * nodes at d = 4, n > 8 million at d = 32) return PA_ERR_CAPACITY before any GPU
 * work.  The first call in a CUDA context looks the array's address up with
 * cudaGetSymbolAddress (with that context's device current) and caches it under
 * the context's ID, so a context created anew after cudaDeviceReset is looked
 * up again.  All calls on a device share the array, so calls whose GPU work
 * overlaps race on it: issue them on one stream or serialize them.  Each call clears what it uses, generates on `stream`,
 * waits for it, fills *stats (may be NULL) and returns the device status. */
#define PA_NOALLOC_SCRATCH_BYTES (16u << 20)
int pa_generate_noalloc(const pa_params *prm, void *d_edges, uint64_t edges_bytes,
                        pa_stats *stats, void *stream);

/* Progress trace of the generation that last used d_scratch (waits for the
 * stream): up to max_samples pairs (elapsed ns since the launch's first warp
 * started, nodes known complete), 2 x uint64 each, in time order; *count gets
 * the number written.  The device side of the per-stage timing table the
 * reference writes (src/PA/cuPPA/cuPPA_1.cu:84-87,217-223). */
int pa_generate_trace(const pa_params *prm, const void *d_scratch, uint64_t *out,
                      uint32_t max_samples, uint32_t *count, void *stream);

/* ---- captured generations (CUDA graphs) --------------------------------------- */
/* For small graphs, issuing the scratch clear, the sentinel fill and the kernel
 * launch one by one costs about as much as the GPU work.  A plan captures that
 * sequence once, for fixed parameters and buffers, into a CUDA graph;
 * pa_plan_launch replays it on `stream` with one graph launch and writes what
 * pa_generate would.  The buffers must outlive the plan and must not be used by
 * anything else while a replay runs; read the status with
 * pa_generate_finish(d_scratch, ...).  No counterpart in the reference. */
typedef struct pa_plan pa_plan;
int pa_plan_create(const pa_params *prm, void *d_edges, uint64_t edges_bytes, void *d_scratch,
                   uint64_t scratch_bytes, pa_plan **out);
int pa_plan_launch(pa_plan *plan, void *stream);
int pa_plan_destroy(pa_plan *plan);

/* ---- post-processing ------------------------------------------------------ */
/* Sort every node's d pairs by dst in place (or into d_out): the canonical edge
 * list -- all (u, v) with u > v sorted by (u, v). */
int pa_canonicalize(const pa_params *prm, const void *d_edges, void *d_out, void *stream);
/* Undirected degree of every node: d_deg is int64[n]. */
int pa_degrees(const pa_params *prm, const void *d_edges, int64_t *d_deg, void *stream);

/* Position-keyed digest of `count` ids of id_bits width at d_ids: d_acc[0]
 * (device uint64) gains the sum and d_acc[1] the xor of
 *   h = fmix64(fmix64(pos * 0x9E3779B97F4A7C15 + 0x632BE59BD9B4E019) ^ x),
 * x the id sign-extended to 64 bits, pos = index_base + i, fmix64 MurmurHash3's
 * 64-bit finalizer.  A fingerprint of a whole graph that never leaves the
 * device: pass an edge list as 2 * pa_edge_count() ids (src of edge e at 2e,
 * dst at 2e+1), a CSR as its rowptr (64-bit) and col.  The digest of a
 * concatenation is the sum and xor of its parts' digests taken with their
 * index bases, so a graph can be digested in pieces; clear d_acc to start one.
 * Queued on `stream`.  No counterpart in the reference. */
int pa_digest(const void *d_ids, uint64_t count, uint32_t id_bits, uint64_t index_base,
              uint64_t *d_acc, void *stream);

/* ---- CSR ------------------------------------------------------------------ */
/* Undirected CSR of a generated edge list (PAIRS layout, slot or canonical
 * order): every edge appears in both rows, and every row is sorted ascending.
 * d_rowptr is int64[n+1]; d_col holds 2 * pa_edge_count() ids of id_bits width.
 * Sizes of the three buffers: */
int pa_csr_bytes(const pa_params *prm, uint64_t *rowptr_bytes, uint64_t *col_bytes,
                 uint64_t *scratch_bytes);
/* Builds the CSR on `stream` and waits for it (for its error word).  The in
 * parts come from a stable radix sort of the pairs by destination; the column
 * buffer doubles as sort space during the call.  d_col and d_scratch must be
 * 16-byte aligned.  Graphs of 2^32 nodes or more: PA_ERR_NOT_SUPPORTED. */
int pa_build_csr(const pa_params *prm, const void *d_edges, int64_t *d_rowptr, void *d_col,
                 void *d_scratch, uint64_t scratch_bytes, void *stream);

/* ---- batches ---------------------------------------------------------------- */
/* Many independent graphs in shared launches (no counterpart in the reference,
 * which makes one graph per run): one fill, one start-kernel launch over every
 * graph's start region and one tail launch over the rest, the work of all
 * graphs interleaved level by level.  prms[i] describes graph i (all of one id
 * width, every n < 2^32 - 64; tile_passes is taken from prms[0]); graph i is
 * written to d_edges[i] (edges_bytes[i] >= pa_edges_bytes(prms[i])) exactly as
 * pa_generate would write it.  The call copies a small table to the device and
 * waits for that copy, then returns with the launches queued; read the status
 * with pa_generate_finish(d_scratch, ...). */
int pa_batch_scratch_bytes(const pa_params *prms, uint32_t count, uint64_t *bytes);
int pa_batch_generate(const pa_params *prms, uint32_t count, void *const *d_edges,
                      const uint64_t *edges_bytes, void *d_scratch, uint64_t scratch_bytes,
                      void *stream);

/* ---- request server ------------------------------------------------------------ */
/* A served stream of independent generation requests (no counterpart in the
 * reference, which makes one graph per process run, src/main.cu:105-116).  One
 * control thread per server owns its CUDA streams on its device: it admits
 * queued requests while their device memory (edge buffer + generation scratch)
 * fits the budget, launches everything admitted as one batch
 * (pa_batch_generate's launches) whenever a lane has fewer than max_inflight
 * batches on the GPU -- so requests that arrive while a batch runs form the
 * next one -- and marks each request done when its batch's completion event
 * has fired; it never waits on the GPU.  Two lanes share the budget: requests
 * of at most express_edges edges run in the express lane, on a stream of the
 * device's highest priority with a memory pool of its own, so a small request
 * that arrives while a large batch runs starts at that batch's next kernel
 * boundary; a lane's launches queue in order on its stream.
 * A result stays in device memory, owned by the server, until
 * pa_server_release (or until it has been finished for ttl_ns).  Submit, poll,
 * wait and release may be called from any thread. */
typedef struct pa_server pa_server;

/* pa_server_config.outputs: what a finished request keeps on the device (a
 * mask; 0 = PAIRS).  With CSR the server builds each graph's undirected CSR
 * (pa_build_csr) right after its batch, in the same stream. */
enum { PA_OUT_PAIRS = 1, PA_OUT_CSR = 2 };

typedef struct pa_server_config {
    uint64_t budget_bytes;   /* device memory for admitted requests; 0 = 3/4 of free memory */
    uint32_t max_batch;      /* requests per launch; 0 = 4096                              */
    uint32_t max_inflight;   /* batches queued on the GPU at once per lane; 0 = 4          */
    uint32_t max_queue;      /* queued (not yet admitted) requests; 0 = unlimited          */
    int32_t device;          /* CUDA device; -1 = the caller's current device              */
    uint64_t ttl_ns;         /* finished results unreleased this long are freed; 0 = never */
    uint64_t aging_ns;       /* a queued request that has waited this long is not passed
                                over by smaller ones; 0 = 100 ms                           */
    uint32_t outputs;        /* PA_OUT_* mask; 0 = PA_OUT_PAIRS                            */
    uint32_t express_edges;  /* requests of at most this many edges use the express lane;
                                0 = 2^22                                                   */
} pa_server_config;

typedef struct pa_result {
    const void *edges;       /* device pointer (the PAIRS layout), valid until release;
                                NULL unless the server keeps PA_OUT_PAIRS                */
    uint64_t n_edges;
    uint64_t edges_bytes;
    int32_t status;          /* pa_status of the generation                              */
    uint32_t batch_size;     /* requests in the launch that produced it                  */
    uint64_t t_submit_ns;    /* server clock: ns since pa_server_create                   */
    uint64_t t_start_ns;     /* its batch was launched                                    */
    uint64_t t_done_ns;      /* the control thread saw the batch complete                 */
    const int64_t *rowptr;   /* with PA_OUT_CSR: int64[n + 1], valid until release        */
    const void *col;         /* with PA_OUT_CSR: 2 * n_edges ids of id_bits width         */
    uint64_t col_bytes;
} pa_result;

typedef struct pa_server_stats {
    uint64_t submitted, completed, released, expired, failed;
    uint64_t batches;        /* launches so far                                           */
    uint64_t queued;         /* waiting for admission now                                 */
    uint64_t running;        /* admitted, not finished                                    */
    uint64_t bytes_in_use;   /* budget held by admitted and unreleased requests           */
    uint64_t budget_bytes;
    uint64_t edges_done;     /* edges of completed requests                               */
} pa_server_stats;

int pa_server_config_init(pa_server_config *cfg);
/* Start a server (its control thread and stream); *out gets the handle. */
int pa_server_create(const pa_server_config *cfg, pa_server **out);
/* Queue a request (a copy of *prm is kept; id widths may differ between
 * requests).  PA_ERR_CAPACITY: it can never fit the budget; PA_ERR_BUSY: the
 * queue is full.  *ticket identifies it from then on. */
int pa_server_submit(pa_server *srv, const pa_params *prm, uint64_t *ticket);
/* PA_OK with *out filled once the request is finished (its own outcome in
 * out->status), PA_ERR_BUSY while it is queued or running, PA_ERR_NOT_FOUND for
 * an unknown, released or expired ticket. */
int pa_server_poll(pa_server *srv, uint64_t ticket, pa_result *out);
/* As poll, but blocks up to timeout_ns (0 = no limit) for the request to finish. */
int pa_server_wait(pa_server *srv, uint64_t ticket, uint64_t timeout_ns, pa_result *out);
/* Give a finished (or still queued) request's memory back to the budget;
 * PA_ERR_BUSY while it runs.  The caller's own reads of the result must have
 * completed. */
int pa_server_release(pa_server *srv, uint64_t ticket);
int pa_server_stats_get(pa_server *srv, pa_server_stats *out);
/* Stop the control thread, wait for the GPU work, free everything.  No other
 * thread may be inside a pa_server_* call on this handle. */
int pa_server_destroy(pa_server *srv);

/* The server's admission queue on its own (host logic, no GPU), for tests and
 * for callers that schedule their own launches.  Arrival order is kept: a
 * request whose bytes fit the free budget is admitted; one that does not is
 * passed over, unless it has waited aging_ns, which stops the scan so that a
 * large request is not starved by a stream of small ones. */
typedef struct pa_sched pa_sched;
pa_sched *pa_sched_create(uint64_t budget_bytes, uint64_t aging_ns, uint32_t max_queue);
void pa_sched_destroy(pa_sched *q);
/* PA_OK, PA_ERR_CAPACITY (bytes > budget), PA_ERR_BUSY (queue full),
 * PA_ERR_INVALID (ticket already known). */
int pa_sched_submit(pa_sched *q, uint64_t ticket, uint64_t bytes, uint64_t now_ns);
/* Admit up to cap requests; their tickets go to out[], the count is returned. */
uint32_t pa_sched_admit(pa_sched *q, uint64_t now_ns, uint64_t *out, uint32_t cap);
/* Return `bytes` of an admitted request to the budget (all of them when bytes
 * is UINT64_MAX, which also forgets the ticket; a queued request is withdrawn).
 * PA_ERR_NOT_FOUND if unknown. */
int pa_sched_release(pa_sched *q, uint64_t ticket, uint64_t bytes);
/* Lanes (the request server keeps small requests in a lane of their own): a
 * request queued in `lane` (0..31) is admitted only by scans that include its
 * lane in lane_mask; an aged request that does not fit stops the admission of
 * its own lane only.  pa_sched_submit / pa_sched_admit are lane 0 and all lanes. */
int pa_sched_submit_lane(pa_sched *q, uint64_t ticket, uint64_t bytes, uint64_t now_ns,
                         uint32_t lane);
uint32_t pa_sched_admit_lanes(pa_sched *q, uint64_t now_ns, uint64_t *out, uint32_t cap,
                              uint32_t lane_mask);
uint64_t pa_sched_in_use(const pa_sched *q);
uint64_t pa_sched_queued(const pa_sched *q);

/* ---- several GPUs: router and batch partition ------------------------------- */
/* One graph never spans GPUs (any copy read may land on any earlier node), so
 * more GPUs serve more graphs.  A router owns one request server per device
 * (cfg copied, cfg.device replaced) and places each request on the server whose
 * routed, unreleased bytes (edge list, plus CSR arrays with PA_OUT_CSR) would be
 * the smallest fraction of its budget (pa_route_pick).  Its tickets name the
 * server; poll / wait / release behave as pa_server_*.  No data moves between
 * GPUs.  At most 255 devices; a device may be listed more than once. */
typedef struct pa_router pa_router;
int pa_router_create(const pa_server_config *cfg, const int32_t *devices, uint32_t n_devices,
                     pa_router **out);
int pa_router_submit(pa_router *r, const pa_params *prm, uint64_t *ticket);
int pa_router_poll(pa_router *r, uint64_t ticket, pa_result *out);
int pa_router_wait(pa_router *r, uint64_t ticket, uint64_t timeout_ns, pa_result *out);
int pa_router_release(pa_router *r, uint64_t ticket);
/* The CUDA device whose memory holds the ticket's result. */
int pa_router_device_of(pa_router *r, uint64_t ticket, int32_t *device);
/* Statistics of server `index` (0..size-1), or summed over all with index == size. */
int pa_router_stats_get(pa_router *r, uint32_t index, pa_server_stats *out);
uint32_t pa_router_size(const pa_router *r);
/* Destroys every server (each as pa_server_destroy) and the router; no thread may
 * be inside a pa_router_* call on this handle.  Submit, poll, wait and release
 * may be called from any threads concurrently. */
int pa_router_destroy(pa_router *r);
/* The placement rule alone (host arithmetic): the index i minimising
 * (load_bytes[i] + request_bytes) / budget_bytes[i], exactly; ties go to the
 * lowest index. */
uint32_t pa_route_pick(const uint64_t *load_bytes, const uint64_t *budget_bytes, uint32_t n,
                       uint64_t request_bytes);
/* Split a batch over k parts (one per GPU / process): instances largest first
 * (edge bytes), each to the part with the fewest bytes so far, ties to the lowest
 * part; part_of[i] in [0, k).  Deterministic: every process gets the same split. */
int pa_batch_partition(const pa_params *prms, uint32_t count, uint32_t k, uint32_t *part_of);

/* ---- files ------------------------------------------------------------------ */
enum { PA_FORMAT_TEXT = 0, PA_FORMAT_BINARY = 1 };
/* Receives the output bytes in order; return 0 to go on, nonzero to stop (the
 * call then returns PA_ERR_IO).  Called from a thread of the library, one call
 * at a time; `data` is valid until the call returns. */
typedef int (*pa_sink_fn)(void *ctx, const void *data, uint64_t bytes);

/* Stream the graph in d_edges (either layout) to `sink`: TEXT = one "u v\n" line
 * per edge, the format of PAHelper::writeGraphToDisk
 * (src/PA/SPA/PAHelper.hpp:163-177; with PA_SEED_STAR_REF also its row order);
 * BINARY = little-endian (src, dst) id pairs of id_bits each.  Order: the seed
 * edges, then rows u = d+1..n-1 in slot order.  The text is formatted on the
 * device; chunks of about chunk_edges edges (0 = 2^24) are copied to pinned host
 * memory while the next chunk is formatted and the previous one is sunk.  Runs
 * after the work already queued on `stream`; waits.  *bytes_out (optional) gets
 * the byte count. */
int pa_stream_edges(const pa_params *prm, const void *d_edges, int format, uint64_t chunk_edges,
                    pa_sink_fn sink, void *ctx, void *stream, uint64_t *bytes_out);
/* pa_stream_edges keeps its staging memory (two pinned host buffers and two
 * device buffers of one chunk each) for the next call on the same device;
 * pa_stream_trim frees it (PA_ERR_BUSY while a stream is running). */
int pa_stream_trim(void);
/* pa_stream_edges into the file `path` (created or truncated); waits. */
int pa_write_edges(const pa_params *prm, const void *d_edges, const char *path, int format,
                   void *stream);
/* Generate and write in one call (library-owned device memory, freed before
 * return): with layout PA_LAYOUT_SLOTS the device holds only the targets, so
 * graphs whose edge list is larger than the GPU's memory can be written.
 * *stats (optional) as pa_generate_finish. */
int pa_generate_to_file(const pa_params *prm, const char *path, int format, pa_stats *stats,
                        uint64_t *bytes_out);
/* Write the "Degree,Count" CSV of cuPPA::printDegreeDistribution
 * (src/PA/cuPPA/cuPPA.cu:103-165) for the graph in d_edges; degrees and their
 * histogram are computed on the device (temporaries allocated and freed with
 * cudaMallocAsync/cudaFreeAsync on `stream`); waits. */
int pa_write_degree_distribution(const pa_params *prm, const void *d_edges, const char *path,
                                 void *stream);

/* ---- convenience handle (library-owned memory) ----------------------------- */
typedef struct pa_graph {
    pa_params params;
    void *edges;            /* device, edges_bytes                                        */
    uint64_t n_edges;
    uint64_t edges_bytes;
    void *scratch;          /* device, scratch_bytes                                      */
    uint64_t scratch_bytes;
} pa_graph;

/* Allocate edges + scratch on the current device for prm (no generation). */
int pa_graph_create(const pa_params *prm, pa_graph *g);
/* Generate into g on `stream` and wait; stats may be NULL. */
int pa_graph_generate(pa_graph *g, void *stream, pa_stats *stats);
/* Free what pa_graph_create allocated; safe on a zeroed handle. */
int pa_graph_destroy(pa_graph *g);

/* ---- errors --------------------------------------------------------------- */
const char *pa_strerror(int status);
/* The cudaError_t of the last PA_ERR_CUDA / PA_ERR_OOM on the calling thread. */
int pa_last_cuda_error(void);
int pa_abi_version(void);

#ifdef __cplusplus
}
#endif

#endif /* CUPPA_PA_H_ */
