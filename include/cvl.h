/*
 * cvl.h -- C ABI of the B200 curvelet-construction engine (libcvl.so).
 *
 * The engine is a drop-in for the reference cpu_curvelet path
 *   preprocess (spatial hash + neighbour CSR)
 *   -> pairwise curve-bundle formation
 *   -> greedy edge-chain growth, dedup and record,
 * computed in FP64 by hand-written sm_100a CUDA kernels on one GPU.
 *
 * Conventions: plain C types; every entry point returns an int status
 * (CVL_OK = 0, negative on error) unless stated; cvl_last_error() gives a
 * one-line reason for the calling thread's last failure. An engine handle is
 * used by one host thread at a time. Inputs are caller-owned and only read
 * during the call; results are engine-owned until freed.
 *
 * Reference citations are path:line within the reference project
 * (C-H-Chien/Curvelet_Construction_on_GPU).
 */
#ifndef CVL_H
#define CVL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define CVL_OK 0
#define CVL_EINVAL (-1)       /* invalid argument (reference: preprocess.hpp:197-199 returns false) */
#define CVL_ENOMEM (-2)       /* device or host allocation failed, or over the memory budget */
#define CVL_ECUDA (-3)        /* a CUDA runtime call failed */
#define CVL_EUNSUPPORTED (-4) /* parameters outside what the kernels are built for */
#define CVL_ETIMEDOUT (-5)    /* a bounded wait expired (serving) */
#define CVL_EOVERFLOW (-6)    /* a capacity was exceeded (reported, never silently truncated) */
#define CVL_EAGAIN (-7)       /* request not finished yet (serving poll) */
#define CVL_ENODEV (-8)       /* no usable CUDA device */

/* ---- parameters ------------------------------------------------------ */
/* Mirrors CurveletParams, cpu_curvelet/param_settings.hpp:9-24 (same names,
 * same defaults, same meaning). gap, curvelet_style and out_type are accepted
 * and ignored exactly as the reference ignores them (main.cpp:29,32,94-95). */
typedef struct cvl_params {
    double nrad;             /* neighbour radius, px (3.5) */
    double gap;              /* unused by the curvelet path; the contour gap of cvl_run_contours (1.5) */
    double dx;               /* edge position uncertainty, px (0.4) */
    double dt_deg;           /* edge orientation uncertainty, degrees (15) */
    double dt_rad;           /* the same in radians, as CurveletCPU's ctor takes it (cpu_curvelet.hpp:82-83);
                                used as is when > 0, else dt = (dt_deg / 180) * pi (main.cpp:24) (0) */
    double max_k;            /* curvature bound (0.3) */
    unsigned curvelet_style; /* 2 = anchor-leading bidirectional (the only style the path runs) */
    unsigned group_max_sz;   /* maximum edges per curvelet, anchor included (4); 1..16 supported */
    unsigned out_type;       /* unused by the path (0) */
    double sx;               /* bundle grid step in position, px (0.1) */
    double st;               /* bundle grid step in orientation, rad (0.08) */
    int edge_data_sz;        /* values per edge row, >= 4 (4) */
    unsigned max_candidates; /* neighbour cap per anchor (128); 1..1024 supported */
} cvl_params;

/* Fills the reference defaults (param_settings.hpp:11-23). */
void cvl_params_default(cvl_params *p);

/* ---- engine ----------------------------------------------------------- */
typedef struct cvl_engine cvl_engine;

typedef struct cvl_engine_cfg {
    int device;               /* CUDA device ordinal (0) */
    size_t mem_budget_bytes;  /* device memory the engine may hold; 0 = no limit */
    int cell_size;            /* initial spatial-hash block edge of every tuning bucket: 2, 4 or 8;
                                 0 = 4 up to 512 Ki edges and 8 above */
    int seeds_per_group;      /* initial seeds per group of every tuning bucket: 4 or 8; 0 = 4 */
    int bundle_slots;         /* reserved, unused (0) */
    int warps_per_block;      /* reserved, unused (0) */
    int stream_priority;      /* the engine stream's priority: 0 = default, negative = higher
                                 (clamped to cudaDeviceGetStreamPriorityRange) (0) */
} cvl_engine_cfg;

void cvl_engine_cfg_default(cvl_engine_cfg *cfg);
int cvl_engine_create(const cvl_engine_cfg *cfg, cvl_engine **out);
/* No reference counterpart. Runs two built-in maps (about 520 and 75,000 edges)
 * through the engine's forms of the path (kernel by kernel, and the graphs of the
 * two small size buckets), so that the kernels are loaded and the workspace pools
 * hold memory before the first real input: a process's first run otherwise pays
 * module loading and allocation. The engine's settings are unchanged afterwards. */
int cvl_engine_warmup(cvl_engine *e);
/* Also frees the engine's batches that are still alive (their handles become
 * invalid), and any batch result of the engine can then no longer be read. */
void cvl_engine_destroy(cvl_engine *e);

/* One-line description of the calling thread's last error ("" if none). */
const char *cvl_last_error(void);
/* Library version string. */
const char *cvl_version(void);

/* ---- results ---------------------------------------------------------- */
typedef struct cvl_result cvl_result;

/* Flags reported in cvl_result_view.flags. */
#define CVL_FLAG_TRUNCATED 1u /* some anchor reached max_candidates (preprocess.hpp:224-229) */

typedef struct cvl_result_view {
    uint32_t num_curvelets;  /* rows, = CurveletCPU::num_curvelets() (cpu_curvelet.hpp:95) */
    uint32_t chain_width;    /* group_max_sz + 1 (cpu_curvelet.hpp:96) */
    const uint32_t *chains;  /* [num_curvelets][chain_width], row-major, 1-based edge ids,
                                zero padded: _edge_chain_final[0:num_curvelets] (cpu_curvelet.hpp:258-280) */
    const double *info;      /* [num_curvelets][10], row-major: the info file's rows
                                (main.cpp:81-88; columns per cpu_curvelet.hpp:246-255) */
    uint32_t valid_pairs;    /* form_pairwise_bundles' count (cpu_curvelet.hpp:305-361) */
    int64_t total_neighbor_pairs;  /* CPUNeighborGraph::total_neighbor_pairs (preprocess.hpp:248) */
    uint32_t max_num_of_neighbors; /* CPUNeighborGraph::max_num_of_neighbors (preprocess.hpp:243-245) */
    uint32_t truncated_anchors;    /* anchors that reached max_candidates (preprocess.hpp:224-229) */
    uint32_t num_edges;
    uint32_t flags;                /* CVL_FLAG_* */
    double device_ms;              /* device time of the compute (CUDA events), excluding copies */
} cvl_result_view;

/* The one-shot plain form: one edge map (AoS rows of edge_data_sz doubles,
 * host memory) -> curvelets, i.e. run_curvelet<double> without the file I/O
 * (main.cpp:20-96: build_neighbor_csr_graph + CurveletCPU::form_pairwise_bundles
 * + CurveletCPU::build_curvelets_greedy). Copies in, computes, copies out. */
int cvl_run(cvl_engine *e, const double *edges, int32_t num_edges, int32_t edge_data_sz,
            const cvl_params *p, cvl_result **out);

/* The same in the reference's --float mode (run_curvelet<float>, main.cpp:110):
 * edges as float, the path computed with the reference's float-mode types (its
 * float arithmetic, and the double expressions it rounds to float). The result
 * has the same layout (info holds the float values as doubles). */
int cvl_run_f32(cvl_engine *e, const float *edges, int32_t num_edges, int32_t edge_data_sz,
                const cvl_params *p, cvl_result **out);

/* The plain form on edges already in device memory, e.g. written by an edge
 * detector on the same GPU, so they never cross to the host. d_edges is a
 * device (or managed) pointer on the engine's device, AoS rows of edge_data_sz
 * doubles, read in place. The engine's stream waits for ready_event (a
 * cudaEvent_t the producer recorded after writing the edges) or, if it is NULL,
 * for nothing: the caller then has already finished writing them.
 * out != NULL: results come back as cvl_run's. out == NULL: they stay on the
 * device, readable through cvl_engine_device_results until the engine's next run.
 * CVL_EINVAL for a host pointer or one on another device. */
int cvl_run_device(cvl_engine *e, const double *d_edges, int32_t num_edges, int32_t edge_data_sz,
                   const cvl_params *p, void *ready_event, cvl_result **out);

/* Device-resident outputs of the engine's last cvl_run_device: chains and info
 * laid out as in cvl_result_view, in the engine's device memory. They are valid
 * until the engine runs again or is destroyed. done_event (may be NULL) receives
 * a cudaEvent_t to wait on before reading them from another stream; the engine
 * owns it. */
typedef struct cvl_device_results {
    uint32_t num_curvelets;
    uint32_t chain_width;
    const uint32_t *chains; /* device pointer */
    const double *info;     /* device pointer */
    void *done_event;       /* cudaEvent_t recorded after the outputs were written */
} cvl_device_results;
int cvl_engine_device_results(cvl_engine *e, cvl_device_results *out);

/* Views a result. chains/info point into page-locked host memory owned by the
 * result; they stay valid until cvl_result_free, which may also be called after
 * the engine was destroyed. */
int cvl_result_get(const cvl_result *r, cvl_result_view *view);
void cvl_result_free(cvl_result *r);

/* ---- the reference's staged template API ------------------------------ */
/* Neighbour graph: build_neighbor_csr_graph<T> (preprocess.hpp:186-274) and
 * CPUNeighborGraph<T> (preprocess.hpp:18-31). neighbor_radius is the pixel-cell
 * window half width (the reference passes 3u, main.cpp:48). */
typedef struct cvl_graph cvl_graph;
typedef struct cvl_graph_view {
    int32_t num_edges;
    int64_t total_neighbor_pairs;
    uint32_t max_num_of_neighbors;
    uint32_t truncated_anchors;
    const int32_t *neighbor_offsets; /* [num_edges + 1] (int64 totals above 2^31 are rejected) */
    const int32_t *neighbor_ids;     /* [total_neighbor_pairs], ascending distance */
    const double *neighbor_dist2;    /* [total_neighbor_pairs] */
} cvl_graph_view;

int cvl_build_neighbor_graph(cvl_engine *e, const double *edges, int32_t num_edges, int32_t edge_data_sz,
                             double rad, unsigned neighbor_radius, unsigned max_candidates, cvl_graph **out);
int cvl_graph_get(const cvl_graph *g, cvl_graph_view *view);
void cvl_graph_free(cvl_graph *g);

/* CurveletCPU::form_pairwise_bundles (cpu_curvelet.hpp:305-361): the number of
 * (anchor, neighbour) pairs with a valid curve bundle, over the graph's pairs. */
int cvl_form_pairwise_bundles(cvl_engine *e, const cvl_graph *g, const cvl_params *p, uint32_t *valid_pairs);

/* CurveletCPU::build_curvelets_greedy (cpu_curvelet.hpp:363-634) over a graph
 * built by cvl_build_neighbor_graph. */
int cvl_build_curvelets(cvl_engine *e, const cvl_graph *g, const cvl_params *p, cvl_result **out);

/* CurveletCPU::compute_curve_bundle for n independent pairs (cpu_curvelet.hpp:637-819):
 * pairs[i] = (te_x, te_y, te_theta, le_x, le_y, le_theta). Writes bmin/bmax
 * [n][cells] and valid[n] (1 = the reference's hyp_LookEdge true). cells =
 * P*Q of the grid (cpu_curvelet.hpp:73-74) is returned in *cells. */
int cvl_pair_bundles(cvl_engine *e, const double *pairs, int32_t n, const cvl_params *p,
                     double *bmin, double *bmax, uint8_t *valid, int32_t *cells);

/* ---- failure injection (tests) ----------------------------------------
 * No reference counterpart (the reference only prints errors,
 * cpu_curvelet/data_io.hpp:27-76). From this call on, `after` more device or
 * page-locked allocations of the library succeed, then every one fails as if
 * the memory were exhausted (the call that needed it returns CVL_ENOMEM), until
 * the next call; -1 turns it off. Host side only: nothing on the GPU fails.
 * CVL_FAIL_ALLOC_AFTER=<after> in the environment arms it when the library
 * loads. */
int cvl_debug_fail_allocations(int64_t after);

/* ---- checking entry points ------------------------------------------- */
/* No reference counterpart: they exist so that tests can reach the device code of
 * the transport at chosen operands.
 *
 * cvl_check_pair_bundles_literal: cvl_pair_bundles through the reference's two
 * branches as written (cpu_curvelet.hpp:693-809, one formula per branch) on the
 * same device trig values, where cvl_pair_bundles runs the rewritten arithmetic of
 * the path's bundle kernel. The two must agree bit for bit. */
int cvl_check_pair_bundles_literal(cvl_engine *e, const double *pairs, int32_t n, const cvl_params *p,
                                   double *bmin, double *bmax, uint8_t *valid, int32_t *cells);
/* cvl_check_transport_cells: one orientation column (cells (i, j), i < P) of the
 * transport per row of ops[n][10] = (DX, DY, tt, s_m, s_p, cos(T0 - dt),
 * sin(T0 - dt), cos(T0 + dt), sin(T0 + dt), branch1 != 0), the operands of
 * cpu_curvelet.hpp:693-809 given directly, so that cells built to cancel reach the
 * device. out[n][4][P]: the path's rewritten arithmetic (bmin, then bmax), then
 * the reference's two branches as written (bmin, bmax). quotients selects how the
 * rewritten arithmetic forms its two k_dx quotients: 0 two IEEE divisions, 1 one
 * correctly rounded reciprocal and Markstein's corrections, each operand's range
 * checked per cell (the bundle kernel's form on certified runs). *rows = P. */
int cvl_check_transport_cells(cvl_engine *e, const double *ops, int32_t n, const cvl_params *p, int32_t quotients,
                              double *out, int32_t *rows);

/* ---- pair bundles without any allocation ------------------------------ */
/* No reference counterpart. The same computation and outputs as
 * cvl_pair_bundles, plus the number of valid pairs (the count
 * form_pairwise_bundles keeps, cpu_curvelet.hpp:305-361). It needs no engine
 * and allocates no device memory: no cudaMalloc/cudaFree and no library
 * allocator (on success it makes no host allocation either; a failure stores
 * its message in a thread-local string). Device work goes through one fixed scratch area per
 * device, a static device array of CVL_NOALLOC_SCRATCH_BYTES, on the calling
 * thread's default stream (cudaStreamPerThread), on the current device.
 *
 * It is for callers that must not allocate device memory during the call:
 * cudaFree synchronises the whole device, and cudaMalloc can fail or stall
 * once a framework allocator has reserved the memory. Examples are a process
 * whose memory is already fully reserved, and a latency-bound loop.
 *
 * Limit: the scratch holds the call's pairs, bundles and flags at once:
 *   256 + a(48 n) + 2 a(8 n cells) + a(n) <= CVL_NOALLOC_SCRATCH_BYTES,
 * where a(x) rounds x up to 256. That is 15,872 pairs for the default
 * 7 x 9 = 63-cell grid. Larger n returns CVL_EOVERFLOW and does no work; split
 * the pairs over several calls.
 *
 * The scratch is part of the library's device code: every CUDA context in which
 * the library's kernels are loaded holds its 16 MiB until the context ends,
 * whether or not this entry point is ever called.
 *
 * The first call on a device does the set-up (it looks up the scratch's
 * address with the device current), and so does the first call after the
 * device's context was destroyed and created again (cudaDeviceReset, for one):
 * the address is kept with the id of the context it belongs to. Make the first
 * call before any stream capture on the device. No call may be made while the
 * calling thread's stream (cudaStreamPerThread) is capturing: the call
 * synchronises that stream, so it returns CVL_EINVAL instead. Calls that overlap
 * in time on one device, from several host threads, share the scratch and race:
 * serialise them. Each call clears its valid-pair counter before use and returns
 * after its results are in the caller's host buffers. */
#define CVL_NOALLOC_SCRATCH_BYTES (16u << 20)
int cvl_pair_bundles_noalloc(const double *pairs, int32_t n, const cvl_params *p, double *bmin, double *bmax,
                             uint8_t *valid, uint32_t *valid_pairs, int32_t *cells);

/* ---- device-resident maps (benchmarks, batching) ---------------------- */
/* A ragged batch of edge maps kept in device memory: maps[m] has counts[m]
 * rows of edge_data_sz doubles, concatenated in edges. */
typedef struct cvl_batch cvl_batch;

int cvl_batch_upload(cvl_engine *e, const double *edges, const int32_t *counts, int32_t num_maps,
                     int32_t edge_data_sz, cvl_batch **out);
/* Replaces a batch's maps with new ones. The device buffer is reused when it is
 * large enough (grow-only), so a steady stream of batches makes no device
 * allocation and no device-wide synchronisation. */
int cvl_batch_refill(cvl_batch *b, const double *edges, const int32_t *counts, int32_t num_maps,
                     int32_t edge_data_sz);
/* The same with map m's rows at parts[m] (counts[m] rows each): the maps are
 * copied straight from where they are, with no host-side concatenation. */
int cvl_batch_refill_parts(cvl_batch *b, const double *const *parts, const int32_t *counts, int32_t num_maps,
                           int32_t edge_data_sz);
void cvl_batch_free(cvl_batch *b);

/* Runs the whole path over every map of a device-resident batch in one pass
 * (ragged: one spatial hash, one neighbour pass, one fused bundle/growth pass,
 * one compaction for all maps). Results stay in device memory; device_ms is
 * filled. Per-map results are read with cvl_batch_result_*. */
typedef struct cvl_batch_result cvl_batch_result;
int cvl_batch_run(cvl_engine *e, const cvl_batch *b, const cvl_params *p, cvl_batch_result **out);
/* Downloads (once, into page-locked memory) and views map m of a batch result;
 * the view lives as long as the batch result. */
int cvl_batch_result_map(cvl_batch_result *r, int32_t m, cvl_result_view *view);
/* Map m of a batch result as an independent result (its own page-locked
 * copy, freed with cvl_result_free): only that map's rows cross PCIe. */
int cvl_batch_result_take_map(cvl_batch_result *r, int32_t m, cvl_result **out);
/* Totals of a batch run over all its maps. */
typedef struct cvl_batch_stats {
    double device_ms;              /* device time of the batch compute (CUDA events) */
    uint64_t num_curvelets;
    uint64_t valid_pairs;          /* pairs with a valid bundle */
    uint64_t total_pairs;          /* neighbour pairs */
    uint64_t close_pairs;          /* pairs closer than 2 dx: default bundle, no transport (cpu_curvelet.hpp:682) */
    uint32_t max_num_of_neighbors;
    uint32_t truncated_anchors;
    uint32_t num_maps;
    uint32_t launches;             /* kernels launched by the run */
} cvl_batch_stats;
int cvl_batch_result_stats(const cvl_batch_result *r, cvl_batch_stats *out);
void cvl_batch_result_free(cvl_batch_result *r);

/* Many maps from host memory to host results in one call, each map as cvl_run
 * would return it (out[m], freed with cvl_result_free). edges holds the maps'
 * rows back to back (counts[m] rows each). The maps go through the path in groups
 * of whole maps of about group_edges edges (<= 0: a sixth of the total, clamped
 * to [1 Mi, 8 Mi], with the smallest maps, about a sixteenth of the edges, held
 * back for a last group of their own). While one group computes on the engine's
 * stream, the next group's edges go up on a second stream and the previous
 * group's results come down to page-locked host memory on a third, so both
 * overlap the compute (page-locked input edges make the uploads asynchronous).
 * Each view's device_ms is the whole call's device time. On error nothing is
 * returned. */
int cvl_run_maps(cvl_engine *e, const double *edges, const int32_t *counts, int32_t num_maps, int32_t edge_data_sz,
                 const cvl_params *p, int64_t group_edges, cvl_result **out);

/* ---- serving: continuous batching with memory-budget admission ----------
 * No reference counterpart (the reference runs one map per process). A server
 * owns `workers` engines on one device, each with its own stream and
 * workspace. Each engine works in its own host thread:
 *   1. It takes waiting requests from its lane's queue in arrival order, up to
 *      max_batch_edges per launch, while the admission budget allows.
 *   2. It uploads them as one ragged batch and runs the whole path.
 *   3. It hands each map's result to its request.
 * Requests that arrive while others are on the GPU are folded into the next
 * launch of a free worker, and the workers' launches overlap on the device.
 *
 * Maps of at least large_map_edges edges go to a separate lane, so small
 * maps do not queue behind them. With two or more workers, the last worker
 * prefers the large lane and the others the small one. An idle large-lane
 * worker takes small maps; a small-lane worker takes large maps only when
 * small_takes_large is set. Small-lane workers run on the device's highest stream
 * priority, so their kernels go ahead of a large map's between its blocks.
 * A request's edges are copied at submit into page-locked memory that the
 * server reuses, and go from there to the device.
 *
 * Admission: a request holds its footprint of the budget from upload to result.
 * The footprint is the device workspace of a launch of that map alone
 * (cvl_engine_workspace_bytes), at pairs_per_edge and curvelets_per_edge, less the
 * bundle chunk, which each worker holds once. With admit_bytes_per_edge set, the
 * footprint is admit_bytes_per_edge x the map's edges instead. A request that can
 * never fit (or has more than max_map_edges edges) is refused at submit with
 * CVL_ENOMEM. One server serves one cvl_params.
 *
 * Memory: each worker reserves at creation the workspace of the largest launch
 * its lane takes (cvl_engine_reserve_workspace): max_batch_edges edges for a
 * small-lane worker, max_map_edges for a large-lane one, each at pairs_per_edge
 * and curvelets_per_edge, never more than the budget admits. A launch within that
 * shape allocates no device memory, so the stream never waits on a memory
 * mapping; a launch beyond it grows the worker's workspace (device_grows). */
typedef struct cvl_server cvl_server;
typedef struct cvl_server_cfg {
    int device;                    /* CUDA device ordinal (0) */
    int workers;                   /* engines working concurrently (4) */
    size_t mem_budget_bytes;       /* device bytes that admitted requests may hold at once (40 GiB) */
    size_t admit_bytes_per_edge;   /* 0: a request's footprint by the workspace formula above; else this
                                      many bytes per edge (0) */
    int64_t max_batch_edges;       /* edges folded into one launch at most; a larger map runs alone (2 Mi) */
    int64_t large_map_edges;       /* maps with at least this many edges use the large lane (1,000,000) */
    size_t host_reserve_bytes;     /* page-locked host memory set aside at creation for each worker's results
                                      and for the queued requests, so that serving does not pin memory (2 GiB) */
    int small_takes_large;         /* 1: a small-lane worker with an empty lane takes large maps;
                                      0: it keeps free for small maps (0: measured to cut the small maps'
                                      p99 from 120-170 ms to 20-45 ms at 35-80 maps/s, for no throughput) */
    int large_workers;             /* workers that serve the large lane first, the last ones, in
                                      [1, workers - 1]; 0 = half of them, at least one (0: 2 of 4 workers,
                                      measured to cut the large maps' p99 by 10-30% at 50-80 maps/s and
                                      keep the small maps' within 22-38 ms) */
    int large_yield_ms;            /* a large-lane launch holds back between its chunks while small-lane
                                      work is queued or running, for at most this long each time; 0 = never (10) */
    size_t device_reserve_bytes;   /* extra device memory each worker's engine maps into its memory pool at
                                      creation, for launches beyond the reserved workspace (0) */
    int64_t max_map_edges;         /* largest map accepted, and the large-lane workspace's edges (4 Mi) */
    double pairs_per_edge;         /* neighbour pairs per edge the footprint and the reservations assume (40;
                                      the synthetic workloads average 16) */
    double curvelets_per_edge;     /* curvelets per edge they assume (8; the synthetic workloads average 3) */
} cvl_server_cfg;

typedef struct cvl_server_stats {
    uint64_t submitted, completed, failed;
    uint64_t queued;               /* waiting for admission */
    uint64_t in_flight;            /* admitted, result not ready */
    uint64_t launches;             /* batch runs */
    uint64_t edges_completed;
    size_t admitted_bytes;         /* budget held right now */
    double p50_ms, p95_ms, p99_ms; /* submit -> result ready, over completed requests */
    double max_ms;
    /* where the workers' time went, summed over launches (ms of host wall time) */
    double upload_ms;              /* requests' edges to the device */
    double run_ms;                 /* cvl_batch_run */
    double device_ms;              /* of which the device time of the runs (CUDA events) */
    double result_ms;              /* each map's rows to its page-locked result */
    double queue_ms;               /* summed over requests: submit -> taken by a worker */
    /* memory growth so far (each stalls the calling worker; page-locked growth can
     * hold up the process's other CUDA calls too) */
    uint64_t device_grows;         /* device workspace allocations of the workers' engines */
    double device_grow_ms;         /* host time of those calls */
    uint64_t host_grows;           /* page-locked chunks pinned: request staging and results */
    double host_grow_ms;           /* host time of those cudaMallocHost calls */
    size_t reserved_bytes;         /* device workspace the workers reserved at creation */
} cvl_server_stats;

void cvl_server_cfg_default(cvl_server_cfg *cfg);
int cvl_server_create(const cvl_server_cfg *cfg, const cvl_params *p, cvl_server **out);
/* Copies the map (AoS rows of edge_data_sz doubles) and queues it; never blocks
 * on the device. *id names the request. */
int cvl_server_submit(cvl_server *s, const double *edges, int32_t num_edges, int32_t edge_data_sz, uint64_t *id);
/* The request's result (caller frees it with cvl_result_free), or CVL_EAGAIN
 * while it is queued or running. A request's result is handed out once. */
int cvl_server_poll(cvl_server *s, uint64_t id, cvl_result **out);
/* As poll, waiting up to timeout_us microseconds (< 0: no limit); CVL_ETIMEDOUT
 * if the result is not ready by then (the request stays queued). */
int cvl_server_wait(cvl_server *s, uint64_t id, int64_t timeout_us, cvl_result **out);
/* The earliest finished request whose result was not handed out yet, in
 * completion order: *id names it and *out is its result. Waits up to
 * timeout_us (< 0: no limit); CVL_ETIMEDOUT if none finished by then, CVL_EAGAIN
 * at once if no request is queued or running. */
int cvl_server_next(cvl_server *s, int64_t timeout_us, uint64_t *id, cvl_result **out);
int cvl_server_stats_get(cvl_server *s, cvl_server_stats *out);
/* Latency (ms, submit -> result ready), edge count and id of each completed
 * request, in completion order; returns how many were written (<= cap). ids
 * may be NULL. */
int64_t cvl_server_latencies(cvl_server *s, double *ms, int64_t *edges, uint64_t *ids, int64_t cap);
/* Where each completed request's time went, in completion order (host wall
 * clock, ms): waiting to be taken into a launch; its launch's upload and run
 * (cvl_batch_run, the path on the device); from the end of the run until its own
 * rows were copied to its result. total_ms is submit -> result ready. Returns how
 * many were written (<= cap). */
typedef struct cvl_request_times {
    uint64_t id;
    int64_t edges;
    double queue_ms, upload_ms, run_ms, result_ms, total_ms;
    int32_t launch_maps;  /* maps folded into its launch */
    int32_t worker;       /* the worker that ran it */
} cvl_request_times;
int64_t cvl_server_request_times(cvl_server *s, cvl_request_times *out, int64_t cap);
/* Finishes the requests already admitted, drops the queued ones, stops the
 * workers and releases everything. */
void cvl_server_destroy(cvl_server *s);

/* ---- edge files ----------------------------------------------------------
 * read_TO_edges_from_file (data_io.hpp:22-79) for any path, multi-threaded:
 * the same values and the same error messages (in cvl_last_error) as the
 * reference's stream reader on every input. A path ending in ".cvle" is read as
 * the binary format of cvl_write_edges_binary instead. *edges is freed with
 * cvl_free_edges. nthreads 0: all hardware threads; -1: the stream reader
 * alone, line by line (the reference's loop, for comparisons). */
int cvl_read_edges(const char *path, int32_t values_per_edge, int32_t nthreads, double **edges, int64_t *num_edges);
/* The same into float, as read_TO_edges_from_file<float> reads (each number
 * converted straight to float, not through double); text files only. */
int cvl_read_edges_f32(const char *path, int32_t values_per_edge, int32_t nthreads, float **edges,
                       int64_t *num_edges);
/* Frees the rows of cvl_read_edges or cvl_read_edges_f32. */
void cvl_free_edges(void *edges);
/* Binary edge file: "CVLEDGE1", uint32 values_per_edge, uint32 0, uint64
 * num_edges, then the rows as little-endian doubles (no reference counterpart). */
int cvl_write_edges_binary(const char *path, const double *edges, int64_t num_edges, int32_t values_per_edge);

/* ---- tuning and the autotuner -------------------------------------------
 * No reference counterpart. An engine keeps one tuning per size bucket of the
 * batch (its total edges); every tuning gives the same results bit for bit,
 * only the time changes. cvl_engine_autotune searches them on a
 * device-resident batch by timing the whole path, and installs the best. */
#define CVL_TUNING_BUCKETS 4          /* batches of <= 64 Ki, <= 512 Ki, <= 4 Mi, and more edges */
typedef struct cvl_tuning {
    int cell_size;                    /* spatial-hash block edge in pixel cells: 2, 4 or 8 (4; 8 above 512 Ki edges) */
    int bundle_blocks_per_sm;         /* bundle kernel's register budget: 3 or 4 resident blocks per SM (4) */
    int growth_blocks_per_sm;         /* growth kernel's register budget: 4, 6 or 8 resident blocks of 4 warps per SM
                                         (8: 63 registers; grids other than the default 63-cell one take 6 for 8) */
    int seeds_per_group;              /* chain-growth seeds walked together per warp: 4 or 8 (4) */
    int anchors_per_warp;             /* chain-growth anchors per warp: 1..32 (8) */
    int64_t chunk_pairs;              /* neighbour pairs whose bundles are held in HBM at once (4 Mi; 8 Mi above 4 Mi edges) */
} cvl_tuning;
/* The bucket a batch of num_edges edges uses. */
int cvl_tuning_bucket(int64_t num_edges);
int cvl_engine_get_tuning(cvl_engine *e, int bucket, cvl_tuning *t);
/* bucket -1 sets every bucket. CVL_EINVAL for values outside the ranges above. */
int cvl_engine_set_tuning(cvl_engine *e, int bucket, const cvl_tuning *t);
/* Coordinate descent over the tuning of the batch's bucket. It runs `passes`
 * sweeps over the knobs, each candidate timed as the median of 3 runs of the
 * whole path (device time), and keeps a change only when it is faster by more
 * than 1%. The best tuning is installed for that bucket and written to *best,
 * and its time to *best_ms. The batch's results are not kept. */
int cvl_engine_autotune(cvl_engine *e, const cvl_batch *b, const cvl_params *p, int passes, cvl_tuning *best,
                        double *best_ms);

/* ---- workspace by shape ------------------------------------------------
 * No reference counterpart (the reference allocates its worst case,
 * N (max_degree + 1) 2 output rows, per run: cpu_curvelet.hpp:59-67). The
 * engine sizes its device workspace to each launch: buffers grow when a launch
 * needs more than any before it, and are kept. The shape of a launch is what
 * decides the sizes: */
typedef struct cvl_workspace_shape {
    int64_t num_edges;      /* edges of the launch, all maps together */
    int64_t num_pairs;      /* neighbour pairs (total_neighbor_pairs) */
    int64_t num_curvelets;  /* curvelets written (at most num_pairs: each seed grows at most one) */
    int32_t num_maps;       /* maps folded into the launch */
    int32_t edge_data_sz;   /* values per edge row (4) */
} cvl_workspace_shape;
/* Device bytes of the workspace a launch of that shape takes on this engine (its
 * tuning sets the bundle chunk), the launch's input rows included, in *total; of
 * that, the one bundle chunk a launch holds whatever its maps, in *per_launch
 * (may be NULL). */
int cvl_engine_workspace_bytes(cvl_engine *e, const cvl_workspace_shape *s, const cvl_params *p, size_t *total,
                               size_t *per_launch);
/* Allocates the workspace of that shape now, so that later runs within it (edges,
 * pairs, curvelets and maps at most the shape's) allocate no device memory: cvl_run
 * and cvl_batch_run (a batch holds its own rows: cvl_batch_refill reuses a buffer
 * large enough). */
int cvl_engine_reserve_workspace(cvl_engine *e, const cvl_workspace_shape *s, const cvl_params *p);
/* The engine's device memory: bytes its workspace and batches hold, and the
 * allocations made so far with their host time. */
typedef struct cvl_engine_memory {
    size_t held_bytes;
    uint64_t device_grows;
    double device_grow_ms;
} cvl_engine_memory;
int cvl_engine_memory_get(cvl_engine *e, cvl_engine_memory *out);

/* ---- CUDA graphs of the path ------------------------------------------
 * No reference counterpart. A run (cvl_run, cvl_batch_run, ...) of up to 64 Ki
 * edges (tuning bucket 0) or 512 Ki edges (bucket 1), in double, replays a CUDA
 * graph of the whole path captured for the bucket's capacities (edges, 4,096
 * maps, 2 or 8 bundle chunks, 8 curvelets per edge): the kernels read the run's
 * sizes from device memory, so one graph serves every run of its bucket, with
 * one host synchronisation where the kernel-by-kernel path has three. A graph is
 * captured on a bucket's first run and again when the parameters, the tuning or
 * the buffers change (up to 6 kept per engine). A run beyond a capacity is
 * flagged on the device and run again kernel by kernel; the results are the same
 * either way. CVL_NO_GRAPHS in the environment turns graphs off for new engines. */
int cvl_engine_set_graphs(cvl_engine *e, int enable);
typedef struct cvl_engine_graphs {
    int32_t enabled;
    int32_t graphs;      /* captured graphs held */
    uint64_t captures;   /* graphs captured so far */
    uint64_t replays;    /* runs that replayed a graph */
    uint64_t fallbacks;  /* of those, runs beyond a capacity, run again kernel by kernel */
} cvl_engine_graphs;
int cvl_engine_graph_stats(cvl_engine *e, cvl_engine_graphs *out);

/* Writes a buffer larger than the L2 cache on the engine's stream and waits
 * (timing hygiene between benchmark iterations). */
int cvl_engine_flush_l2(cvl_engine *e);

/* Per-kernel device times (ms) of the engine's last run: fills up to cap
 * entries of names/ms and returns the count (or a negative status). */
int cvl_engine_last_kernel_times(cvl_engine *e, const char **names, double *ms, int cap);

/* Kernels the engine launched in its last run (>= 0), or a negative status. */
int cvl_engine_last_launch_count(cvl_engine *e);

/* Measures the device's FP64 FMA throughput (TFLOP/s, 2 flops per FMA) with a
 * register-resident dependent-chain loop; the roofline denominator for the
 * FP64-bound bundle kernel. */
int cvl_measure_fp64_peak(cvl_engine *e, double *tflops);

/* ---- Downstream: curvelets -> edgel link graph -> contour fragments ----------
 * The reference's original_code stage after curvelet formation:
 *   form_curvelet_process::construct_the_link_graph   (form_curvelet_process.cpp:453-520)
 *   form_curvelet_process::extract_regular_contours_from_the_link_graph and
 *   extract_one_chains_from_the_link_graph            (form_curvelet_process.cpp:529-654)
 *   edgel_link_graph, curve_fragment_graph            (edgel_link_graph.hpp, curve_fragment_graph.hpp)
 * Every curvelet with at least min_group_size edges links its consecutive edges
 * (a link joins two edges in either direction; its direction is that of its first
 * occurrence, anchors ascending); one-chains are then traced from each legal
 * start edge in ascending id order, a step taken only while the two edges are
 * closer than gap, and chains of more than 2 edges are kept. */
typedef struct cvl_contour_params {
    uint32_t min_group_size; /* construct_the_link_graph(4, ...), form_curvelet_process.cpp:79 */
    double gap;              /* 1.5, original_code/main.cpp:146 */
    /* C^1 polyarcs along the fragments: fit_polyarcs_to_all_edgel_chains
     * (form_curvelet_process.cpp:661-796), output type 2 of original_code/main.cpp.
     * The bundle grid steps are CC_curve_model_3d's fixed 0.1 px and 0.08 rad. */
    int fit_polyarcs;        /* 1: fit them (0) */
    double dx;               /* position uncertainty, px (0.4, main.cpp:148) */
    double dt_rad;           /* orientation uncertainty, rad ((15/180) pi, main.cpp:149) */
    double max_k;            /* curvature bound (0.3, main.cpp:151) */
    double rad;              /* compute_properties' R: the grouping radius (3.5, main.cpp:145) */
    double token_len;        /* compute_properties' token length (1, main.cpp:150) */
} cvl_contour_params;

void cvl_contour_params_default(cvl_contour_params *p);

typedef struct cvl_contours cvl_contours;

/* Links in _cLinks order (parent id ascending, then creation order) and fragments
 * in the order of their start edge (curve_fragment_graph::_frags). All ids are
 * 0-based edge indices. Arrays live in page-locked memory owned by the result. */
typedef struct cvl_contours_view {
    int64_t num_links;
    const int32_t *link_parent; /* edgel_link::_pe */
    const int32_t *link_child;  /* edgel_link::_ce */
    const int32_t *link_votes;  /* edgel_link::_vote */
    int64_t num_fragments;
    const int64_t *fragment_offsets; /* [num_fragments + 1] */
    const int32_t *fragment_ids;
    int32_t max_fragment_length; /* curve_fragment_graph::edgel_chain_max_length */
    int32_t num_edges;
    float device_ms; /* the stage's device time (cvl_run_contours: the whole path) */
    /* polyarcs (fit_polyarcs = 1; else 0 and NULL), polyarcmap order: fragments in
     * order, each one's polyarcs from its start. Each polyarc's chain is a run of
     * its fragment's ids. info columns per curvelet::set_output (curvelet.cpp:132-144,
     * CC_curve_model_3d.cpp:530-545): 0 forward (1), 1-2 the best cell's k_max and
     * k_min, 3 the start edge's orientation, 4-5 its position, 6 theta, 7 k, 8 length,
     * 9 quality, 10-11 the arc's centre (0 for a line: the reference leaves them unset). */
    int64_t num_polyarcs;
    const int64_t *polyarc_offsets; /* [num_polyarcs + 1] into polyarc_ids */
    const int32_t *polyarc_ids;     /* 0-based edge ids */
    const double *polyarc_info;     /* [num_polyarcs][12] */
} cvl_contours_view;

/* The stage on curvelets the caller holds: chains as cvl_result_view gives them
 * ([num_curvelets][chain_width], column 0 = anchor + 1, then the chain, 1-based,
 * zero-padded), rows grouped by anchor in ascending order. CVL_EINVAL for ids
 * outside the map, rows out of anchor order, or chain_width outside [2, 64]. */
int cvl_link_contours(cvl_engine *e, const double *edges, int32_t num_edges, int32_t edge_data_sz,
                      const uint32_t *chains, int64_t num_curvelets, int32_t chain_width,
                      const cvl_contour_params *cp, cvl_contours **out);

/* Edges -> curvelets -> link graph -> fragments in one pass on the device (the
 * curvelets never leave it). curvelets_out may be NULL; otherwise it receives
 * the curvelets as cvl_run returns them. cp NULL: the defaults, with p->gap. */
int cvl_run_contours(cvl_engine *e, const double *edges, int32_t num_edges, int32_t edge_data_sz,
                     const cvl_params *p, const cvl_contour_params *cp, cvl_result **curvelets_out,
                     cvl_contours **out);

int cvl_contours_get(const cvl_contours *c, cvl_contours_view *view);
void cvl_contours_free(cvl_contours *c);

#ifdef __cplusplus
}
#endif

#endif /* CVL_H */
