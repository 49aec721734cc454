// cvl_engine.cu -- host engine and C ABI (include/cvl.h) of the curvelet path.
//
// One engine = one CUDA device + one stream + a grow-only device workspace.
// A run over a ragged batch of maps (a single map for the plain form):
//   H2D edges -> (a) binning -> (b) neighbour count, scan -> [sync: pair total]
//   -> (b) neighbour fill -> (c+d) fused bundles/growth/dedup/record
//   -> scan of per-anchor counts -> [sync: curvelet total] -> (e) finalize -> D2H
// The two syncs size the CSR/record and output buffers exactly; everything
// else stays on the device.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda.h>
#include <nvtx3/nvToolsExt.h>

#include "../../include/cvl.h"
#include "cvl_internal.h"
#include "cvl_pinned.h"
#include "cvl_contours.cuh"
#include "cvl_path.cuh"
#include "cvl_polyarcs.cuh"
#include "cvl_scan.cuh"

using namespace cvl;

namespace {

thread_local std::string g_err;

int fail(int code, const std::string &msg) {
    g_err = msg;
    return code;
}

#define CVL_CUDA(call)                                                                         \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail(CVL_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CVL_TRY(call)              \
    do {                           \
        int rc_ = (call);          \
        if (rc_ != CVL_OK) return rc_; \
    } while (0)

struct DBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

int g_launches_snapshot();

// Pairs per bundle chunk: a chunk's bundles (1 KB per pair for the default grid)
// stay in device memory between the transport and growth kernels.
constexpr unsigned long long CHUNK_PAIRS_DEFAULT = 4ull << 20;

inline unsigned next_pow2(unsigned long long v) {
    unsigned long long p = 1;
    while (p < v) p <<= 1;
    return (unsigned)p;
}

}  // namespace

int cvl_fail(int code, const std::string &msg) { return fail(code, msg); }

// ---- allocation-failure injector ----------------------------------------------------
// Allocations left before every device or page-locked allocation of the library
// fails as if the memory were exhausted; -1: off. Armed by cvl_debug_fail_allocations
// or, when the library loads, by CVL_FAIL_ALLOC_AFTER=<k> in the environment.
static std::atomic<int64_t> g_fail_after{[] {
    const char *v = std::getenv("CVL_FAIL_ALLOC_AFTER");
    return v ? (int64_t)std::strtoll(v, nullptr, 10) : (int64_t)-1;
}()};

bool cvl_alloc_fault_injected() {
    int64_t left = g_fail_after.load();
    while (left > 0) {
        if (g_fail_after.compare_exchange_weak(left, left - 1)) return false;
    }
    return left == 0;
}

void cvl_engine_set_yield(cvl_engine *e, cvl_yield_fn fn, void *ctx);

// Results live in page-locked memory (cvl::PinnedArena): device-to-host copies
// at full PCIe/C2C rate and no per-call pinning. The arena is shared by the
// engine and its live results, so a result may outlive its engine.
using PinnedPool = cvl::PinnedArena;

struct cvl_engine {
    int device = 0;
    cudaStream_t stream = nullptr;
    // The workspace comes from the engine's own stream-ordered pool: growing a
    // buffer frees the old one in stream order (cudaFreeAsync) instead of with
    // cudaFree, which would wait for every stream of the device (other engines'
    // work included). The pool keeps what it has (release threshold: no limit).
    cudaMemPool_t pool = nullptr;
    cudaDeviceProp prop{};
    size_t budget = 0;
    size_t held = 0;
    std::atomic<uint64_t> dev_grows{0}, dev_grow_ns{0};  // workspace allocations and their host time
    int cell_size = 4;
    int seeds_per_group = 4;
    int slots = 10;
    unsigned long long generation = 0;
    std::shared_ptr<PinnedPool> pinned = std::make_shared<PinnedPool>();

    // workspace
    DBuf edges, map_off, ehash, bcount, bstart, bfill, pos_of, orig_of;
    DBuf bx, by, bth, bsp, bcp, bsm, bcm, bcell, bmap;
    DBuf ncand, deg, pair_off, csr_ids, csr_d2, rec_ids, rec_k, rec_meta, count, out_off;
    DBuf chains, info, stats, err, work, scratch, scratch_chain, scratch_res, scan_tmp, flush, deg_orig, off_orig,
        gids, gd2, run_cnt, rec_base, pcls, pflag, pair_anchor, atrig, bund, chunk_start, crank;
    cvl_tuning tune[CVL_TUNING_BUCKETS];                   // per size bucket of the batch
    cvl_yield_fn yield_fn = nullptr;                       // called between chunks (serving)
    void *yield_ctx = nullptr;
    cudaEvent_t chunk_done = nullptr;
    std::vector<cvl_batch *> batches;                      // live batches, freed with the engine
    unsigned long long arena_hint = 0;  // record arena size that the last input needed
    DBuf pairs_in, pb_min, pb_max, pb_valid;
    // cvl_run_device: what its last run left on the device
    unsigned long long dev_curvelets = 0;
    int dev_width = 0;
    unsigned long long dev_generation = ~0ull;
    cudaEvent_t dev_done = nullptr;
    // cvl_run_maps: the other group's outputs, a copy stream and its events
    DBuf chains_alt, info_alt, edges_alt;
    cudaStream_t copy_stream = nullptr;
    cudaStream_t upload_stream = nullptr;  // cvl_run_maps: the next group's edges
    cudaEvent_t uploaded[2] = {nullptr, nullptr}, consumed[2] = {nullptr, nullptr};
    cudaEvent_t computed[2] = {nullptr, nullptr};
    cudaEvent_t copied[2] = {nullptr, nullptr};
    // downstream stage (link graph, contour fragments)
    struct ContourBufs {
        DBuf chains_in, cnt, off, cursor, bucket, outdeg, indeg, child, parent, succ, pred, flags, linked, firsts,
            region, ctr, fsrc, fnf, fnb, isfrag, flen, fidx, idoff, loff, lpe, lce, lvotes, fragoff, fragids, err,
            pstart, psize, pinfo, pcount, poff, pstart2, psize2, pinfo2;
        DBuf *all(int i) {
            DBuf *b[] = {&chains_in, &cnt, &off, &cursor, &bucket, &outdeg, &indeg, &child, &parent, &succ,
                         &pred, &flags, &linked, &firsts, &region, &ctr, &fsrc, &fnf, &fnb, &isfrag,
                         &flen, &fidx, &idoff, &loff, &lpe, &lce, &lvotes, &fragoff, &fragids, &err,
                         &pstart, &psize, &pinfo, &pcount, &poff, &pstart2, &psize2, &pinfo2};
            return i < (int)(sizeof(b) / sizeof(b[0])) ? b[i] : nullptr;
        }
    } cw;

    // CUDA graphs of the path for the small size buckets: each captured once for a
    // key (parameters, buffers, input pointers) and replayed for every run whose sizes
    // fit the bucket's capacities (the kernels read the run's sizes on the device)
    struct GraphSlot {
        std::string key;
        cudaGraphExec_t exec = nullptr;
        int launches = 0;
        uint64_t last_use = 0;
    };
    std::vector<GraphSlot> graphs;
    bool graphs_on = std::getenv("CVL_NO_GRAPHS") == nullptr;
    // direct runs on queue-pulling persistent grids (CVL_NO_PERSIST: short blocks)
    bool persist_on = std::getenv("CVL_NO_PERSIST") == nullptr;
    // the transport's k_dx quotient pairs on one reciprocal (CVL_NO_SHARED_QUOTIENTS: divisions)
    bool shared_quot_on = std::getenv("CVL_NO_SHARED_QUOTIENTS") == nullptr;
    uint64_t ws_epoch = 0;                         // workspace (re)allocations so far
    uint64_t graph_replays = 0, graph_fallbacks = 0, graph_captures = 0, graph_clock = 0;
    DBuf gdims, gchunks, gread;
    unsigned char *gread_host = nullptr;           // page-locked: the runs' sizes and the readback

    // per-kernel timing of the last run
    std::vector<const char *> mark_names;
    std::vector<cudaEvent_t> marks;
    size_t nmarks = 0;
    std::vector<std::pair<const char *, double>> last_times;
    double last_device_ms = 0.0;

    int alloc(DBuf &b, size_t bytes) {
        if (bytes == 0) bytes = 16;
        if (b.bytes >= bytes) return CVL_OK;
        size_t want = std::max(bytes, b.bytes + b.bytes / 2);
        want = (want + 255) & ~(size_t)255;
        if (b.p) {
            cudaFreeAsync(b.p, stream);
            held -= b.bytes;
            b.p = nullptr;
            b.bytes = 0;
        }
        if (budget && held + want > budget) {
            want = bytes;
            if (held + want > budget)
                return fail(CVL_ENOMEM, "device memory budget exceeded (" + std::to_string(held + want) + " > " +
                                            std::to_string(budget) + " bytes)");
        }
        const auto t_grow = std::chrono::steady_clock::now();
        cudaError_t e = cvl_alloc_fault_injected() ? cudaErrorMemoryAllocation
                                                   : cudaMallocFromPoolAsync(&b.p, want, pool, stream);
        dev_grow_ns += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                           std::chrono::steady_clock::now() - t_grow).count();
        ++dev_grows;
        if (e != cudaSuccess) {
            b.p = nullptr;
            cudaGetLastError();
            return fail(CVL_ENOMEM, std::string("device allocation of ") + std::to_string(want) +
                                        " bytes: " + cudaGetErrorString(e));
        }
        b.bytes = want;
        held += want;
        ++ws_epoch;
        return CVL_OK;
    }

    void mark(const char *name) {
        if (nmarks == marks.size()) {
            cudaEvent_t ev;
            cudaEventCreate(&ev);
            marks.push_back(ev);
            mark_names.push_back(name);
        }
        mark_names[nmarks] = name;
        cudaEventRecord(marks[nmarks], stream);
        ++nmarks;
        nvtxMarkA(name);  // the stage's end on the host timeline (profilers)
    }

    int last_launches = 0;

    void collect_marks() {
        last_launches = g_launches_snapshot();
        last_times.clear();
        last_device_ms = 0.0;
        if (nmarks < 2) return;
        cudaEventSynchronize(marks[nmarks - 1]);
        for (size_t k = 1; k < nmarks; ++k) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, marks[k - 1], marks[k]);
            last_times.emplace_back(mark_names[k], (double)ms);
        }
        float tot = 0.f;
        cudaEventElapsedTime(&tot, marks[0], marks[nmarks - 1]);
        last_device_ms = tot;
    }

    void release_all() {
        DBuf *all[] = {&edges, &map_off, &ehash, &bcount, &bstart, &bfill, &pos_of, &orig_of, &bx, &by, &bth, &bsp,
                       &bcp, &bsm, &bcm, &bcell, &bmap, &ncand, &deg, &pair_off, &csr_ids, &csr_d2, &rec_ids,
                       &rec_k, &rec_meta, &count, &out_off, &chains, &info, &stats, &err, &work, &scratch,
                       &scratch_chain, &scratch_res, &run_cnt, &rec_base, &pcls, &pflag, &pair_anchor, &atrig, &bund, &chunk_start, &crank, &scan_tmp, &flush, &deg_orig, &off_orig, &gids, &gd2, &pairs_in, &pb_min,
                       &pb_max, &pb_valid, &chains_alt, &info_alt, &edges_alt, &gdims, &gchunks, &gread};
        for (DBuf *b : all) {
            if (b->p) cudaFreeAsync(b->p, stream);
            b->p = nullptr;
            b->bytes = 0;
        }
        for (int i = 0; DBuf *b = cw.all(i); ++i) {
            if (b->p) cudaFreeAsync(b->p, stream);
            b->p = nullptr;
            b->bytes = 0;
        }
        held = 0;
    }
};

struct cvl_result {
    std::shared_ptr<PinnedPool> pool;
    void *chains_p = nullptr;  // pinned, from pool
    void *info_p = nullptr;
    cvl_result_view v{};
    ~cvl_result() {
        if (pool) {
            pool->put(chains_p);
            pool->put(info_p);
        }
    }
};

struct cvl_graph {
    std::vector<double> edges;  // AoS copy, edge_data_sz per row
    int sz = 4;
    int n = 0;
    double rad = 3.5;
    unsigned neighbor_radius = 3;
    unsigned max_candidates = 128;
    std::vector<int32_t> offsets, ids;
    std::vector<double> d2;
    cvl_graph_view v{};
};

struct cvl_batch {
    cvl_engine *eng = nullptr;
    void *d_edges = nullptr;
    void *d_map_off = nullptr;
    size_t edges_cap = 0;    // bytes allocated at d_edges
    size_t map_off_cap = 0;  // entries allocated at d_map_off
    int num_maps = 0;
    int sz = 4;
    int n = 0;
    std::vector<int32_t> map_off;
};

struct cvl_batch_result {
    cvl_engine *eng = nullptr;
    unsigned long long generation = 0;
    std::shared_ptr<PinnedPool> pinned;
    int num_maps = 0;
    int n = 0;
    int width = 0;
    std::vector<int32_t> map_off;
    std::vector<MapStats> stats;
    std::vector<unsigned long long> cv_off;  // per-map curvelet offsets [M+1]
    double device_ms = 0.0;
    int launches = 0;
    bool downloaded = false;
    uint32_t *chains = nullptr;  // pinned, from the engine's pool (all maps)
    double *info = nullptr;
    bool truncated_any = false;
    ~cvl_batch_result() {
        if (pinned) {
            pinned->put(chains);
            pinned->put(info);
        }
    }
};

namespace {

// ---- tuning -------------------------------------------------------------------
int bucket_of(long long n) {
    if (n <= (64LL << 10)) return 0;
    if (n <= (512LL << 10)) return 1;
    if (n <= (4LL << 20)) return 2;
    return 3;
}

cvl_tuning default_tuning(int cell_size, int seeds_per_group) {
    cvl_tuning t;
    t.cell_size = cell_size;
    t.bundle_blocks_per_sm = 4;
    // measured on the 64-map batch: 8 (63 registers, 32 one-warp blocks per SM) 174.8 ms,
    // 6 (72 registers) 187.3 ms, 4 slower still; grids other than the default take 6 for 8
    t.growth_blocks_per_sm = 8;
    t.seeds_per_group = seeds_per_group;
    t.anchors_per_warp = 8;
    t.chunk_pairs = (int64_t)CHUNK_PAIRS_DEFAULT;
    return t;
}

int check_tuning(const cvl_tuning &t) {
    if (t.cell_size != 2 && t.cell_size != 4 && t.cell_size != 8)
        return fail(CVL_EINVAL, "tuning: cell_size must be 2, 4 or 8");
    if (t.bundle_blocks_per_sm != 3 && t.bundle_blocks_per_sm != 4)
        return fail(CVL_EINVAL, "tuning: bundle_blocks_per_sm must be 3 or 4");
    if (t.growth_blocks_per_sm != 4 && t.growth_blocks_per_sm != 6 && t.growth_blocks_per_sm != 8)
        return fail(CVL_EINVAL, "tuning: growth_blocks_per_sm must be 4, 6 or 8");
    if (t.seeds_per_group != 4 && t.seeds_per_group != 8) return fail(CVL_EINVAL, "tuning: seeds_per_group must be 4 or 8");
    if (t.anchors_per_warp < 1 || t.anchors_per_warp > 32) return fail(CVL_EINVAL, "tuning: anchors_per_warp in [1, 32]");
    if (t.chunk_pairs < (1 << 16) || t.chunk_pairs > (1LL << 30))
        return fail(CVL_EINVAL, "tuning: chunk_pairs in [65536, 2^30]");
    return CVL_OK;
}

// ---- parameters -> model ---------------------------------------------------
// The model of run_curvelet<T> (main.cpp:21-29): parameters converted to T as
// the reference converts them, and its derived constants computed in T.
template <typename T>
int make_model(const cvl_engine *e, const cvl_params *p, double rad, unsigned nbr_radius, unsigned max_cand,
               ModelT<T> &md, int &cpl) {
    if (!p) return fail(CVL_EINVAL, "params is NULL");
    if (!(p->sx > 0) || !(p->st > 0)) return fail(CVL_EINVAL, "sx and st must be > 0");
    if (!std::isfinite(p->dx) || !std::isfinite(p->dt_deg) || !std::isfinite(p->dt_rad) || !std::isfinite(p->max_k) || !std::isfinite(p->nrad) ||
        !std::isfinite(rad))
        return fail(CVL_EINVAL, "non-finite parameter");
    if (p->group_max_sz < 1 || p->group_max_sz > (unsigned)GMS_MAX)
        return fail(CVL_EUNSUPPORTED, "group_max_sz must be in [1, 16]");
    if (max_cand < 1 || max_cand > 1024) return fail(CVL_EUNSUPPORTED, "max_candidates must be in [1, 1024]");
    if (nbr_radius > 64) return fail(CVL_EUNSUPPORTED, "neighbor_radius must be <= 64");
    md.nrad = T(p->nrad);
    const T rad_t = T(rad);
    md.rad_sqr = rad_t * rad_t;  // rad * rad (preprocess.hpp:221)
    md.dx = T(p->dx);
    md.dx2 = md.dx * md.dx;
    md.four_dx_dx = T(4) * md.dx * md.dx;
    md.dt = (p->dt_rad > 0) ? T(p->dt_rad) : T(p->dt_deg / 180.0) * T(CVL_PI);  // main.cpp:24
    md.sx = T(p->sx);
    md.st = T(p->st);
    md.max_k = T(p->max_k);
    const double Pd = 2 * std::floor((double)(md.dx / md.sx) + 0.5) + 1;  // cpu_curvelet.hpp:73
    const double Qd = 2 * std::floor((double)(md.dt / md.st) + 0.5) + 1;  // cpu_curvelet.hpp:74
    if (!(Pd >= 1 && Pd <= 128 && Qd >= 1 && Qd <= QMAX))
        return fail(CVL_EUNSUPPORTED, "bundle grid out of range (P <= 128, Q <= 32 required)");
    md.P = (int)Pd;
    md.Q = (int)Qd;
    md.cells = md.P * md.Q;
    if (md.cells > 128) return fail(CVL_EUNSUPPORTED, "bundle grid larger than 128 cells");
    cpl = (md.cells + 31) / 32;
    md.gms = (int)p->group_max_sz;
    md.max_cand = (int)max_cand;
    md.w = (int)nbr_radius;
    {
        // hash block edge: a power of two (the block of a pixel cell is cell >> sbits)
        const int S = (e && e->cell_size > 0) ? e->cell_size : 4;
        int sb = 0;
        while ((1 << sb) < S && sb < 6) ++sb;
        if ((1 << sb) != S) return fail(CVL_EINVAL, "cell_size must be a power of two in [1, 64]");
        md.sbits = sb;
    }
    md.hash_mask = 0;
    // the FP64 transport's shared-reciprocal quotients need dx and sx in [2^-40, 2^40]
    // (certify_* in cvl_kernels.cuh covers the run's own operands)
    md.shared_quot = (std::is_same<T, double>::value && (!e || e->shared_quot_on) && p->dx >= 0x1p-40 &&
                      p->dx <= 0x1p40 && p->sx >= 0x1p-40 && p->sx <= 0x1p40)
                         ? 1
                         : 0;
    return CVL_OK;
}

// CVL_SYNC_CHECK=1 in the environment synchronizes after every launch so that a
// device-side error is reported against the kernel that raised it.
const bool g_sync_check = std::getenv("CVL_SYNC_CHECK") != nullptr;

// kernels launched by this thread since the last run started (cvl_engine_last_launch_count)
thread_local int g_launches = 0;

int g_launches_snapshot() { return g_launches; }

int check_launch(const char *what) {
    ++g_launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CVL_ECUDA, std::string("launch ") + what + ": " + cudaGetErrorString(e));
    if (g_sync_check) {
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) return fail(CVL_ECUDA, std::string("kernel ") + what + " failed: " + cudaGetErrorString(e));
    }
    return CVL_OK;
}

// Host<->device copies in pieces of at most 32 MiB: the copy engines take
// commands in turn across streams, so a large map's transfer does not hold up
// a small map's for the whole of its length.
cudaError_t copy_pieces(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s) {
    constexpr size_t PIECE = (size_t)32 << 20;
    for (size_t o = 0; o < bytes; o += PIECE) {
        const cudaError_t ce =
            cudaMemcpyAsync((char *)dst + o, (const char *)src + o, std::min(PIECE, bytes - o), kind, s);
        if (ce != cudaSuccess) return ce;
    }
    return cudaSuccess;
}

// Device -> page-locked host copy of results. RESULT_COPY_SM (the default) copies with a
// small kernel (RESULT_COPY_BLOCKS blocks), which slows concurrent path kernels far less
// than a copy-engine transfer does; CVL_RESULT_COPY=ce in the environment selects the
// copy engine (cudaMemcpyAsync in pieces). A copy that no path kernel runs beside
// (alone) takes the copy engine, which is faster (53 against 38 GB/s measured).
constexpr int RESULT_COPY_BLOCKS = 16;
const bool g_result_copy_sm = [] {
    const char *v = std::getenv("CVL_RESULT_COPY");
    return !(v && std::strcmp(v, "ce") == 0);
}();

cudaError_t copy_pieces(void *dst, const void *src, size_t bytes, cudaMemcpyKind kind, cudaStream_t s);

inline cudaError_t copy_result_to_host(void *dst, const void *src, size_t bytes, cudaStream_t s, bool alone = false) {
    if (!bytes) return cudaSuccess;
    if (alone || !g_result_copy_sm || (bytes & 3) || (((uintptr_t)src | (uintptr_t)dst) & 3))
        return copy_pieces(dst, src, bytes, cudaMemcpyDeviceToHost, s);
    const int wide = ((((uintptr_t)src | (uintptr_t)dst) | bytes) & 15) == 0 ? 1 : 0;
    k_copy_to_host<<<RESULT_COPY_BLOCKS, 256, 0, s>>>(src, dst, bytes, wide);
    return cudaGetLastError();
}

// Grids of short blocks: `per_block` work items per block and no cap, so a
// kernel of a large map never holds an SM for long and a higher-priority
// stream's blocks start as soon as any block ends (the kernels stride over
// their items, so any grid is correct).
inline int short_grid(long long n, long long per_block) {
    long long g = (n + per_block - 1) / per_block;
    return (int)std::max(1LL, std::min(g, 0x7fffffffLL));
}

inline int grid_for(const cvl_engine *e, long long n, int threads, int per_sm = 16) {
    long long g = (n + threads - 1) / threads;
    const long long cap = (long long)e->prop.multiProcessorCount * per_sm;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

// ---- scans -------------------------------------------------------------------
template <typename TIn, typename TOut>
int scan_rec(cvl_engine *e, const TIn *in, size_t n, TOut *out, char *&tmp, size_t &left) {
    if (n == 0) {
        CVL_CUDA(cudaMemsetAsync(out, 0, sizeof(TOut), e->stream));
        return CVL_OK;
    }
    const size_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
    if (nb == 1) {
        k_scan_tiles<TIn, TOut><<<1, SCAN_THREADS, 0, e->stream>>>(in, n, nullptr, out);
        return check_launch("k_scan_tiles");
    }
    const size_t need = (2 * nb + 1) * sizeof(TOut);
    if (need > left) return fail(CVL_EOVERFLOW, "scan temp too small");
    TOut *sums = (TOut *)tmp;
    TOut *offs = sums + nb;
    tmp += need;
    left -= need;
    k_scan_reduce<TIn, TOut><<<(unsigned)nb, SCAN_THREADS, 0, e->stream>>>(in, n, sums);
    CVL_TRY(check_launch("k_scan_reduce"));
    CVL_TRY((scan_rec<TOut, TOut>(e, sums, nb, offs, tmp, left)));
    k_scan_tiles<TIn, TOut><<<(unsigned)nb, SCAN_THREADS, 0, e->stream>>>(in, n, offs, out);
    return check_launch("k_scan_tiles");
}

template <typename TIn, typename TOut>
int scan(cvl_engine *e, const TIn *in, size_t n, TOut *out) {
    const size_t tmp_bytes = (n / SCAN_TILE + 64) * 4 * sizeof(unsigned long long) + 4096;
    CVL_TRY(e->alloc(e->scan_tmp, tmp_bytes));
    char *tmp = (char *)e->scan_tmp.p;
    size_t left = e->scan_tmp.bytes;
    return scan_rec<TIn, TOut>(e, in, n, out, tmp, left);
}

// ---- the pipeline -------------------------------------------------------------
struct RunOut {
    std::vector<MapStats> stats;
    std::vector<unsigned long long> cv_off;  // per map
    unsigned long long total_pairs = 0;
    unsigned long long total_curvelets = 0;
    unsigned max_deg = 0;
};

template <typename T, int CPL, int MINB>
int launch_bundles(cvl_engine *e, BundleArgsT<T> &a, int blocks) {
    // one block per PPB pairs and no grid stride: short blocks, so that a
    // higher-priority stream's blocks get SMs as soon as any block ends
    constexpr int pair_bytes = 2 * 32 * CPL * (int)sizeof(T);
    const long long ppb = bundles_pairs_per_block(a.md.Q, pair_bytes);
    if (!a.cd && !a.queue) {  // a graph run or a queue-pulling grid keeps the given grid
        const long long need = ((long long)(a.p_end - a.p_begin) + ppb - 1) / ppb;
        blocks = (int)std::max(1LL, std::min<long long>(need, 0x7fffffffLL));
    }
    if constexpr (std::is_same<T, double>::value) {
        const size_t smem = (size_t)ppb * pair_bytes;
        if (a.shared_quot) {  // the k_dx quotient pairs on one reciprocal
            if (a.queue)
                k_bundles<T, CPL, MINB, true, QUOT_SHARED><<<blocks, BUNDLE_THREADS, smem, e->stream>>>(a);
            else
                k_bundles<T, CPL, MINB, false, QUOT_SHARED><<<blocks, BUNDLE_THREADS, smem, e->stream>>>(a);
            return check_launch("k_bundles");
        }
        if (a.queue) {  // the queue-pulling variant
            k_bundles<T, CPL, MINB, true><<<blocks, BUNDLE_THREADS, smem, e->stream>>>(a);
            return check_launch("k_bundles");
        }
    }
    k_bundles<T, CPL, MINB><<<blocks, BUNDLE_THREADS, (size_t)ppb * pair_bytes, e->stream>>>(a);
    return check_launch("k_bundles");
}

template <typename T, int CPL, int K, int MINB>
int launch_growth(cvl_engine *e, GrowthArgsT<T> &a, size_t smem, int blocks) {
    if constexpr (std::is_same<T, double>::value) {
        if (a.queue) {  // a graph run: the queue-pulling variant on the given persistent grid
            CVL_CUDA(cudaFuncSetAttribute(k_growth<T, CPL, K, MINB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem));
            k_growth<T, CPL, K, MINB, true><<<blocks, GROWTH_THREADS, smem, e->stream>>>(a);
            return check_launch("k_growth");
        }
    }
    CVL_CUDA(cudaFuncSetAttribute(k_growth<T, CPL, K, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (!a.cd && !a.queue) {  // a graph run or a queue-pulling grid keeps the given grid
        // a warp per anchor and anchors_per_warp anchors per warp: short blocks (a
        // higher-priority stream's blocks get SMs as soon as any block ends)
        const long long per_block = (GROWTH_THREADS / 32) * (long long)a.anchors_per_warp;
        blocks = (int)std::max(1LL, std::min<long long>(((long long)a.a_end - a.a_begin + per_block - 1) / per_block,
                                                        0x7fffffffLL));
    }
    k_growth<T, CPL, K, MINB><<<blocks, GROWTH_THREADS, smem, e->stream>>>(a);
    return check_launch("k_growth");
}

template <typename T>
using bundles_fn = int (*)(cvl_engine *, BundleArgsT<T> &, int);
template <typename T>
using growth_fn = int (*)(cvl_engine *, GrowthArgsT<T> &, size_t, int);

// Float mode (a parity mode) runs the default variants only.
void pick_kernels(int cpl, const cvl_tuning &, bundles_fn<float> &bf, growth_fn<float> &gf) {
    switch (cpl) {
        case 1: bf = launch_bundles<float, 1, 4>; gf = launch_growth<float, 1, 4, 4>; break;
        case 3: bf = launch_bundles<float, 3, 4>; gf = launch_growth<float, 3, 4, 4>; break;
        case 4: bf = launch_bundles<float, 4, 4>; gf = launch_growth<float, 4, 4, 4>; break;
        default: bf = launch_bundles<float, 2, 4>; gf = launch_growth<float, 2, 4, 4>; break;
    }
}

// The kernel variants a tuning selects (seeds_per_group 8 only for grids of up to
// 64 cells, where its register footprint fits).
void pick_kernels(int cpl, const cvl_tuning &t, bundles_fn<double> &bf, growth_fn<double> &gf) {
    const bool b3 = t.bundle_blocks_per_sm == 3;
    const bool g6 = t.growth_blocks_per_sm == 6;
    const bool g8 = t.growth_blocks_per_sm == 8;  // 64 registers: 32 one-warp blocks per SM
    const bool k8 = t.seeds_per_group == 8 && cpl <= 2;
    switch (cpl) {
        case 1:
            bf = b3 ? launch_bundles<double, 1, 3> : launch_bundles<double, 1, 4>;
            gf = k8 ? launch_growth<double, 1, 8, 4> : (g6 ? launch_growth<double, 1, 4, 6> : launch_growth<double, 1, 4, 4>);
            break;
        case 3:
            bf = b3 ? launch_bundles<double, 3, 3> : launch_bundles<double, 3, 4>;
            gf = g6 ? launch_growth<double, 3, 4, 6> : launch_growth<double, 3, 4, 4>;
            break;
        case 4:
            bf = b3 ? launch_bundles<double, 4, 3> : launch_bundles<double, 4, 4>;
            gf = g6 ? launch_growth<double, 4, 4, 6> : launch_growth<double, 4, 4, 4>;
            break;
        default:
            bf = b3 ? launch_bundles<double, 2, 3> : launch_bundles<double, 2, 4>;
            gf = k8 ? launch_growth<double, 2, 8, 4>
                    : (g8 ? launch_growth<double, 2, 4, 8>
                          : (g6 ? launch_growth<double, 2, 4, 6> : launch_growth<double, 2, 4, 4>));
            break;
    }
}

// Whether a direct run of n edges on this engine runs its chunks on persistent grids.
inline bool persistent_chunks(const cvl_engine *e, long long n) {
    return e->persist_on && !e->yield_fn && n > (64 << 10);
}
// growth warps of a persistent grid at most (SMs x 4 x the largest register budget), for
// the record arena's chunk tails in the workspace formula
constexpr unsigned long long PERSIST_GROWTH_WARPS_MAX = 160ull * 4 * 8;

// mode: 0 = full run, 1 = count valid pairs only, 2 = neighbour graph only
template <typename R>
int run_pipeline_direct(cvl_engine *e, const R *d_edges, int n, int sz, const int *d_map_off,
                 const std::vector<int32_t> &map_off_host, ModelT<R> md, int cpl, int mode, bool want_d2,
                 RunOut &ro) {
    const int M = (int)map_off_host.size() - 1;
    cudaStream_t s = e->stream;
    // one NVTX range per run on the host timeline, a mark at each stage's end
    struct NvtxRun {
        NvtxRun() { nvtxRangePushA("cvl path"); }
        ~NvtxRun() { nvtxRangePop(); }
    } nvtx_run;
    e->nmarks = 0;
    ++e->generation;
    g_launches = 0;
    e->mark("start");

    const cvl_tuning &tn = e->tune[bucket_of(n)];
    md.sbits = tn.cell_size == 2 ? 1 : (tn.cell_size == 8 ? 3 : 2);
    const unsigned T = next_pow2(std::max<unsigned long long>((unsigned long long)n, 1024ull));
    md.hash_mask = T - 1;

    // ---- workspace for N-sized arrays
    CVL_TRY(e->alloc(e->ehash, sizeof(unsigned) * n));
    CVL_TRY(e->alloc(e->bcount, sizeof(unsigned) * (T + 1)));
    CVL_TRY(e->alloc(e->bstart, sizeof(unsigned) * (T + 1)));
    CVL_TRY(e->alloc(e->bfill, sizeof(unsigned) * (T + 1)));
    CVL_TRY(e->alloc(e->pos_of, sizeof(int) * n));
    CVL_TRY(e->alloc(e->bx, sizeof(R) * n));
    CVL_TRY(e->alloc(e->by, sizeof(R) * n));
    CVL_TRY(e->alloc(e->bth, sizeof(R) * n));
    CVL_TRY(e->alloc(e->bsp, sizeof(R) * n));
    CVL_TRY(e->alloc(e->bcp, sizeof(R) * n));
    CVL_TRY(e->alloc(e->bsm, sizeof(R) * n));
    CVL_TRY(e->alloc(e->bcm, sizeof(R) * n));
    CVL_TRY(e->alloc(e->bcell, sizeof(int2) * n));
    CVL_TRY(e->alloc(e->orig_of, sizeof(int) * n));
    CVL_TRY(e->alloc(e->bmap, sizeof(int) * n));
    CVL_TRY(e->alloc(e->ncand, sizeof(unsigned) * n));
    CVL_TRY(e->alloc(e->deg, sizeof(unsigned) * n));
    CVL_TRY(e->alloc(e->pair_off, sizeof(unsigned long long) * (n + 1)));
    CVL_TRY(e->alloc(e->count, sizeof(unsigned) * n));
    CVL_TRY(e->alloc(e->run_cnt, sizeof(unsigned) * 2 * (size_t)n));
    CVL_TRY(e->alloc(e->rec_base, sizeof(unsigned) * 2 * (size_t)n));
    CVL_TRY(e->alloc(e->out_off, sizeof(unsigned long long) * (n + 1)));
    CVL_TRY(e->alloc(e->stats, sizeof(MapStats) * M));
    CVL_TRY(e->alloc(e->err, sizeof(unsigned) * 4));
    CVL_TRY(e->alloc(e->work, sizeof(unsigned long long) * 4));  // arena counter, -, work queues

    BinnedT<R> B;
    B.x = (R *)e->bx.p;
    B.y = (R *)e->by.p;
    B.th = (R *)e->bth.p;
    B.sp = (R *)e->bsp.p;
    B.cp = (R *)e->bcp.p;
    B.sm = (R *)e->bsm.p;
    B.cm = (R *)e->bcm.p;
    B.cell = (int2 *)e->bcell.p;
    B.orig = (int *)e->orig_of.p;
    B.map = (int *)e->bmap.p;
    unsigned *err = (unsigned *)e->err.p;
    MapStats *stats = (MapStats *)e->stats.p;
    unsigned long long *arena_ctr = (unsigned long long *)e->work.p;

    CVL_CUDA(cudaMemsetAsync(e->bcount.p, 0, sizeof(unsigned) * (T + 1), s));
    CVL_CUDA(cudaMemsetAsync(e->bfill.p, 0, sizeof(unsigned) * (T + 1), s));
    CVL_CUDA(cudaMemsetAsync(e->stats.p, 0, sizeof(MapStats) * M, s));
    CVL_CUDA(cudaMemsetAsync(e->err.p, 0, sizeof(unsigned) * 4, s));
    CVL_CUDA(cudaMemsetAsync(e->work.p, 0, sizeof(unsigned long long) * 4, s));

    // ---- (a) binning
    const int gb = short_grid(n, 256);
    unsigned *uncertified = (unsigned *)((unsigned long long *)e->work.p + 2);  // zeroed with the counters
    k_bin_keys<<<gb, 256, 0, s>>>(d_edges, sz, n, d_map_off, M, md, (unsigned *)e->ehash.p, (unsigned *)e->bcount.p,
                                  err, uncertified, nullptr);
    CVL_TRY(check_launch("k_bin_keys"));
    CVL_TRY((scan<unsigned, unsigned>(e, (const unsigned *)e->bcount.p, T, (unsigned *)e->bstart.p)));
    k_bin_scatter<<<gb, 256, 0, s>>>(d_edges, sz, n, d_map_off, M, md, (const unsigned *)e->ehash.p,
                                     (const unsigned *)e->bstart.p, (unsigned *)e->bfill.p, B, (int *)e->pos_of.p,
                                     nullptr);
    CVL_TRY(check_launch("k_bin_scatter"));
    e->mark("bin");

    // ---- (b) neighbour count, CSR offsets, chunk boundaries
    const int nb_wpb = 8;
    const size_t nb_smem = (size_t)nb_wpb * nbr_smem_per_warp(md.max_cand);
    CVL_CUDA(cudaFuncSetAttribute(k_nb<R, NB_COUNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nb_smem));
    CVL_CUDA(cudaFuncSetAttribute(k_nb<R, NB_FILL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nb_smem));
    const int gn = short_grid(n, (long long)nb_wpb * 4);  // a warp per anchor, 4 anchors per warp
    NbArgsT<R> na{};
    na.md = md;
    na.B = B;
    na.bstart = (const unsigned *)e->bstart.p;
    na.N = n;
    na.M = M;
    na.ncand = (unsigned *)e->ncand.p;
    na.stats = stats;
    na.pair_off = (const unsigned long long *)e->pair_off.p;
    na.err = err;
    k_nb<R, NB_COUNT><<<gn, nb_wpb * 32, 0, s>>>(na);  // no candidate staging
    CVL_TRY(check_launch("k_nb<COUNT>"));
    k_deg_from_ncand<<<gb, 256, 0, s>>>(n, md.max_cand, (const unsigned *)e->ncand.p, (unsigned *)e->deg.p, nullptr);
    CVL_TRY(check_launch("k_deg_from_ncand"));
    CVL_TRY((scan<unsigned, unsigned long long>(e, (const unsigned *)e->deg.p, n,
                                                (unsigned long long *)e->pair_off.p)));
    // chunk boundaries over anchors: a chunk holds at most CHUNK_PAIRS + max_deg pairs
    const unsigned long long per_chunk = std::max<unsigned long long>((unsigned long long)tn.chunk_pairs, 1024ull);
    const int max_chunks = 4096;
    CVL_TRY(e->alloc(e->chunk_start, sizeof(int) * (max_chunks + 1)));
    CVL_CUDA(cudaMemsetAsync(e->chunk_start.p, 0, sizeof(int) * (max_chunks + 1), s));
    k_chunk_starts<<<gb, 256, 0, s>>>(n, (const unsigned long long *)e->pair_off.p + 1, per_chunk, max_chunks,
                                     (int *)e->chunk_start.p, nullptr);
    CVL_TRY(check_launch("k_chunk_starts"));
    e->mark("neighbors_count");

    // sync 1: pair total, max degree, chunk boundaries
    ro.stats.assign(M, MapStats{});
    unsigned h_err = 0;
    std::vector<int> cstart(max_chunks + 1, 0);
    CVL_CUDA(cudaMemcpyAsync(&ro.total_pairs, (unsigned long long *)e->pair_off.p + n, sizeof(unsigned long long),
                             cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(ro.stats.data(), stats, sizeof(MapStats) * M, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(cstart.data(), e->chunk_start.p, sizeof(int) * (max_chunks + 1), cudaMemcpyDeviceToHost,
                             s));
    CVL_CUDA(cudaStreamSynchronize(s));
    if (h_err & ERR_NONFINITE) return fail(CVL_EINVAL, "non-finite or out-of-range (|v| >= 1e9) edge coordinate");
    ro.max_deg = 0;
    for (const MapStats &st : ro.stats) ro.max_deg = std::max(ro.max_deg, st.max_deg);
    const unsigned long long P = ro.total_pairs;
    int nchunks = (int)std::min<unsigned long long>((P + per_chunk - 1) / per_chunk, (unsigned long long)max_chunks);
    if (nchunks < 1) nchunks = 1;
    if ((P + per_chunk - 1) / per_chunk > (unsigned long long)max_chunks)
        return fail(CVL_EUNSUPPORTED, "input needs more than 4096 pair chunks");
    cstart[nchunks] = n;

    // ---- (b) neighbour fill: CSR, pair classes, pair -> anchor, anchor trig
    CVL_TRY(e->alloc(e->csr_ids, sizeof(int) * P));
    if (want_d2) CVL_TRY(e->alloc(e->csr_d2, sizeof(R) * P));
    const bool path = (mode != 2);
    if (path) {
        CVL_TRY(e->alloc(e->pcls, P));
        CVL_TRY(e->alloc(e->pflag, P));
        CVL_TRY(e->alloc(e->pair_anchor, sizeof(int) * P));
        CVL_TRY(e->alloc(e->atrig, sizeof(R) * (size_t)n * (2 * md.Q + 2)));
    }
    na.csr_ids = (int *)e->csr_ids.p;
    na.csr_d2 = want_d2 ? (R *)e->csr_d2.p : nullptr;
    na.pcls = path ? (unsigned char *)e->pcls.p : nullptr;
    na.pair_anchor = path ? (int *)e->pair_anchor.p : nullptr;
    na.atrig = path ? (R *)e->atrig.p : nullptr;
    na.uncertified = uncertified;
    k_nb<R, NB_FILL><<<gn, nb_wpb * 32, nb_smem, s>>>(na);
    CVL_TRY(check_launch("k_nb<FILL>"));
    e->mark("neighbors_fill");
    if (mode == 2) {
        e->mark("end");
        return CVL_OK;
    }

    // ---- (c) + (d) per chunk
    bundles_fn<R> bf;
    growth_fn<R> gf;
    pick_kernels(cpl, tn, bf, gf);
    const size_t gsmem = (size_t)(GROWTH_THREADS / 32) * growth_smem_per_warp(md.max_cand, md.gms);
    const unsigned long long max_chunk_pairs = per_chunk + (unsigned long long)ro.max_deg + 1;
    const unsigned long long chunk_cap = std::min<unsigned long long>(P + 1, max_chunk_pairs);
    CVL_TRY(e->alloc(e->bund, sizeof(R) * 64 * (size_t)cpl * chunk_cap));
    const int bblocks = e->prop.multiProcessorCount * 8;
    const int gblocks = e->prop.multiProcessorCount * 8;

    // Without a yield hook (no higher-priority work to make room for), the chunks run on
    // persistent grids that pull their work from device queues (measured on the 64-map
    // batch: 509.2 -> 492.1 ms; bundles -3.7%, growth -4.7%). A launch that yields keeps
    // short blocks, so that a higher-priority stream takes SMs as soon as any block ends.
    // Runs above 64 Ki edges (smaller ones replay a graph).
    const int persist_warps = e->prop.multiProcessorCount * 4 * tn.growth_blocks_per_sm;
    const bool persist = persistent_chunks(e, n) && std::is_same<R, double>::value &&
                         (unsigned long long)persist_warps <= PERSIST_GROWTH_WARPS_MAX;
    for (int attempt = 0;; ++attempt) {
        // the growth warps reserve the arena in chunks of at most GROWTH_ARENA_CHUNK
        // records, no more than their anchors (anchors_per_warp): the chunk tails they
        // leave unused are at most one record per anchor plus one chunk per launch; a
        // persistent grid's warp, whatever its anchors, leaves at most one chunk per launch
        unsigned long long cap = std::max<unsigned long long>(e->arena_hint, 4ull * (unsigned long long)n + 4096ull) +
                                 (unsigned long long)n + (unsigned long long)GROWTH_ARENA_CHUNK * (nchunks + 1) +
                                 (persist ? (unsigned long long)GROWTH_ARENA_CHUNK * persist_warps * nchunks : 0ull);
        if (mode == 0) {
            CVL_TRY(e->alloc(e->rec_ids, sizeof(unsigned) * cap * md.gms));
            CVL_TRY(e->alloc(e->rec_k, sizeof(double) * cap * 2));
            CVL_TRY(e->alloc(e->rec_meta, sizeof(unsigned) * cap));
        } else {
            cap = 0;
        }
        CVL_TRY(e->alloc(e->crank, sizeof(unsigned short) * CELLS_MAX));
        k_cell_ranks<R><<<1, 128, 0, s>>>(md, (unsigned short *)e->crank.p);
        CVL_TRY(check_launch("k_cell_ranks"));
        Records rec;
        rec.ids = (unsigned *)e->rec_ids.p;
        rec.k = (double *)e->rec_k.p;
        rec.meta = (unsigned *)e->rec_meta.p;
        std::vector<unsigned long long> h_poff(nchunks + 1);
        for (int c = 0; c <= nchunks; ++c)
            CVL_CUDA(cudaMemcpyAsync(&h_poff[c], (unsigned long long *)e->pair_off.p + cstart[c],
                                     sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        unsigned h_uncertified = 0;
        CVL_CUDA(cudaMemcpyAsync(&h_uncertified, uncertified, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        CVL_CUDA(cudaStreamSynchronize(s));
        const int shared_quot = (md.shared_quot && !h_uncertified) ? 1 : 0;
        unsigned *queues = (unsigned *)((unsigned long long *)e->work.p + 3);
        for (int c = 0; c < nchunks; ++c) {
            const int a0 = cstart[c], a1 = cstart[c + 1];
            if (a1 <= a0) continue;
            if (e->yield_fn && c > 0) {
                // let the previous chunk finish, then give the hook the chance to hold
                // this stream back while others' work goes first
                if (!e->chunk_done) CVL_CUDA(cudaEventCreateWithFlags(&e->chunk_done, cudaEventDisableTiming));
                CVL_CUDA(cudaEventRecord(e->chunk_done, s));
                CVL_CUDA(cudaEventSynchronize(e->chunk_done));
                e->yield_fn(e->yield_ctx);
            }
            BundleArgsT<R> ba{};
            ba.md = md;
            ba.B = B;
            ba.p_begin = h_poff[c];
            ba.p_end = h_poff[c + 1];
            ba.csr_ids = (const int *)e->csr_ids.p;
            ba.pair_anchor = (const int *)e->pair_anchor.p;
            ba.pcls = (const unsigned char *)e->pcls.p;
            ba.atrig = (const R *)e->atrig.p;
            ba.bund = (R *)e->bund.p;
            ba.pflag = (unsigned char *)e->pflag.p;
            ba.shared_quot = shared_quot;  // the host read the run's certification above
            if (persist) {
                CVL_CUDA(cudaMemsetAsync(queues, 0, 2 * sizeof(unsigned), s));
                ba.queue = queues;
            }
            if (ba.p_end > ba.p_begin) {
                CVL_TRY(bf(e, ba, persist ? e->prop.multiProcessorCount * 16 : bblocks));
            }
            e->mark("bundles");
            GrowthArgsT<R> ga{};
            ga.md = md;
            ga.B = B;
            ga.M = M;
            ga.a_begin = a0;
            ga.a_end = a1;
            ga.p_begin = h_poff[c];
            ga.pair_off = (const unsigned long long *)e->pair_off.p;
            ga.csr_ids = (const int *)e->csr_ids.p;
            ga.pcls = (const unsigned char *)e->pcls.p;
            ga.pflag = (const unsigned char *)e->pflag.p;
            ga.bund = (const R *)e->bund.p;
            ga.rec = rec;
            ga.arena_cap = cap;
            ga.arena_ctr = arena_ctr;
            ga.rec_base = (unsigned *)e->rec_base.p;
            ga.run_cnt = (unsigned *)e->run_cnt.p;
            ga.count = (unsigned *)e->count.p;
            ga.stats = stats;
            ga.count_only = (mode == 1) ? 1 : 0;
            ga.err = err;
            ga.cell_rank = (const unsigned short *)e->crank.p;
            ga.anchors_per_warp = tn.anchors_per_warp;
            if (persist) ga.queue = queues + 1;
            CVL_TRY(gf(e, ga, gsmem, persist ? persist_warps : gblocks));
            e->mark("growth");
        }

        if (mode == 1) {
            CVL_CUDA(cudaMemcpyAsync(ro.stats.data(), stats, sizeof(MapStats) * M, cudaMemcpyDeviceToHost, s));
            CVL_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
            e->mark("end");
            CVL_CUDA(cudaStreamSynchronize(s));
            if (h_err) return fail(CVL_EOVERFLOW, "kernel reported error bits " + std::to_string(h_err));
            return CVL_OK;
        }

        // ---- output positions (anchor-major, compact_curvelet_output)
        CVL_TRY((scan<unsigned, unsigned long long>(e, (const unsigned *)e->count.p, n,
                                                    (unsigned long long *)e->out_off.p)));
        std::vector<unsigned long long> tmp(M + 1);
        for (int m = 0; m <= M; ++m)
            CVL_CUDA(cudaMemcpyAsync(&tmp[m], (unsigned long long *)e->out_off.p + map_off_host[m],
                                     sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        unsigned long long used = 0;
        CVL_CUDA(cudaMemcpyAsync(ro.stats.data(), stats, sizeof(MapStats) * M, cudaMemcpyDeviceToHost, s));
        CVL_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        CVL_CUDA(cudaMemcpyAsync(&used, arena_ctr, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
        CVL_CUDA(cudaStreamSynchronize(s));
        if ((h_err & ERR_ARENA) && attempt == 0) {
            // the record arena was too small: size it to what this input needs and run the
            // bundle/growth stages again (valid_pairs is recounted from zero)
            e->arena_hint = used + used / 8 + 4096;
            for (MapStats &st : ro.stats) st.valid_pairs = 0;
            CVL_CUDA(cudaMemcpyAsync(stats, ro.stats.data(), sizeof(MapStats) * M, cudaMemcpyHostToDevice, s));
            CVL_CUDA(cudaMemsetAsync(e->err.p, 0, sizeof(unsigned) * 4, s));
            CVL_CUDA(cudaMemsetAsync(e->work.p, 0, sizeof(unsigned long long) * 2, s));
            continue;
        }
        if (h_err) return fail(CVL_EOVERFLOW, "kernel reported error bits " + std::to_string(h_err));
        ro.cv_off = tmp;
        const unsigned long long C = ro.cv_off[M];
        ro.total_curvelets = C;
        const int W = md.gms + 1;
        CVL_TRY(e->alloc(e->chains, sizeof(unsigned) * C * W));
        CVL_TRY(e->alloc(e->info, sizeof(double) * C * 10));
        k_finalize<R><<<gb, 256, 0, s>>>(md, d_edges, sz, n, d_map_off, M, rec, (const unsigned *)e->rec_base.p,
                                      (const unsigned *)e->run_cnt.p, (const unsigned long long *)e->out_off.p, C,
                                      (unsigned *)e->chains.p, (double *)e->info.p, nullptr);
        CVL_TRY(check_launch("k_finalize"));
        e->mark("finalize");
        return CVL_OK;
    }
}

// ---- the workspace of a launch, by shape ----------------------------------------
// The device buffers run_pipeline (mode 0, FP64) takes for a launch of shape s, with
// the sizes it asks for once the counts are known: the same buffers and the same
// requests, with each count at the shape's value (a chunk of bundles at its largest).
// A buffer that already holds a request's size is reused as it is, so a workspace
// allocated from this plan serves every launch within the shape with no allocation.
struct WsItem {
    DBuf cvl_engine::*buf;
    size_t bytes;
    bool per_launch;  // the bundle chunk: one per launch, whatever the maps
};

// tune: the engine's tuning per bucket (it sets the bundle chunk); arena_hint: the
// record arena a past input needed (0 for a footprint alone)
std::vector<WsItem> workspace_plan(const cvl_tuning *tune, unsigned long long arena_hint, const Model &md, int cpl,
                                   const cvl_workspace_shape &s) {
    const unsigned long long n = (unsigned long long)std::max<int64_t>(s.num_edges, 1);
    const unsigned long long P = (unsigned long long)std::max<int64_t>(s.num_pairs, 0);
    const unsigned long long C = (unsigned long long)std::max<int64_t>(s.num_curvelets, 0);
    const unsigned long long M = (unsigned long long)std::max<int32_t>(s.num_maps, 1);
    const cvl_tuning &tn = tune[bucket_of((long long)n)];
    const unsigned long long T = next_pow2(std::max<unsigned long long>(n, 1024ull));
    const size_t R = sizeof(double);
    std::vector<WsItem> v;
    auto add = [&](DBuf cvl_engine::*b, unsigned long long bytes, bool per_launch = false) {
        v.push_back({b, (size_t)std::max<unsigned long long>(bytes, 16ull), per_launch});
    };
    using E = cvl_engine;
    // the input rows and map offsets (cvl_run's upload; a batch holds its own instead)
    add(&E::edges, sizeof(double) * n * (unsigned long long)std::max<int32_t>(s.edge_data_sz, 4));
    add(&E::map_off, 4 * (M + 1));
    // N-sized (run_pipeline's first block)
    add(&E::ehash, 4 * n);
    add(&E::bcount, 4 * (T + 1));
    add(&E::bstart, 4 * (T + 1));
    add(&E::bfill, 4 * (T + 1));
    add(&E::pos_of, 4 * n);
    for (DBuf E::*b : {&E::bx, &E::by, &E::bth, &E::bsp, &E::bcp, &E::bsm, &E::bcm}) add(b, R * n);
    add(&E::bcell, 8 * n);
    add(&E::orig_of, 4 * n);
    add(&E::bmap, 4 * n);
    add(&E::ncand, 4 * n);
    add(&E::deg, 4 * n);
    add(&E::pair_off, 8 * (n + 1));
    add(&E::count, 4 * n);
    add(&E::run_cnt, 8 * n);
    add(&E::rec_base, 8 * n);
    add(&E::out_off, 8 * (n + 1));
    add(&E::stats, sizeof(MapStats) * M);
    add(&E::err, 16);
    add(&E::work, 32);
    add(&E::scan_tmp, (T / SCAN_TILE + 64) * 4 * sizeof(unsigned long long) + 4096);  // the largest scan: T
    add(&E::chunk_start, 4 * (4096 + 1));
    // pair-sized (after the count)
    add(&E::csr_ids, 4 * P);
    add(&E::pcls, P);
    add(&E::pflag, P);
    add(&E::pair_anchor, 4 * P);
    add(&E::atrig, R * n * (unsigned long long)(2 * md.Q + 2));
    // one chunk of bundles (max_deg <= max_candidates)
    const unsigned long long per_chunk = std::max<unsigned long long>((unsigned long long)tn.chunk_pairs, 1024ull);
    const unsigned long long chunk_cap =
        std::min<unsigned long long>(P + 1, per_chunk + (unsigned long long)md.max_cand + 1);
    add(&E::bund, R * 64 * (unsigned long long)cpl * chunk_cap, true);
    // the record arena (run_pipeline's cap, with room for C records)
    const unsigned long long nchunks = std::max<unsigned long long>((P + per_chunk - 1) / per_chunk, 1ull);
    const unsigned long long cap =
        std::max<unsigned long long>(std::max<unsigned long long>(arena_hint, C), 4ull * n + 4096ull) + n +
        (unsigned long long)GROWTH_ARENA_CHUNK * (nchunks + 1) +
        (n > (64 << 10) ? (unsigned long long)GROWTH_ARENA_CHUNK * PERSIST_GROWTH_WARPS_MAX * nchunks : 0ull);
    add(&E::rec_ids, 4 * cap * (unsigned long long)md.gms);
    add(&E::rec_k, 16 * cap);
    add(&E::rec_meta, 4 * cap);
    add(&E::crank, 2 * CELLS_MAX);
    // outputs
    add(&E::chains, 4 * C * (unsigned long long)(md.gms + 1));
    add(&E::info, 80 * C);
    return v;
}

inline size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

// ---- the path as a CUDA graph, one per size bucket ---------------------------------
// Runs of up to 64 Ki edges (bucket 0) and 512 Ki edges (bucket 1) replay a graph
// captured for the bucket's capacities: every kernel is launched for the bucket's
// edges, maps and bundle chunks and reads the run's own sizes (RunDims) and chunk
// ranges (ChunkDims, computed on the device) from device memory, so that one graph
// serves every run of the bucket, with one host synchronisation at its end instead
// of the direct path's three. A run that exceeds a capacity (more pairs than the
// bucket's chunks hold, more curvelets than its outputs, a record-arena overflow)
// is flagged on the device and run again by the direct path, with the same results.
struct GraphCaps {
    int N;  // edges
    int M;  // maps
    int K;  // bundle chunks
    int curvelets_per_edge;
};
constexpr GraphCaps GRAPH_CAPS[2] = {{64 << 10, 4096, 2, 8}, {512 << 10, 4096, 8, 8}};
constexpr size_t GRAPH_SLOTS = 6;  // captured graphs kept per engine (least recently used goes)

size_t graph_readback_bytes() {
    // totals + per-map curvelet offsets, per-map statistics, error bits
    return (size_t)(2 + GRAPH_CAPS[1].M + 1) * 8 + sizeof(MapStats) * (size_t)GRAPH_CAPS[1].M + 16;
}

// CVL_OK with ro filled; CVL_EAGAIN when the run is not for a graph or did not fit
// (the caller runs the direct path); another status on a real error.
int run_pipeline_graph(cvl_engine *e, const double *d_edges, int n, int sz, const int *d_map_off,
                       const std::vector<int32_t> &map_off_host, Model md, int cpl, RunOut &ro) {
    const int M = (int)map_off_host.size() - 1;
    const int b = bucket_of(n);
    if (!e->graphs_on || g_sync_check || b > 1) return CVL_EAGAIN;
    const GraphCaps cap = GRAPH_CAPS[b];
    if (n > cap.N || M > cap.M) return CVL_EAGAIN;
    cudaStream_t s = e->stream;
    const cvl_tuning &tn = e->tune[b];
    md.sbits = tn.cell_size == 2 ? 1 : (tn.cell_size == 8 ? 3 : 2);
    const unsigned T = next_pow2(std::max<unsigned long long>((unsigned long long)cap.N, 1024ull));
    md.hash_mask = T - 1;
    const unsigned long long per_chunk = std::max<unsigned long long>((unsigned long long)tn.chunk_pairs, 1024ull);

    // the workspace at the bucket's capacities (no-ops once it is there)
    cvl_workspace_shape sh;
    sh.num_edges = cap.N;
    sh.num_pairs = (int64_t)(per_chunk * (unsigned long long)cap.K);
    sh.num_curvelets = (int64_t)cap.N * cap.curvelets_per_edge;
    sh.num_maps = cap.M;
    sh.edge_data_sz = sz;
    // (the input rows and map offsets are the caller's, already in place: they are
    // not reallocated here)
    for (const WsItem &w : workspace_plan(e->tune, e->arena_hint, md, cpl, sh)) {
        if (w.buf == &cvl_engine::edges || w.buf == &cvl_engine::map_off) continue;
        CVL_TRY(e->alloc(e->*(w.buf), w.bytes));
    }
    CVL_TRY(e->alloc(e->gdims, sizeof(RunDims)));
    CVL_TRY(e->alloc(e->gchunks, sizeof(ChunkDims) * (size_t)cap.K));
    CVL_TRY(e->alloc(e->gread, (size_t)(2 + cap.M + 1) * 8));
    if (!e->gread_host) {
        void *h = nullptr;
        if (cvl_alloc_fault_injected() || cudaMallocHost(&h, graph_readback_bytes() + sizeof(RunDims) + 64) != cudaSuccess) {
            cudaGetLastError();
            return fail(CVL_ENOMEM, "page-locked graph readback could not be allocated");
        }
        e->gread_host = (unsigned char *)h;
    }
    const unsigned long long C_cap = (unsigned long long)sh.num_curvelets;
    const unsigned long long nchunks_cap = (unsigned long long)cap.K;
    const unsigned long long arena_cap =
        std::max<unsigned long long>(std::max<unsigned long long>(e->arena_hint, C_cap), 4ull * cap.N + 4096ull) +
        (unsigned long long)cap.N + (unsigned long long)GROWTH_ARENA_CHUNK * (nchunks_cap + 1);
    unsigned long long *rb_h = (unsigned long long *)e->gread_host;
    MapStats *stats_h = (MapStats *)(e->gread_host + (size_t)(2 + cap.M + 1) * 8);
    unsigned *err_h = (unsigned *)((unsigned char *)stats_h + sizeof(MapStats) * (size_t)cap.M);
    RunDims *dims_h = (RunDims *)(e->gread_host + graph_readback_bytes() + 32);

    // what the graph is captured for
    std::string key((const char *)&md, sizeof(md));
    const void *ptrs[] = {d_edges, d_map_off, e->chains.p, e->info.p};
    key.append((const char *)ptrs, sizeof(ptrs));
    const unsigned long long nums[] = {(unsigned long long)b, (unsigned long long)sz, (unsigned long long)cpl,
                                       e->ws_epoch, arena_cap, per_chunk};
    key.append((const char *)nums, sizeof(nums));
    key.append((const char *)&tn, sizeof(tn));
    cvl_engine::GraphSlot *slot = nullptr;
    for (auto &g : e->graphs)
        if (g.key == key) slot = &g;

    e->nmarks = 0;
    ++e->generation;
    g_launches = 0;
    if (!slot) {
        bundles_fn<double> bf;
        growth_fn<double> gf;
        pick_kernels(cpl, tn, bf, gf);
        const int nb_wpb = 8;
        const size_t nb_smem = (size_t)nb_wpb * nbr_smem_per_warp(md.max_cand);
        CVL_CUDA(cudaFuncSetAttribute(k_nb<double, NB_COUNT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nb_smem));
        CVL_CUDA(cudaFuncSetAttribute(k_nb<double, NB_FILL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)nb_smem));
        const size_t gsmem = (size_t)(GROWTH_THREADS / 32) * growth_smem_per_warp(md.max_cand, md.gms);
        BinnedT<double> B;
        B.x = (double *)e->bx.p;
        B.y = (double *)e->by.p;
        B.th = (double *)e->bth.p;
        B.sp = (double *)e->bsp.p;
        B.cp = (double *)e->bcp.p;
        B.sm = (double *)e->bsm.p;
        B.cm = (double *)e->bcm.p;
        B.cell = (int2 *)e->bcell.p;
        B.orig = (int *)e->orig_of.p;
        B.map = (int *)e->bmap.p;
        unsigned *err = (unsigned *)e->err.p;
        MapStats *stats = (MapStats *)e->stats.p;
        unsigned long long *arena_ctr = (unsigned long long *)e->work.p;
        const RunDims *dd = (const RunDims *)e->gdims.p;
        ChunkDims *cdp = (ChunkDims *)e->gchunks.p;
        const int sms = e->prop.multiProcessorCount;
        const int N = cap.N;
        CVL_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
        auto enqueue = [&]() -> int {
            CVL_CUDA(cudaMemsetAsync(e->bcount.p, 0, sizeof(unsigned) * (T + 1), s));
            CVL_CUDA(cudaMemsetAsync(e->bfill.p, 0, sizeof(unsigned) * (T + 1), s));
            CVL_CUDA(cudaMemsetAsync(e->stats.p, 0, sizeof(MapStats) * cap.M, s));
            CVL_CUDA(cudaMemsetAsync(e->err.p, 0, 16, s));
            CVL_CUDA(cudaMemsetAsync(e->work.p, 0, 32, s));
            CVL_CUDA(cudaMemsetAsync(e->count.p, 0, sizeof(unsigned) * N, s));
            CVL_CUDA(cudaMemsetAsync(e->chunk_start.p, 0, sizeof(int) * (cap.K + 1), s));
            const int gb = short_grid(N, 256);
            unsigned *uncertified = (unsigned *)((unsigned long long *)e->work.p + 2);  // zeroed above
            k_bin_keys<<<gb, 256, 0, s>>>(d_edges, sz, N, d_map_off, cap.M, md, (unsigned *)e->ehash.p,
                                          (unsigned *)e->bcount.p, err, uncertified, dd);
            CVL_TRY(check_launch("k_bin_keys"));
            CVL_TRY((scan<unsigned, unsigned>(e, (const unsigned *)e->bcount.p, T, (unsigned *)e->bstart.p)));
            k_bin_scatter<<<gb, 256, 0, s>>>(d_edges, sz, N, d_map_off, cap.M, md, (const unsigned *)e->ehash.p,
                                             (const unsigned *)e->bstart.p, (unsigned *)e->bfill.p, B,
                                             (int *)e->pos_of.p, dd);
            CVL_TRY(check_launch("k_bin_scatter"));
            NbArgsT<double> na{};
            na.md = md;
            na.B = B;
            na.bstart = (const unsigned *)e->bstart.p;
            na.N = N;
            na.M = cap.M;
            na.ncand = (unsigned *)e->ncand.p;
            na.stats = stats;
            na.pair_off = (const unsigned long long *)e->pair_off.p;
            na.err = err;
            na.dims = dd;
            na.pair_cap = (unsigned long long)sh.num_pairs;
            const int gn = std::min(short_grid(N, (long long)nb_wpb * 4), sms * 8);
            k_nb<double, NB_COUNT><<<gn, nb_wpb * 32, 0, s>>>(na);  // no candidate staging
            CVL_TRY(check_launch("k_nb<COUNT>"));
            k_deg_from_ncand<<<gb, 256, 0, s>>>(N, md.max_cand, (const unsigned *)e->ncand.p, (unsigned *)e->deg.p, dd);
            CVL_TRY(check_launch("k_deg_from_ncand"));
            CVL_TRY((scan<unsigned, unsigned long long>(e, (const unsigned *)e->deg.p, N,
                                                        (unsigned long long *)e->pair_off.p)));
            k_chunk_starts<<<gb, 256, 0, s>>>(N, (const unsigned long long *)e->pair_off.p + 1, per_chunk, cap.K,
                                             (int *)e->chunk_start.p, dd);
            CVL_TRY(check_launch("k_chunk_starts"));
            k_chunk_dims<<<1, 32, 0, s>>>(dd, (const unsigned long long *)e->pair_off.p, (const int *)e->chunk_start.p,
                                          per_chunk, cap.K, cdp, err);
            CVL_TRY(check_launch("k_chunk_dims"));
            na.csr_ids = (int *)e->csr_ids.p;
            na.csr_d2 = nullptr;
            na.pcls = (unsigned char *)e->pcls.p;
            na.pair_anchor = (int *)e->pair_anchor.p;
            na.atrig = (double *)e->atrig.p;
            na.uncertified = uncertified;
            k_nb<double, NB_FILL><<<gn, nb_wpb * 32, nb_smem, s>>>(na);
            CVL_TRY(check_launch("k_nb<FILL>"));
            k_cell_ranks<double><<<1, 128, 0, s>>>(md, (unsigned short *)e->crank.p);
            CVL_TRY(check_launch("k_cell_ranks"));
            Records rec;
            rec.ids = (unsigned *)e->rec_ids.p;
            rec.k = (double *)e->rec_k.p;
            rec.meta = (unsigned *)e->rec_meta.p;
            // the chunks' work queues (bundle pair tiles, growth anchors)
            unsigned *queues = (unsigned *)((unsigned long long *)e->work.p + 3);
            for (int c = 0; c < cap.K; ++c) {
                CVL_CUDA(cudaMemsetAsync(queues, 0, 2 * sizeof(unsigned), s));
                BundleArgsT<double> ba{};
                ba.md = md;
                ba.B = B;
                ba.csr_ids = (const int *)e->csr_ids.p;
                ba.pair_anchor = (const int *)e->pair_anchor.p;
                ba.pcls = (const unsigned char *)e->pcls.p;
                ba.atrig = (const double *)e->atrig.p;
                ba.bund = (double *)e->bund.p;
                ba.pflag = (unsigned char *)e->pflag.p;
                ba.cd = cdp + c;
                // bucket 1 pulls work from the queues (measured: the 242k-edge map 2.79 ->
                // 2.52 ms); bucket 0's runs are too small for the atomics to pay
                ba.queue = b == 1 ? queues : nullptr;
                if (md.shared_quot) {
                    // the run's certification is known only on the device: both forms go
                    // into the graph, and the one that does not match returns at once
                    ba.uncertified = uncertified;
                    ba.shared_quot = 1;
                    CVL_TRY(bf(e, ba, sms * 16));
                    ba.shared_quot = 0;
                }
                CVL_TRY(bf(e, ba, sms * 16));
                GrowthArgsT<double> ga{};
                ga.md = md;
                ga.B = B;
                ga.M = cap.M;
                ga.pair_off = (const unsigned long long *)e->pair_off.p;
                ga.csr_ids = (const int *)e->csr_ids.p;
                ga.pcls = (const unsigned char *)e->pcls.p;
                ga.pflag = (const unsigned char *)e->pflag.p;
                ga.bund = (const double *)e->bund.p;
                ga.rec = rec;
                ga.arena_cap = arena_cap;
                ga.arena_ctr = arena_ctr;
                ga.rec_base = (unsigned *)e->rec_base.p;
                ga.run_cnt = (unsigned *)e->run_cnt.p;
                ga.count = (unsigned *)e->count.p;
                ga.stats = stats;
                ga.count_only = 0;
                ga.err = err;
                ga.cell_rank = (const unsigned short *)e->crank.p;
                // one arena record per curvelet, no chunk tails: the strided warps take
                // few anchors each
                ga.anchors_per_warp = 1;
                ga.cd = cdp + c;
                ga.queue = b == 1 ? queues + 1 : nullptr;
                CVL_TRY(gf(e, ga, gsmem, sms * 4 * tn.growth_blocks_per_sm));
            }
            CVL_TRY((scan<unsigned, unsigned long long>(e, (const unsigned *)e->count.p, N,
                                                        (unsigned long long *)e->out_off.p)));
            k_finalize<double><<<gb, 256, 0, s>>>(md, d_edges, sz, N, d_map_off, cap.M, rec,
                                                  (const unsigned *)e->rec_base.p, (const unsigned *)e->run_cnt.p,
                                                  (const unsigned long long *)e->out_off.p, C_cap,
                                                  (unsigned *)e->chains.p, (double *)e->info.p, dd);
            CVL_TRY(check_launch("k_finalize"));
            k_graph_readback<<<(cap.M + 1 + 255) / 256, 256, 0, s>>>(dd, (const unsigned long long *)e->pair_off.p,
                                                                     (const unsigned long long *)e->out_off.p,
                                                                     d_map_off, (unsigned long long *)e->gread.p);
            CVL_TRY(check_launch("k_graph_readback"));
            CVL_CUDA(cudaMemcpyAsync(rb_h, e->gread.p, (size_t)(2 + cap.M + 1) * 8, cudaMemcpyDeviceToHost, s));
            CVL_CUDA(cudaMemcpyAsync(stats_h, e->stats.p, sizeof(MapStats) * cap.M, cudaMemcpyDeviceToHost, s));
            CVL_CUDA(cudaMemcpyAsync(err_h, e->err.p, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
            return CVL_OK;
        };
        const int rc = enqueue();
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(s, &graph);
        if (rc != CVL_OK || ce != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            if (rc != CVL_OK) return rc;
            return fail(CVL_ECUDA, std::string("graph capture: ") + cudaGetErrorString(ce));
        }
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) {
            cudaGetLastError();
            return fail(CVL_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(ie));
        }
        if (e->graphs.size() >= GRAPH_SLOTS) {
            auto lru = std::min_element(e->graphs.begin(), e->graphs.end(),
                                        [](const auto &a, const auto &b2) { return a.last_use < b2.last_use; });
            cudaGraphExecDestroy(lru->exec);
            e->graphs.erase(lru);
        }
        e->graphs.push_back({key, exec, g_launches, 0});
        slot = &e->graphs.back();
        ++e->graph_captures;
    }
    slot->last_use = ++e->graph_clock;

    // the run: its sizes to the device, then the graph
    dims_h->N = n;
    dims_h->M = M;
    e->mark("start");
    CVL_CUDA(cudaMemcpyAsync(e->gdims.p, dims_h, sizeof(RunDims), cudaMemcpyHostToDevice, s));
    CVL_CUDA(cudaGraphLaunch(slot->exec, s));
    e->mark("graph");
    CVL_CUDA(cudaStreamSynchronize(s));
    g_launches = slot->launches;
    ++e->graph_replays;
    const unsigned h_err = *err_h;
    if (h_err & ERR_NONFINITE) return fail(CVL_EINVAL, "non-finite or out-of-range (|v| >= 1e9) edge coordinate");
    const unsigned long long P = rb_h[0], C = rb_h[1];
    if ((h_err & (ERR_CAPACITY | ERR_ARENA)) || C > C_cap) {
        ++e->graph_fallbacks;
        return CVL_EAGAIN;
    }
    if (h_err) return fail(CVL_EOVERFLOW, "kernel reported error bits " + std::to_string(h_err));
    ro.stats.assign(stats_h, stats_h + M);
    ro.max_deg = 0;
    for (const MapStats &st : ro.stats) ro.max_deg = std::max(ro.max_deg, st.max_deg);
    ro.total_pairs = P;
    ro.cv_off.assign(rb_h + 2, rb_h + 2 + M + 1);
    ro.total_curvelets = C;
    return CVL_OK;
}

// The workspace of a shape for an engine that replays graphs: each buffer at the
// larger of its size for the shape and its size for the graphs of the buckets that
// runs within the shape can use (buckets 0 and 1 up to the shape's edges), and the
// graphs' own small buffers.
std::vector<WsItem> workspace_plan_with_graphs(const cvl_tuning *tune, unsigned long long arena_hint, const Model &md,
                                               int cpl, const cvl_workspace_shape &s, bool graphs) {
    std::vector<WsItem> v = workspace_plan(tune, arena_hint, md, cpl, s);
    if (!graphs) return v;
    const int top = std::min(bucket_of((long long)s.num_edges), 1);
    for (int b = 0; b <= top; ++b) {
        const GraphCaps cap = GRAPH_CAPS[b];
        const unsigned long long per_chunk = std::max<unsigned long long>((unsigned long long)tune[b].chunk_pairs, 1024ull);
        cvl_workspace_shape g;
        g.num_edges = cap.N;
        g.num_pairs = (int64_t)(per_chunk * (unsigned long long)cap.K);
        g.num_curvelets = (int64_t)cap.N * cap.curvelets_per_edge;
        g.num_maps = cap.M;
        g.edge_data_sz = s.edge_data_sz;
        for (const WsItem &w : workspace_plan(tune, arena_hint, md, cpl, g)) {
            if (w.buf == &cvl_engine::edges || w.buf == &cvl_engine::map_off) continue;  // the caller's input
            for (WsItem &x : v)
                if (x.buf == w.buf) x.bytes = std::max(x.bytes, w.bytes);
        }
        v.push_back({&cvl_engine::gdims, sizeof(RunDims), false});
        v.push_back({&cvl_engine::gchunks, sizeof(ChunkDims) * (size_t)cap.K, false});
        v.push_back({&cvl_engine::gread, (size_t)(2 + cap.M + 1) * 8, false});
    }
    return v;
}

// The path: a bucket's graph where the run fits one, else the kernels launched one by one.
template <typename R>
int run_pipeline(cvl_engine *e, const R *d_edges, int n, int sz, const int *d_map_off,
                 const std::vector<int32_t> &map_off_host, ModelT<R> md, int cpl, int mode, bool want_d2,
                 RunOut &ro) {
    if constexpr (std::is_same<R, double>::value) {
        if (mode == 0 && !want_d2) {
            const int rc = run_pipeline_graph(e, d_edges, n, sz, d_map_off, map_off_host, md, cpl, ro);
            if (rc != CVL_EAGAIN) return rc;
        }
    }
    return run_pipeline_direct(e, d_edges, n, sz, d_map_off, map_off_host, md, cpl, mode, want_d2, ro);
}

template <typename T>
int upload(cvl_engine *e, const T *edges, int n, int sz, const std::vector<int32_t> &map_off) {
    CVL_TRY(e->alloc(e->edges, sizeof(T) * (size_t)n * sz));
    CVL_TRY(e->alloc(e->map_off, sizeof(int) * map_off.size()));
    CVL_CUDA(cudaMemcpyAsync(e->edges.p, edges, sizeof(T) * (size_t)n * sz, cudaMemcpyHostToDevice, e->stream));
    CVL_CUDA(cudaMemcpyAsync(e->map_off.p, map_off.data(), sizeof(int) * map_off.size(), cudaMemcpyHostToDevice,
                             e->stream));
    return CVL_OK;
}

int check_edges_args(const void *edges, int32_t n, int32_t sz) {
    if (n <= 0 || sz < 4 || edges == nullptr)  // preprocess.hpp:197-199
        return fail(CVL_EINVAL, "num_edges must be > 0, edge_data_sz >= 4 and edges non-NULL");
    return CVL_OK;
}

int fill_view_from_run(cvl_engine *e, const RunOut &ro, int n, int width, cvl_result *r) {
    const unsigned long long C = ro.total_curvelets;
    r->pool = e->pinned;
    r->chains_p = e->pinned->get(sizeof(unsigned) * (C ? C : 1) * width);
    r->info_p = e->pinned->get(sizeof(double) * (C ? C : 1) * 10);
    if (!r->chains_p || !r->info_p) return fail(CVL_ENOMEM, "page-locked result buffers could not be allocated");
    if (C) {
        CVL_CUDA(cudaMemcpyAsync(r->chains_p, e->chains.p, sizeof(unsigned) * C * width, cudaMemcpyDeviceToHost,
                                 e->stream));
        CVL_CUDA(cudaMemcpyAsync(r->info_p, e->info.p, sizeof(double) * C * 10, cudaMemcpyDeviceToHost, e->stream));
    }
    CVL_CUDA(cudaStreamSynchronize(e->stream));
    cvl_result_view &v = r->v;
    v.num_curvelets = (uint32_t)C;
    v.chain_width = (uint32_t)width;
    v.chains = (const uint32_t *)r->chains_p;
    v.info = (const double *)r->info_p;
    v.valid_pairs = ro.stats.empty() ? 0 : ro.stats[0].valid_pairs;
    v.total_neighbor_pairs = (int64_t)ro.total_pairs;
    v.max_num_of_neighbors = ro.max_deg;
    v.truncated_anchors = ro.stats.empty() ? 0 : ro.stats[0].truncated;
    v.num_edges = (uint32_t)n;
    v.flags = v.truncated_anchors ? CVL_FLAG_TRUNCATED : 0u;
    v.device_ms = e->last_device_ms;
    return CVL_OK;
}

}  // namespace

// =============================================================================
// C ABI
// =============================================================================
extern "C" {

void cvl_params_default(cvl_params *p) {
    if (!p) return;
    p->nrad = 3.5;
    p->gap = 1.5;
    p->dx = 0.4;
    p->dt_deg = 15.0;
    p->dt_rad = 0.0;
    p->max_k = 0.3;
    p->curvelet_style = 2;
    p->group_max_sz = 4;
    p->out_type = 0;
    p->sx = 0.1;
    p->st = 0.08;
    p->edge_data_sz = 4;
    p->max_candidates = 128;
}

void cvl_engine_cfg_default(cvl_engine_cfg *c) {
    if (!c) return;
    c->device = 0;
    c->mem_budget_bytes = 0;
    c->cell_size = 0;
    c->seeds_per_group = 0;
    c->bundle_slots = 0;
    c->stream_priority = 0;
    c->warps_per_block = 0;
}

const char *cvl_last_error(void) { return g_err.c_str(); }

int cvl_debug_fail_allocations(int64_t after) {
    if (after < -1) return fail(CVL_EINVAL, "after must be >= -1");
    g_fail_after.store(after);
    return CVL_OK;
}

const char *cvl_version(void) { return "cvl 0.1.0 (sm_100a, FP64)"; }

int cvl_engine_create(const cvl_engine_cfg *cfg, cvl_engine **out) {
    if (!out) return fail(CVL_EINVAL, "out is NULL");
    *out = nullptr;
    cvl_engine_cfg c;
    cvl_engine_cfg_default(&c);
    if (cfg) c = *cfg;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(CVL_ENODEV, "no CUDA device");
    }
    if (c.device < 0 || c.device >= ndev) return fail(CVL_EINVAL, "device ordinal out of range");
    cvl_engine *e = new cvl_engine();
    e->device = c.device;
    e->budget = c.mem_budget_bytes;
    e->cell_size = c.cell_size > 0 ? c.cell_size : 4;
    e->seeds_per_group = (c.seeds_per_group == 8) ? 8 : 4;
    {
        // measured on B200: 4-pixel blocks for batches up to 512 Ki edges, 8-pixel
        // blocks above (the spatial hash then touches fewer buckets per window)
        for (int b = 0; b < CVL_TUNING_BUCKETS; ++b) {
            const int dflt = b >= 2 ? 8 : 4;
            const int cs = (c.cell_size == 2 || c.cell_size == 4 || c.cell_size == 8) ? c.cell_size : dflt;
            e->tune[b] = default_tuning(cs, e->seeds_per_group);
        }
        // batches above 4 Mi edges: bundle chunks of 8 Mi pairs (an 8 GB bundle
        // buffer), half the bundle/growth launches of 4 Mi; measured on the 64-map
        // batch (33.7M edges): 1.6% faster than 4 Mi. 16 Mi was 0.6% faster again on
        // the resident batch but 4.5% slower through cvl_run_maps (its result copies
        // run beside the compute); smaller chunks were slower everywhere
        e->tune[CVL_TUNING_BUCKETS - 1].chunk_pairs = (int64_t)(8ull << 20);
    }
    e->slots = c.bundle_slots > 0 ? c.bundle_slots : 10;
    cudaError_t ce = cudaSetDevice(e->device);
    if (ce == cudaSuccess) ce = cudaGetDeviceProperties(&e->prop, e->device);
    if (ce == cudaSuccess) {
        int least = 0, greatest = 0;
        ce = cudaDeviceGetStreamPriorityRange(&least, &greatest);
        // lower numbers are higher priorities; clamp to the device's range
        const int prio = std::min(std::max(c.stream_priority, greatest), least);
        if (ce == cudaSuccess) ce = cudaStreamCreateWithPriority(&e->stream, cudaStreamNonBlocking, prio);
    }
    if (ce == cudaSuccess) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = e->device;
        ce = cudaMemPoolCreate(&e->pool, &props);
        if (ce == cudaSuccess) {
            uint64_t keep = UINT64_MAX;
            ce = cudaMemPoolSetAttribute(e->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    if (ce != cudaSuccess) {
        if (e->pool) cudaMemPoolDestroy(e->pool);
        if (e->stream) cudaStreamDestroy(e->stream);
        delete e;
        return fail(CVL_ECUDA, std::string("engine init: ") + cudaGetErrorString(ce));
    }
    if (e->prop.major < 10) {
        cudaMemPoolDestroy(e->pool);
        cudaStreamDestroy(e->stream);
        delete e;
        return fail(CVL_ENODEV, "device is not sm_100 class (the library is built for sm_100a only)");
    }
    *out = e;
    return CVL_OK;
}

void cvl_engine_destroy(cvl_engine *e) {
    if (!e) return;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    while (!e->batches.empty()) cvl_batch_free(e->batches.back());
    e->release_all();
    cudaStreamSynchronize(e->stream);
    for (cudaEvent_t ev : e->marks) cudaEventDestroy(ev);
    for (auto &g : e->graphs)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    if (e->gread_host) cudaFreeHost(e->gread_host);
    if (e->chunk_done) cudaEventDestroy(e->chunk_done);
    if (e->dev_done) cudaEventDestroy(e->dev_done);
    if (e->copy_stream) {
        cudaStreamSynchronize(e->copy_stream);
        cudaStreamSynchronize(e->upload_stream);
        for (int k = 0; k < 2; ++k) {
            cudaEventDestroy(e->computed[k]);
            cudaEventDestroy(e->copied[k]);
            cudaEventDestroy(e->uploaded[k]);
            cudaEventDestroy(e->consumed[k]);
        }
        cudaStreamDestroy(e->copy_stream);
        cudaStreamDestroy(e->upload_stream);
    }
    cudaStreamDestroy(e->stream);
    if (e->pool) cudaMemPoolDestroy(e->pool);
    delete e;
}

}  // extern "C"

// run_curvelet<T> on one map: the plain form in either scalar type.
template <typename T>
static int run_plain(cvl_engine *e, const T *edges, int32_t num_edges, int32_t edge_data_sz, const cvl_params *p,
                     cvl_result **out) {
    if (!e || !out) return fail(CVL_EINVAL, "engine/out is NULL");
    *out = nullptr;
    CVL_TRY(check_edges_args(edges, num_edges, edge_data_sz));
    CVL_CUDA(cudaSetDevice(e->device));
    ModelT<T> md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, p ? p->nrad : 0.0, 3u, p ? p->max_candidates : 0u, md, cpl));
    std::vector<int32_t> mo = {0, num_edges};
    CVL_TRY(upload(e, edges, num_edges, edge_data_sz, mo));
    RunOut ro;
    CVL_TRY(run_pipeline(e, (const T *)e->edges.p, num_edges, edge_data_sz, (const int *)e->map_off.p, mo, md, cpl,
                         0, false, ro));
    e->collect_marks();
    cvl_result *r = new cvl_result();
    int rc = fill_view_from_run(e, ro, num_edges, md.gms + 1, r);
    if (rc != CVL_OK) {
        delete r;
        return rc;
    }
    *out = r;
    return CVL_OK;
}

extern "C" {

int cvl_run(cvl_engine *e, const double *edges, int32_t num_edges, int32_t edge_data_sz, const cvl_params *p,
            cvl_result **out) {
    return run_plain<double>(e, edges, num_edges, edge_data_sz, p, out);
}

int cvl_run_f32(cvl_engine *e, const float *edges, int32_t num_edges, int32_t edge_data_sz, const cvl_params *p,
                cvl_result **out) {
    return run_plain<float>(e, edges, num_edges, edge_data_sz, p, out);
}

int cvl_result_get(const cvl_result *r, cvl_result_view *view) {
    if (!r || !view) return fail(CVL_EINVAL, "result/view is NULL");
    *view = r->v;
    return CVL_OK;
}

void cvl_result_free(cvl_result *r) { delete r; }

int cvl_build_neighbor_graph(cvl_engine *e, const double *edges, int32_t num_edges, int32_t edge_data_sz, double rad,
                             unsigned neighbor_radius, unsigned max_candidates, cvl_graph **out) {
    if (!e || !out) return fail(CVL_EINVAL, "engine/out is NULL");
    *out = nullptr;
    CVL_TRY(check_edges_args(edges, num_edges, edge_data_sz));
    CVL_CUDA(cudaSetDevice(e->device));
    cvl_params p;
    cvl_params_default(&p);
    p.nrad = rad;
    p.max_candidates = max_candidates;
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, &p, rad, neighbor_radius, max_candidates, md, cpl));
    std::vector<int32_t> mo = {0, num_edges};
    CVL_TRY(upload(e, edges, num_edges, edge_data_sz, mo));
    RunOut ro;
    CVL_TRY(run_pipeline(e, (const double *)e->edges.p, num_edges, edge_data_sz, (const int *)e->map_off.p, mo, md,
                         cpl, 2, true, ro));
    if (ro.total_pairs > 0x7fffffffull) return fail(CVL_EOVERFLOW, "more than 2^31 neighbour pairs");
    const int n = num_edges;
    const unsigned long long P = ro.total_pairs;
    CVL_TRY(e->alloc(e->deg_orig, sizeof(unsigned) * n));
    CVL_TRY(e->alloc(e->off_orig, sizeof(unsigned long long) * (n + 1)));
    CVL_TRY(e->alloc(e->gids, sizeof(int) * P));
    CVL_TRY(e->alloc(e->gd2, sizeof(double) * P));
    const int gb = grid_for(e, n, 256);
    k_graph_degrees<<<gb, 256, 0, e->stream>>>(n, (const int *)e->orig_of.p, (const unsigned long long *)e->pair_off.p,
                                              (unsigned *)e->deg_orig.p);
    CVL_TRY(check_launch("k_graph_degrees"));
    CVL_TRY((scan<unsigned, unsigned long long>(e, (const unsigned *)e->deg_orig.p, n,
                                                (unsigned long long *)e->off_orig.p)));
    k_graph_export<<<gb, 256, 0, e->stream>>>(n, (const int *)e->orig_of.p, (const int *)e->map_off.p, 1,
                                             (const unsigned long long *)e->pair_off.p, (const int *)e->csr_ids.p,
                                             (const double *)e->csr_d2.p, (const unsigned long long *)e->off_orig.p,
                                             (int *)e->gids.p, (double *)e->gd2.p);
    CVL_TRY(check_launch("k_graph_export"));
    e->mark("export");
    cvl_graph *g = new cvl_graph();
    g->edges.assign(edges, edges + (size_t)n * edge_data_sz);
    g->sz = edge_data_sz;
    g->n = n;
    g->rad = rad;
    g->neighbor_radius = neighbor_radius;
    g->max_candidates = max_candidates;
    std::vector<unsigned long long> off(n + 1);
    g->ids.resize(P);
    g->d2.resize(P);
    cudaMemcpyAsync(off.data(), e->off_orig.p, sizeof(unsigned long long) * (n + 1), cudaMemcpyDeviceToHost, e->stream);
    if (P) {
        cudaMemcpyAsync(g->ids.data(), e->gids.p, sizeof(int) * P, cudaMemcpyDeviceToHost, e->stream);
        cudaMemcpyAsync(g->d2.data(), e->gd2.p, sizeof(double) * P, cudaMemcpyDeviceToHost, e->stream);
    }
    cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) {
        delete g;
        return fail(CVL_ECUDA, std::string("graph download: ") + cudaGetErrorString(ce));
    }
    e->collect_marks();
    g->offsets.resize(n + 1);
    for (int i = 0; i <= n; ++i) g->offsets[i] = (int32_t)off[i];
    g->v.num_edges = n;
    g->v.total_neighbor_pairs = (int64_t)P;
    g->v.max_num_of_neighbors = ro.max_deg;
    g->v.truncated_anchors = ro.stats[0].truncated;
    g->v.neighbor_offsets = g->offsets.data();
    g->v.neighbor_ids = g->ids.data();
    g->v.neighbor_dist2 = g->d2.data();
    *out = g;
    return CVL_OK;
}

int cvl_graph_get(const cvl_graph *g, cvl_graph_view *view) {
    if (!g || !view) return fail(CVL_EINVAL, "graph/view is NULL");
    *view = g->v;
    return CVL_OK;
}

void cvl_graph_free(cvl_graph *g) { delete g; }

static int graph_pipeline(cvl_engine *e, const cvl_graph *g, const cvl_params *p, int mode, RunOut &ro, int &width) {
    if (!e || !g) return fail(CVL_EINVAL, "engine/graph is NULL");
    CVL_CUDA(cudaSetDevice(e->device));
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, g->rad, g->neighbor_radius, g->max_candidates, md, cpl));
    std::vector<int32_t> mo = {0, g->n};
    CVL_TRY(upload(e, g->edges.data(), g->n, g->sz, mo));
    CVL_TRY(run_pipeline(e, (const double *)e->edges.p, g->n, g->sz, (const int *)e->map_off.p, mo, md, cpl, mode,
                         false, ro));
    width = md.gms + 1;
    return CVL_OK;
}

int cvl_form_pairwise_bundles(cvl_engine *e, const cvl_graph *g, const cvl_params *p, uint32_t *valid_pairs) {
    if (!valid_pairs) return fail(CVL_EINVAL, "valid_pairs is NULL");
    RunOut ro;
    int width = 0;
    CVL_TRY(graph_pipeline(e, g, p, 1, ro, width));
    e->collect_marks();
    *valid_pairs = ro.stats[0].valid_pairs;
    return CVL_OK;
}

int cvl_build_curvelets(cvl_engine *e, const cvl_graph *g, const cvl_params *p, cvl_result **out) {
    if (!out) return fail(CVL_EINVAL, "out is NULL");
    *out = nullptr;
    RunOut ro;
    int width = 0;
    CVL_TRY(graph_pipeline(e, g, p, 0, ro, width));
    e->collect_marks();
    cvl_result *r = new cvl_result();
    int rc = fill_view_from_run(e, ro, g->n, width, r);
    if (rc != CVL_OK) {
        delete r;
        return rc;
    }
    *out = r;
    return CVL_OK;
}

namespace {

// Pairs through k_pair_bundles on the engine's stream (form 0: the production
// transport; form 1: the reference's two branches as written).
int pair_bundles_form(cvl_engine *e, const double *pairs, int32_t n, const cvl_params *p, int form, double *bmin,
                      double *bmax, uint8_t *valid, int32_t *cells) {
    if (!e || !pairs || !bmin || !bmax || !valid || !cells || n < 0) return fail(CVL_EINVAL, "invalid argument");
    CVL_CUDA(cudaSetDevice(e->device));
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, p ? p->nrad : 0.0, 3u, p ? std::max(p->max_candidates, 1u) : 1u, md, cpl));
    *cells = md.cells;
    if (n == 0) return CVL_OK;
    CVL_TRY(e->alloc(e->pairs_in, sizeof(double) * 6 * n));
    CVL_TRY(e->alloc(e->pb_min, sizeof(double) * (size_t)n * md.cells));
    CVL_TRY(e->alloc(e->pb_max, sizeof(double) * (size_t)n * md.cells));
    CVL_TRY(e->alloc(e->pb_valid, (size_t)n));
    cudaStream_t s = e->stream;
    CVL_CUDA(cudaMemcpyAsync(e->pairs_in.p, pairs, sizeof(double) * 6 * n, cudaMemcpyHostToDevice, s));
    const int blocks = grid_for(e, n, 4, 16);
    k_pair_bundles<<<blocks, 128, 0, s>>>(md, (const double *)e->pairs_in.p, n, form, (double *)e->pb_min.p,
                                          (double *)e->pb_max.p, (unsigned char *)e->pb_valid.p, nullptr);
    CVL_TRY(check_launch("k_pair_bundles"));
    CVL_CUDA(cudaMemcpyAsync(bmin, e->pb_min.p, sizeof(double) * (size_t)n * md.cells, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(bmax, e->pb_max.p, sizeof(double) * (size_t)n * md.cells, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(valid, e->pb_valid.p, (size_t)n, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaStreamSynchronize(s));
    return CVL_OK;
}

}  // namespace

int cvl_pair_bundles(cvl_engine *e, const double *pairs, int32_t n, const cvl_params *p, double *bmin, double *bmax,
                     uint8_t *valid, int32_t *cells) {
    return pair_bundles_form(e, pairs, n, p, 0, bmin, bmax, valid, cells);
}

int cvl_check_pair_bundles_literal(cvl_engine *e, const double *pairs, int32_t n, const cvl_params *p, double *bmin,
                                   double *bmax, uint8_t *valid, int32_t *cells) {
    return pair_bundles_form(e, pairs, n, p, 1, bmin, bmax, valid, cells);
}

int cvl_check_transport_cells(cvl_engine *e, const double *ops, int32_t n, const cvl_params *p, int32_t quotients,
                              double *out, int32_t *rows) {
    if (!e || !ops || !out || !rows || n < 0) return fail(CVL_EINVAL, "invalid argument");
    CVL_CUDA(cudaSetDevice(e->device));
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, p ? p->nrad : 0.0, 3u, p ? std::max(p->max_candidates, 1u) : 1u, md, cpl));
    *rows = md.P;
    if (n == 0) return CVL_OK;
    const size_t out_n = (size_t)n * 4 * md.P;
    CVL_TRY(e->alloc(e->pairs_in, sizeof(double) * 10 * (size_t)n));
    CVL_TRY(e->alloc(e->pb_min, sizeof(double) * out_n));
    cudaStream_t s = e->stream;
    CVL_CUDA(cudaMemcpyAsync(e->pairs_in.p, ops, sizeof(double) * 10 * (size_t)n, cudaMemcpyHostToDevice, s));
    k_transport_cells<<<grid_for(e, n, 128, 8), 128, 0, s>>>(md, (const double *)e->pairs_in.p, n,
                                                             quotients ? QUOT_CHECKED : QUOT_DIVIDE,
                                                             (double *)e->pb_min.p);
    CVL_TRY(check_launch("k_transport_cells"));
    CVL_CUDA(cudaMemcpyAsync(out, e->pb_min.p, sizeof(double) * out_n, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaStreamSynchronize(s));
    return CVL_OK;
}

// ---- device-resident batches -----------------------------------------------------
int cvl_batch_refill_parts(cvl_batch *b, const double *const *parts, const int32_t *counts, int32_t num_maps,
                           int32_t edge_data_sz) {
    if (!b || !parts || !counts || num_maps <= 0 || edge_data_sz < 4) return fail(CVL_EINVAL, "invalid batch arguments");
    for (int m = 0; m < num_maps; ++m)
        if (!parts[m]) return fail(CVL_EINVAL, "a map's edges are NULL");
    cvl_engine *e = b->eng;
    std::vector<int32_t> mo(num_maps + 1, 0);
    for (int m = 0; m < num_maps; ++m) {
        if (counts[m] <= 0) return fail(CVL_EINVAL, "every map needs at least one edge");
        if ((long long)mo[m] + counts[m] > 0x7fffffffLL) return fail(CVL_EOVERFLOW, "batch larger than 2^31 edges");
        mo[m + 1] = mo[m] + counts[m];
    }
    CVL_CUDA(cudaSetDevice(e->device));
    const size_t eb = sizeof(double) * (size_t)mo[num_maps] * edge_data_sz;
    if (eb > b->edges_cap) {
        // grow-only: a refill that fits reuses the buffer (no cudaFree, which would
        // synchronise the whole device)
        const size_t want = std::max(eb, b->edges_cap + b->edges_cap / 4);
        if (b->d_edges) {
            cudaFreeAsync(b->d_edges, e->stream);
            e->held -= b->edges_cap;
            b->d_edges = nullptr;
            b->edges_cap = 0;
        }
        if (e->budget && e->held + want > e->budget) return fail(CVL_ENOMEM, "batch exceeds the device memory budget");
        if (cvl_alloc_fault_injected() || cudaMallocFromPoolAsync(&b->d_edges, want, e->pool, e->stream) != cudaSuccess) {
            cudaGetLastError();
            b->d_edges = nullptr;
            return fail(CVL_ENOMEM, "batch allocation failed");
        }
        b->edges_cap = want;
        e->held += want;
    }
    if ((size_t)mo.size() > b->map_off_cap) {
        const size_t want = std::max(mo.size(), b->map_off_cap * 2);
        if (b->d_map_off) cudaFreeAsync(b->d_map_off, e->stream);
        b->d_map_off = nullptr;
        b->map_off_cap = 0;
        if (cudaMallocFromPoolAsync(&b->d_map_off, sizeof(int) * want, e->pool, e->stream) != cudaSuccess) {
            cudaGetLastError();
            b->d_map_off = nullptr;
            return fail(CVL_ENOMEM, "batch allocation failed");
        }
        b->map_off_cap = want;
    }
    b->num_maps = num_maps;
    b->sz = edge_data_sz;
    b->n = mo[num_maps];
    b->map_off = mo;
    // one copy per contiguous run of parts (a single copy for one concatenated buffer)
    for (int m = 0; m < num_maps;) {
        int k = m + 1;
        while (k < num_maps && parts[k] == parts[k - 1] + (size_t)counts[k - 1] * edge_data_sz) ++k;
        CVL_CUDA(copy_pieces((double *)b->d_edges + (size_t)mo[m] * edge_data_sz, parts[m],
                             sizeof(double) * (size_t)(mo[k] - mo[m]) * edge_data_sz, cudaMemcpyHostToDevice,
                             e->stream));
        m = k;
    }
    CVL_CUDA(cudaMemcpyAsync(b->d_map_off, b->map_off.data(), sizeof(int) * mo.size(), cudaMemcpyHostToDevice,
                             e->stream));
    const cudaError_t ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return fail(CVL_ECUDA, std::string("batch upload: ") + cudaGetErrorString(ce));
    return CVL_OK;
}

int cvl_batch_refill(cvl_batch *b, const double *edges, const int32_t *counts, int32_t num_maps,
                     int32_t edge_data_sz) {
    if (!b || !edges || !counts || num_maps <= 0 || edge_data_sz < 4) return fail(CVL_EINVAL, "invalid batch arguments");
    std::vector<const double *> parts(num_maps);
    size_t o = 0;
    for (int m = 0; m < num_maps; ++m) {
        parts[m] = edges + o;
        o += (size_t)std::max(counts[m], 0) * edge_data_sz;
    }
    return cvl_batch_refill_parts(b, parts.data(), counts, num_maps, edge_data_sz);
}

int cvl_batch_upload(cvl_engine *e, const double *edges, const int32_t *counts, int32_t num_maps, int32_t edge_data_sz,
                     cvl_batch **out) {
    if (!e || !edges || !counts || !out || num_maps <= 0 || edge_data_sz < 4)
        return fail(CVL_EINVAL, "invalid batch arguments");
    *out = nullptr;
    cvl_batch *b = new cvl_batch();
    b->eng = e;
    e->batches.push_back(b);
    const int rc = cvl_batch_refill(b, edges, counts, num_maps, edge_data_sz);
    if (rc != CVL_OK) {
        const std::string msg = g_err;
        cvl_batch_free(b);
        return fail(rc, msg);
    }
    *out = b;
    return CVL_OK;
}

void cvl_batch_free(cvl_batch *b) {
    if (!b) return;
    auto &bs = b->eng->batches;
    bs.erase(std::remove(bs.begin(), bs.end(), b), bs.end());
    cudaSetDevice(b->eng->device);
    if (b->d_edges) {
        cudaFreeAsync(b->d_edges, b->eng->stream);
        b->eng->held -= b->edges_cap;
    }
    if (b->d_map_off) cudaFreeAsync(b->d_map_off, b->eng->stream);
    delete b;
}

int cvl_batch_run(cvl_engine *e, const cvl_batch *b, const cvl_params *p, cvl_batch_result **out) {
    if (!e || !b || !out) return fail(CVL_EINVAL, "engine/batch/out is NULL");
    if (b->eng != e) return fail(CVL_EINVAL, "batch belongs to another engine");
    *out = nullptr;
    CVL_CUDA(cudaSetDevice(e->device));
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, p ? p->nrad : 0.0, 3u, p ? p->max_candidates : 0u, md, cpl));
    RunOut ro;
    CVL_TRY(run_pipeline(e, (const double *)b->d_edges, b->n, b->sz, (const int *)b->d_map_off, b->map_off, md, cpl, 0,
                         false, ro));
    CVL_CUDA(cudaStreamSynchronize(e->stream));
    e->collect_marks();
    cvl_batch_result *r = new cvl_batch_result();
    r->eng = e;
    r->generation = e->generation;
    r->num_maps = b->num_maps;
    r->n = b->n;
    r->width = md.gms + 1;
    r->map_off = b->map_off;
    r->stats = ro.stats;
    r->cv_off = ro.cv_off;
    r->device_ms = e->last_device_ms;
    r->launches = e->last_launches;
    *out = r;
    return CVL_OK;
}

int cvl_batch_result_map(cvl_batch_result *r, int32_t m, cvl_result_view *view) {
    if (!r || !view || m < 0 || m >= r->num_maps) return fail(CVL_EINVAL, "invalid batch result arguments");
    if (!r->downloaded) {
        if (r->eng->generation != r->generation)
            return fail(CVL_EINVAL, "batch result outputs were overwritten by a later run on the engine");
        CVL_CUDA(cudaSetDevice(r->eng->device));
        const unsigned long long C = r->cv_off[r->num_maps];
        r->pinned = r->eng->pinned;
        r->chains = (uint32_t *)r->pinned->get(sizeof(unsigned) * (C ? C : 1) * r->width);
        r->info = (double *)r->pinned->get(sizeof(double) * (C ? C : 1) * 10);
        if (!r->chains || !r->info) return fail(CVL_ENOMEM, "page-locked result buffers could not be allocated");
        if (C) {
            CVL_CUDA(cudaMemcpyAsync(r->chains, r->eng->chains.p, sizeof(unsigned) * C * r->width,
                                     cudaMemcpyDeviceToHost, r->eng->stream));
            CVL_CUDA(cudaMemcpyAsync(r->info, r->eng->info.p, sizeof(double) * C * 10, cudaMemcpyDeviceToHost,
                                     r->eng->stream));
        }
        CVL_CUDA(cudaStreamSynchronize(r->eng->stream));
        r->downloaded = true;
    }
    const unsigned long long c0 = r->cv_off[m], c1 = r->cv_off[m + 1];
    cvl_result_view &v = *view;
    v.num_curvelets = (uint32_t)(c1 - c0);
    v.chain_width = (uint32_t)r->width;
    v.chains = r->chains + c0 * r->width;
    v.info = r->info + c0 * 10;
    v.valid_pairs = r->stats[m].valid_pairs;
    v.total_neighbor_pairs = (int64_t)r->stats[m].pairs;
    v.max_num_of_neighbors = r->stats[m].max_deg;
    v.truncated_anchors = r->stats[m].truncated;
    v.num_edges = (uint32_t)(r->map_off[m + 1] - r->map_off[m]);
    v.flags = v.truncated_anchors ? CVL_FLAG_TRUNCATED : 0u;
    v.device_ms = r->device_ms;
    return CVL_OK;
}

int cvl_batch_result_take_map(cvl_batch_result *r, int32_t m, cvl_result **out) {
    if (!r || !out || m < 0 || m >= r->num_maps) return fail(CVL_EINVAL, "invalid batch result arguments");
    *out = nullptr;
    if (!r->downloaded && r->eng->generation != r->generation)
        return fail(CVL_EINVAL, "batch result outputs were overwritten by a later run on the engine");
    cvl_engine *e = r->eng;
    CVL_CUDA(cudaSetDevice(e->device));
    const unsigned long long c0 = r->cv_off[m], c1 = r->cv_off[m + 1], C = c1 - c0;
    cvl_result *res = new cvl_result();
    res->pool = e->pinned;
    res->chains_p = e->pinned->get(sizeof(unsigned) * (C ? C : 1) * r->width);
    res->info_p = e->pinned->get(sizeof(double) * (C ? C : 1) * 10);
    if (!res->chains_p || !res->info_p) {
        delete res;
        return fail(CVL_ENOMEM, "page-locked result buffers could not be allocated");
    }
    if (C) {
        if (r->downloaded) {
            std::memcpy(res->chains_p, r->chains + c0 * r->width, sizeof(unsigned) * C * r->width);
            std::memcpy(res->info_p, r->info + c0 * 10, sizeof(double) * C * 10);
        } else {
            cudaError_t ce = copy_result_to_host(res->chains_p, (const unsigned *)e->chains.p + c0 * r->width,
                                                 sizeof(unsigned) * C * r->width, e->stream);
            if (ce == cudaSuccess)
                ce = copy_result_to_host(res->info_p, (const double *)e->info.p + c0 * 10, sizeof(double) * C * 10,
                                         e->stream);
            if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
            if (ce != cudaSuccess) {
                delete res;
                return fail(CVL_ECUDA, std::string("result download: ") + cudaGetErrorString(ce));
            }
        }
    }
    cvl_result_view &v = res->v;
    v.num_curvelets = (uint32_t)C;
    v.chain_width = (uint32_t)r->width;
    v.chains = (const uint32_t *)res->chains_p;
    v.info = (const double *)res->info_p;
    v.valid_pairs = r->stats[m].valid_pairs;
    v.total_neighbor_pairs = (int64_t)r->stats[m].pairs;
    v.max_num_of_neighbors = r->stats[m].max_deg;
    v.truncated_anchors = r->stats[m].truncated;
    v.num_edges = (uint32_t)(r->map_off[m + 1] - r->map_off[m]);
    v.flags = v.truncated_anchors ? CVL_FLAG_TRUNCATED : 0u;
    v.device_ms = r->device_ms;
    *out = res;
    return CVL_OK;
}

int cvl_batch_result_stats(const cvl_batch_result *r, cvl_batch_stats *out) {
    if (!r || !out) return fail(CVL_EINVAL, "result/out is NULL");
    cvl_batch_stats st{};
    for (const MapStats &m : r->stats) {
        st.valid_pairs += m.valid_pairs;
        st.total_pairs += m.pairs;
        st.close_pairs += m.close_pairs;
        st.max_num_of_neighbors = std::max<uint32_t>(st.max_num_of_neighbors, m.max_deg);
        st.truncated_anchors += m.truncated;
    }
    st.device_ms = r->device_ms;
    st.num_curvelets = r->cv_off[r->num_maps];
    st.num_maps = (uint32_t)r->num_maps;
    st.launches = (uint32_t)r->launches;
    *out = st;
    return CVL_OK;
}

void cvl_batch_result_free(cvl_batch_result *r) { delete r; }

int cvl_tuning_bucket(int64_t num_edges) { return bucket_of((long long)num_edges); }

}  // extern "C"

void cvl_engine_set_yield(cvl_engine *e, cvl_yield_fn fn, void *ctx) {
    if (!e) return;
    e->yield_fn = fn;
    e->yield_ctx = ctx;
}

int cvl_engine_reserve_device(cvl_engine *e, size_t bytes) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    if (!bytes) return CVL_OK;
    CVL_CUDA(cudaSetDevice(e->device));
    void *p = nullptr;
    if (cvl_alloc_fault_injected() || cudaMallocFromPoolAsync(&p, bytes, e->pool, e->stream) != cudaSuccess) {
        cudaGetLastError();
        return fail(CVL_ENOMEM, "device memory could not be reserved (" + std::to_string(bytes) + " bytes)");
    }
    CVL_CUDA(cudaFreeAsync(p, e->stream));
    CVL_CUDA(cudaStreamSynchronize(e->stream));
    return CVL_OK;
}

static int workspace_bytes_impl(const cvl_tuning *tune, bool graphs, const cvl_workspace_shape *s,
                                const cvl_params *p, size_t *total, size_t *per_launch);

extern "C" {

int cvl_engine_workspace_bytes(cvl_engine *e, const cvl_workspace_shape *s, const cvl_params *p, size_t *total,
                               size_t *per_launch) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    return workspace_bytes_impl(e->tune, e->graphs_on, s, p, total, per_launch);
}

int cvl_engine_reserve_workspace(cvl_engine *e, const cvl_workspace_shape *s, const cvl_params *p) {
    size_t total = 0;
    CVL_TRY(cvl_engine_workspace_bytes(e, s, p, &total, nullptr));
    CVL_CUDA(cudaSetDevice(e->device));
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, p->nrad, 3u, p->max_candidates, md, cpl));
    // the record arena of later runs holds at least the shape's curvelets
    e->arena_hint = std::max<unsigned long long>(e->arena_hint, (unsigned long long)s->num_curvelets);
    for (const WsItem &w : workspace_plan_with_graphs(e->tune, e->arena_hint, md, cpl, *s, e->graphs_on))
        CVL_TRY(e->alloc(e->*(w.buf), w.bytes));
    if (e->graphs_on && !e->gread_host) {  // the graphs' page-locked readback
        void *h = nullptr;
        if (cvl_alloc_fault_injected() || cudaMallocHost(&h, graph_readback_bytes() + sizeof(RunDims) + 64) != cudaSuccess) {
            cudaGetLastError();
            return fail(CVL_ENOMEM, "page-locked graph readback could not be allocated");
        }
        e->gread_host = (unsigned char *)h;
    }
    CVL_CUDA(cudaStreamSynchronize(e->stream));
    return CVL_OK;
}

int cvl_engine_set_graphs(cvl_engine *e, int enable) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    e->graphs_on = enable != 0;
    return CVL_OK;
}

// Rings of edgels (position, tangent orientation, strength 1) centred on a grid of
// tiles: a built-in map of about tiles^2 x 520 edges for the warm-up.
static std::vector<double> warmup_map(int tiles) {
    std::vector<double> v;
    const double two_pi = 2.0 * CVL_PI;
    for (int ty = 0; ty < tiles; ++ty)
        for (int tx = 0; tx < tiles; ++tx) {
            const double cx = 60.0 + 120.0 * tx, cy = 60.0 + 120.0 * ty;
            for (double r : {11.0, 23.0, 48.0}) {
                const int k = (int)(two_pi * r);
                for (int i = 0; i < k; ++i) {
                    const double phi = two_pi * i / k;
                    const double th = std::fmod(phi + 0.5 * CVL_PI, two_pi);
                    v.insert(v.end(), {cx + r * std::cos(phi), cy + r * std::sin(phi), th, 1.0});
                }
            }
        }
    return v;
}

int cvl_engine_warmup(cvl_engine *e) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    cvl_params p;
    cvl_params_default(&p);
    const bool graphs = e->graphs_on;
    // a small map (the bucket-0 graph, or its kernels one by one), and a map above
    // 64 Ki edges (the persistent grids, and the bucket-1 graph)
    const std::vector<double> small = warmup_map(1), large = warmup_map(12);
    int rc = CVL_OK;
    for (const std::vector<double> *m : {&small, &large})
        for (int g = 0; g < 2 && rc == CVL_OK; ++g) {
            e->graphs_on = graphs && g == 0;
            cvl_result *r = nullptr;
            rc = cvl_run(e, m->data(), (int32_t)(m->size() / 4), 4, &p, &r);
            cvl_result_free(r);
            if (!graphs) break;
        }
    e->graphs_on = graphs;
    return rc;
}

int cvl_engine_graph_stats(cvl_engine *e, cvl_engine_graphs *out) {
    if (!e || !out) return fail(CVL_EINVAL, "engine/out is NULL");
    out->enabled = e->graphs_on ? 1 : 0;
    out->graphs = (int32_t)e->graphs.size();
    out->captures = e->graph_captures;
    out->replays = e->graph_replays;
    out->fallbacks = e->graph_fallbacks;
    return CVL_OK;
}

int cvl_engine_memory_get(cvl_engine *e, cvl_engine_memory *out) {
    if (!e || !out) return fail(CVL_EINVAL, "engine/out is NULL");
    out->held_bytes = e->held;
    out->device_grows = e->dev_grows.load();
    out->device_grow_ms = (double)e->dev_grow_ns.load() * 1e-6;
    return CVL_OK;
}

}  // extern "C"

int cvl_workspace_bytes_tuned(const cvl_tuning *tune, const cvl_workspace_shape *s, const cvl_params *p,
                              size_t *total, size_t *per_launch) {
    return workspace_bytes_impl(tune, false, s, p, total, per_launch);
}

static int workspace_bytes_impl(const cvl_tuning *tune, bool graphs, const cvl_workspace_shape *s,
                                const cvl_params *p, size_t *total, size_t *per_launch) {
    if (!tune || !s || !p || !total) return fail(CVL_EINVAL, "tuning/shape/params/total is NULL");
    if (s->num_edges < 1 || s->num_edges > 0x7fffffffLL || s->num_pairs < 0 || s->num_curvelets < 0 ||
        s->num_maps < 1 || s->edge_data_sz < 4)
        return fail(CVL_EINVAL, "workspace shape out of range");
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(nullptr, p, p->nrad, 3u, p->max_candidates, md, cpl));
    size_t t = 0, c = 0;
    for (const WsItem &w : workspace_plan_with_graphs(tune, 0, md, cpl, *s, graphs)) {
        t += round256(w.bytes);
        if (w.per_launch) c += round256(w.bytes);
    }
    *total = t;
    if (per_launch) *per_launch = c;
    return CVL_OK;
}

int cvl_batch_create_reserved(cvl_engine *e, int64_t max_edges, int32_t max_maps, int32_t edge_data_sz,
                              cvl_batch **out) {
    if (!e || !out || max_edges < 1 || max_maps < 1 || edge_data_sz < 4) return fail(CVL_EINVAL, "invalid batch arguments");
    *out = nullptr;
    CVL_CUDA(cudaSetDevice(e->device));
    cvl_batch *b = new cvl_batch();
    b->eng = e;
    const size_t eb = sizeof(double) * (size_t)max_edges * (size_t)edge_data_sz;
    const size_t mb = sizeof(int) * ((size_t)max_maps + 1);
    if (e->budget && e->held + eb > e->budget) {
        delete b;
        return fail(CVL_ENOMEM, "batch exceeds the device memory budget");
    }
    if (cvl_alloc_fault_injected() || cudaMallocFromPoolAsync(&b->d_edges, eb, e->pool, e->stream) != cudaSuccess ||
        cudaMallocFromPoolAsync(&b->d_map_off, mb, e->pool, e->stream) != cudaSuccess) {
        cudaGetLastError();
        if (b->d_edges) cudaFreeAsync(b->d_edges, e->stream);
        if (b->d_map_off) cudaFreeAsync(b->d_map_off, e->stream);
        delete b;
        return fail(CVL_ENOMEM, "batch allocation failed");
    }
    e->dev_grows += 2;
    b->edges_cap = eb;
    b->map_off_cap = (size_t)max_maps + 1;
    e->held += eb;
    b->sz = edge_data_sz;
    e->batches.push_back(b);
    CVL_CUDA(cudaStreamSynchronize(e->stream));
    *out = b;
    return CVL_OK;
}

int cvl_engine_reserve_host(cvl_engine *e, size_t bytes) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    if (bytes && !e->pinned->reserve(bytes)) return fail(CVL_ENOMEM, "page-locked host memory could not be reserved");
    return CVL_OK;
}

extern "C" {

int cvl_engine_get_tuning(cvl_engine *e, int bucket, cvl_tuning *t) {
    if (!e || !t || bucket < 0 || bucket >= CVL_TUNING_BUCKETS) return fail(CVL_EINVAL, "invalid tuning arguments");
    *t = e->tune[bucket];
    return CVL_OK;
}

int cvl_engine_set_tuning(cvl_engine *e, int bucket, const cvl_tuning *t) {
    if (!e || !t || bucket < -1 || bucket >= CVL_TUNING_BUCKETS) return fail(CVL_EINVAL, "invalid tuning arguments");
    CVL_TRY(check_tuning(*t));
    if (bucket < 0) {
        for (cvl_tuning &x : e->tune) x = *t;
    } else {
        e->tune[bucket] = *t;
    }
    return CVL_OK;
}

int cvl_engine_autotune(cvl_engine *e, const cvl_batch *b, const cvl_params *p, int passes, cvl_tuning *best,
                        double *best_ms) {
    if (!e || !b || !p || !best || !best_ms || passes < 1) return fail(CVL_EINVAL, "invalid autotune arguments");
    const int bucket = bucket_of(b->n);
    // one untimed run (workspace growth), then the median of three device times
    auto time_it = [&](const cvl_tuning &t, double &ms) -> int {
        e->tune[bucket] = t;
        double v[4];
        for (int k = 0; k < 4; ++k) {
            cvl_batch_result *r = nullptr;
            CVL_TRY(cvl_batch_run(e, b, p, &r));
            v[k] = r->device_ms;
            cvl_batch_result_free(r);
        }
        std::sort(v + 1, v + 4);
        ms = v[2];
        return CVL_OK;
    };
    cvl_tuning cur = e->tune[bucket];
    double cur_ms = 0.0;
    CVL_TRY(time_it(cur, cur_ms));
    const int64_t chunks[] = {1LL << 20, 4LL << 20, 16LL << 20};
    const int apws[] = {1, 2, 4, 8, 16};
    const int cells[] = {2, 4, 8};
    const int growth[][2] = {{4, 4}, {4, 6}, {4, 8}, {8, 4}};  // (seeds_per_group, blocks per SM)
    for (int pass = 0; pass < passes; ++pass) {
        auto consider = [&](const cvl_tuning &t) -> int {
            if (std::memcmp(&t, &cur, sizeof(t)) == 0) return CVL_OK;
            double ms = 0.0;
            CVL_TRY(time_it(t, ms));
            if (ms < cur_ms * 0.99) {
                cur = t;
                cur_ms = ms;
            }
            return CVL_OK;
        };
        for (int v : {3, 4}) {
            cvl_tuning t = cur;
            t.bundle_blocks_per_sm = v;
            CVL_TRY(consider(t));
        }
        for (const auto &g : growth) {
            cvl_tuning t = cur;
            t.seeds_per_group = g[0];
            t.growth_blocks_per_sm = g[1];
            CVL_TRY(consider(t));
        }
        for (int v : apws) {
            cvl_tuning t = cur;
            t.anchors_per_warp = v;
            CVL_TRY(consider(t));
        }
        for (int v : cells) {
            cvl_tuning t = cur;
            t.cell_size = v;
            CVL_TRY(consider(t));
        }
        for (int64_t v : chunks) {
            cvl_tuning t = cur;
            t.chunk_pairs = v;
            CVL_TRY(consider(t));
        }
    }
    e->tune[bucket] = cur;
    *best = cur;
    *best_ms = cur_ms;
    return CVL_OK;
}

int cvl_engine_flush_l2(cvl_engine *e) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    CVL_CUDA(cudaSetDevice(e->device));
    const size_t bytes = std::max<size_t>((size_t)e->prop.l2CacheSize * 2, (size_t)256 << 20);
    CVL_TRY(e->alloc(e->flush, bytes));
    k_flush<<<e->prop.multiProcessorCount * 8, 256, 0, e->stream>>>((unsigned *)e->flush.p, bytes / 4, 7u);
    CVL_TRY(check_launch("k_flush"));
    CVL_CUDA(cudaStreamSynchronize(e->stream));
    return CVL_OK;
}

int cvl_engine_last_kernel_times(cvl_engine *e, const char **names, double *ms, int cap) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    const int n = (int)e->last_times.size();
    for (int k = 0; k < n && k < cap; ++k) {
        if (names) names[k] = e->last_times[k].first;
        if (ms) ms[k] = e->last_times[k].second;
    }
    return n;
}

int cvl_engine_last_launch_count(cvl_engine *e) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    return e->last_launches;
}

int cvl_measure_fp64_peak(cvl_engine *e, double *tflops) {
    if (!e || !tflops) return fail(CVL_EINVAL, "invalid argument");
    CVL_CUDA(cudaSetDevice(e->device));
    CVL_TRY(e->alloc(e->flush, 1024));
    const int blocks = e->prop.multiProcessorCount * 8, threads = 256, iters = 4096;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    k_fp64_peak<<<blocks, threads, 0, e->stream>>>((double *)e->flush.p, 64, 1.0);  // warm-up
    cudaEventRecord(a, e->stream);
    k_fp64_peak<<<blocks, threads, 0, e->stream>>>((double *)e->flush.p, iters, 1.0);
    cudaEventRecord(b, e->stream);
    cudaError_t ce = cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ce != cudaSuccess) return fail(CVL_ECUDA, std::string("fp64 probe: ") + cudaGetErrorString(ce));
    const double fmas = (double)blocks * threads * iters * 16.0 * 8.0;
    *tflops = 2.0 * fmas / (ms * 1e-3) / 1e12;
    return CVL_OK;
}

}  // extern "C"

// =============================================================================
// Pair bundles without any allocation (cvl_pair_bundles_noalloc)
// =============================================================================
namespace {

// Per-device scratch of cvl_pair_bundles_noalloc, laid out per call as
//   [0, 256)  valid-pair counter (u32; cleared by every call)
//   pairs [n][6] f64 | bmin [n][cells] f64 | bmax [n][cells] f64 | valid [n] u8,
// each piece starting on a 256-byte boundary.
__device__ __align__(256) unsigned char g_noalloc_scratch[CVL_NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;
std::mutex g_noalloc_mu;

size_t noalloc_bytes(size_t n, size_t cells) {
    return 256 + round256(48 * n) + 2 * round256(8 * n * cells) + round256(n);
}

// The set-up of a device: the scratch's device address, looked up with that
// device current. The address belongs to the device's current context, so it is
// kept with that context's id (cuCtxGetId): after a context is destroyed and
// created again (cudaDeviceReset, for one), the module is loaded again, the array
// can land elsewhere, and the next call does the set-up again.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

struct NoallocSetup {
    unsigned long long ctx_id = 0;  // 0: not set up
    unsigned char *base = nullptr;
};
NoallocSetup g_noalloc_setup[NOALLOC_MAX_DEVICES];

int current_context_id(unsigned long long *id) {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    if (!get_current || !get_id) {
        void *f0 = nullptr, *f1 = nullptr;
        cudaDriverEntryPointQueryResult q0{}, q1{};
        CVL_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f0, 12000, cudaEnableDefault, &q0));
        CVL_CUDA(cudaGetDriverEntryPointByVersion("cuCtxGetId", &f1, 12000, cudaEnableDefault, &q1));
        if (q0 != cudaDriverEntryPointSuccess || q1 != cudaDriverEntryPointSuccess || !f0 || !f1)
            return fail(CVL_ECUDA, "the driver does not provide cuCtxGetCurrent / cuCtxGetId");
        get_current = (CtxGetCurrentFn)f0;
        get_id = (CtxGetIdFn)f1;
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx) return fail(CVL_ECUDA, "no current CUDA context");
    if (get_id(ctx, id) != CUDA_SUCCESS) return fail(CVL_ECUDA, "cuCtxGetId failed");
    return CVL_OK;
}

int noalloc_scratch(int dev, unsigned char **out) {
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(CVL_EUNSUPPORTED, "device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    unsigned long long id = 0;
    CVL_TRY(current_context_id(&id));
    NoallocSetup &su = g_noalloc_setup[dev];
    if (su.ctx_id != id || !su.base) {
        void *ptr = nullptr;
        const cudaError_t ce = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (ce != cudaSuccess || !ptr)
            return fail(CVL_ECUDA, std::string("scratch address: ") + cudaGetErrorString(ce));
        su.base = (unsigned char *)ptr;
        su.ctx_id = id;
    }
    *out = su.base;
    return CVL_OK;
}

}  // namespace

extern "C" {

int cvl_pair_bundles_noalloc(const double *pairs, int32_t n, const cvl_params *p, double *bmin, double *bmax,
                             uint8_t *valid, uint32_t *valid_pairs, int32_t *cells) {
    if (!pairs || !bmin || !bmax || !valid || !valid_pairs || !cells || n < 0)
        return fail(CVL_EINVAL, "invalid argument");
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(nullptr, p, p ? p->nrad : 0.0, 3u, p ? std::max(p->max_candidates, 1u) : 1u, md, cpl));
    *cells = md.cells;
    *valid_pairs = 0;
    const size_t need = noalloc_bytes((size_t)n, (size_t)md.cells);
    if (need > CVL_NOALLOC_SCRATCH_BYTES) {
        size_t max_n = 0;
        while (noalloc_bytes(max_n + 1, (size_t)md.cells) <= CVL_NOALLOC_SCRATCH_BYTES) ++max_n;
        return fail(CVL_EOVERFLOW, std::to_string(n) + " pairs need " + std::to_string(need) +
                                       " bytes of scratch; the fixed scratch holds " +
                                       std::to_string((size_t)CVL_NOALLOC_SCRATCH_BYTES) + " bytes, at most " +
                                       std::to_string(max_n) + " pairs of " + std::to_string(md.cells) + " cells");
    }
    if (n == 0) return CVL_OK;
    int dev = 0, ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(CVL_ENODEV, "no CUDA device");
    }
    CVL_CUDA(cudaGetDevice(&dev));
    cudaStream_t s = cudaStreamPerThread;
    // The call ends with a synchronisation of the calling thread's stream, which a
    // capture in progress on that stream would not survive.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    CVL_CUDA(cudaStreamIsCapturing(s, &cap));
    if (cap != cudaStreamCaptureStatusNone)
        return fail(CVL_EINVAL, "cvl_pair_bundles_noalloc cannot run while the calling thread's stream is capturing");
    unsigned char *base = nullptr;
    CVL_TRY(noalloc_scratch(dev, &base));
    int sms = 0;
    CVL_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));

    const size_t cells_n = (size_t)n * md.cells;
    unsigned *d_count = (unsigned *)base;
    double *d_pairs = (double *)(base + 256);
    double *d_bmin = (double *)((unsigned char *)d_pairs + round256(48 * (size_t)n));
    double *d_bmax = (double *)((unsigned char *)d_bmin + round256(8 * cells_n));
    unsigned char *d_valid = (unsigned char *)d_bmax + round256(8 * cells_n);

    CVL_CUDA(cudaMemsetAsync(d_count, 0, sizeof(unsigned), s));
    CVL_CUDA(cudaMemcpyAsync(d_pairs, pairs, 48 * (size_t)n, cudaMemcpyHostToDevice, s));
    long long blocks = ((long long)n + 3) / 4;
    blocks = std::max(1LL, std::min(blocks, (long long)sms * 16));
    k_pair_bundles<<<(int)blocks, 128, 0, s>>>(md, d_pairs, n, 0, d_bmin, d_bmax, d_valid, d_count);
    CVL_TRY(check_launch("k_pair_bundles"));
    CVL_CUDA(cudaMemcpyAsync(bmin, d_bmin, 8 * cells_n, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(bmax, d_bmax, 8 * cells_n, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(valid, d_valid, (size_t)n, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(valid_pairs, d_count, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaStreamSynchronize(s));
    return CVL_OK;
}

}  // extern "C"


// =============================================================================
// Downstream: curvelets -> edgel link graph -> contour fragments (cvl_contours.cuh)
// =============================================================================
struct cvl_contours {
    std::shared_ptr<PinnedPool> pool;
    void *links_p = nullptr;  // pe, ce, votes: 3 x num_links int32
    void *offs_p = nullptr;
    void *ids_p = nullptr;
    std::vector<int64_t> poly_offsets;
    std::vector<int32_t> poly_ids;
    std::vector<double> poly_info;
    cvl_contours_view v{};
    ~cvl_contours() {
        if (pool) {
            pool->put(links_p);
            pool->put(offs_p);
            pool->put(ids_p);
        }
    }
};

namespace {

// The stage on device-resident edges (double AoS) and chains, on the engine's
// stream; copies the link list and the fragments into *c.
int contours_on_device(cvl_engine *e, const double *d_edges, int n, int sz, const unsigned *d_chains, long long C,
                       int W, const cvl_contour_params &cp, cvl_contours *c) {
    using namespace cvlc;
    if (W < 2 || W > 64) return fail(CVL_EINVAL, "chain_width must be in [2, 64]");
    if (n >= (1 << 30)) return fail(CVL_EOVERFLOW, "the link graph takes fewer than 2^30 edges");
    if ((unsigned long long)C * (unsigned long long)(W - 1) >= (1ull << 32))
        return fail(CVL_EOVERFLOW, "too many curvelets for the link graph (rows x (width - 1) >= 2^32)");
    if (!(cp.gap >= 0.0) || !std::isfinite(cp.gap)) return fail(CVL_EINVAL, "gap must be finite and >= 0");
    cudaStream_t s = e->stream;
    auto &w = e->cw;
    const size_t N = (size_t)n;
    const unsigned long long occ_cap = 2ull * (unsigned long long)C * (unsigned long long)std::max(W - 2, 1);
    CVL_TRY(e->alloc(w.cnt, sizeof(unsigned) * N));
    CVL_TRY(e->alloc(w.cursor, sizeof(unsigned) * N));
    CVL_TRY(e->alloc(w.off, sizeof(unsigned long long) * (N + 1)));
    CVL_TRY(e->alloc(w.bucket, sizeof(uint2) * std::max<unsigned long long>(occ_cap, 1)));
    CVL_TRY(e->alloc(w.outdeg, sizeof(int) * N));
    CVL_TRY(e->alloc(w.indeg, sizeof(int) * N));
    CVL_TRY(e->alloc(w.child, sizeof(int) * N));
    CVL_TRY(e->alloc(w.parent, sizeof(int) * N));
    CVL_TRY(e->alloc(w.succ, sizeof(int) * N));
    CVL_TRY(e->alloc(w.pred, sizeof(int) * N));
    CVL_TRY(e->alloc(w.flags, N));
    CVL_TRY(e->alloc(w.linked, N));
    CVL_TRY(e->alloc(w.loff, sizeof(unsigned long long) * (N + 1)));
    CVL_TRY(e->alloc(w.lpe, sizeof(int) * std::max<unsigned long long>(occ_cap / 2, 1)));
    CVL_TRY(e->alloc(w.lce, sizeof(int) * std::max<unsigned long long>(occ_cap / 2, 1)));
    CVL_TRY(e->alloc(w.lvotes, sizeof(int) * std::max<unsigned long long>(occ_cap / 2, 1)));
    CVL_TRY(e->alloc(w.firsts, sizeof(unsigned) * N));
    const unsigned long long region_cap = 3ull * N + 16;
    CVL_TRY(e->alloc(w.region, sizeof(int) * region_cap));
    CVL_TRY(e->alloc(w.ctr, sizeof(unsigned long long) * 2));
    CVL_TRY(e->alloc(w.fsrc, sizeof(unsigned long long) * N));
    CVL_TRY(e->alloc(w.fnf, sizeof(int) * N));
    CVL_TRY(e->alloc(w.fnb, sizeof(int) * N));
    CVL_TRY(e->alloc(w.isfrag, sizeof(unsigned) * N));
    CVL_TRY(e->alloc(w.flen, sizeof(unsigned long long) * N));
    CVL_TRY(e->alloc(w.fidx, sizeof(unsigned) * (N + 1)));
    CVL_TRY(e->alloc(w.idoff, sizeof(unsigned long long) * (N + 1)));
    CVL_TRY(e->alloc(w.fragoff, sizeof(long long) * (N + 1)));
    CVL_TRY(e->alloc(w.fragids, sizeof(int) * region_cap));
    CVL_TRY(e->alloc(w.err, sizeof(unsigned) * 4));

    CVL_CUDA(cudaMemsetAsync(w.cnt.p, 0, sizeof(unsigned) * N, s));
    CVL_CUDA(cudaMemsetAsync(w.cursor.p, 0, sizeof(unsigned) * N, s));
    CVL_CUDA(cudaMemsetAsync(w.ctr.p, 0, sizeof(unsigned long long) * 2, s));
    CVL_CUDA(cudaMemsetAsync(w.fnf.p, 0xff, sizeof(int) * N, s));  // -1: no fragment starts here
    CVL_CUDA(cudaMemsetAsync(w.err.p, 0, sizeof(unsigned) * 4, s));
    unsigned *err = (unsigned *)w.err.p;

    const int rb = (int)std::max(1LL, (C + 255) / 256);
    const int nb = (int)((N + 255) / 256);
    if (C > 0) {
        k_link_count<<<rb, 256, 0, s>>>(d_chains, C, W, cp.min_group_size, n, (unsigned *)w.cnt.p, err);
        CVL_TRY(check_launch("k_link_count"));
    }
    CVL_TRY((scan<unsigned, unsigned long long>(e, (const unsigned *)w.cnt.p, N, (unsigned long long *)w.off.p)));
    if (C > 0) {
        k_link_fill<<<rb, 256, 0, s>>>(d_chains, C, W, cp.min_group_size, n, (const unsigned long long *)w.off.p,
                                       (unsigned *)w.cursor.p, (uint2 *)w.bucket.p);
        CVL_TRY(check_launch("k_link_fill"));
    }
    Graph g;
    g.n = n;
    g.occ_off = (const unsigned long long *)w.off.p;
    g.bucket = (uint2 *)w.bucket.p;
    g.outdeg = (int *)w.outdeg.p;
    g.indeg = (int *)w.indeg.p;
    g.child = (int *)w.child.p;
    g.parent = (int *)w.parent.p;
    g.succ = (int *)w.succ.p;
    g.pred = (int *)w.pred.p;
    g.flags = (unsigned char *)w.flags.p;
    g.linked = (unsigned char *)w.linked.p;
    k_link_degrees<<<nb, 256, 0, s>>>(g);
    CVL_TRY(check_launch("k_link_degrees"));
    CVL_TRY((scan<unsigned, unsigned long long>(e, (const unsigned *)w.outdeg.p, N, (unsigned long long *)w.loff.p)));
    k_link_list<<<nb, 256, 0, s>>>(g, (const unsigned long long *)w.loff.p, (int *)w.lpe.p, (int *)w.lce.p,
                                   (int *)w.lvotes.p);
    CVL_TRY(check_launch("k_link_list"));
    k_link_paths<<<nb, 256, 0, s>>>(g);
    CVL_TRY(check_launch("k_link_paths"));
    FragOut o;
    o.edges = d_edges;
    o.sz = sz;
    o.thres = cp.gap * cp.gap;
    o.first_ids = (unsigned *)w.firsts.p;
    o.first_ctr = (unsigned long long *)w.ctr.p;
    o.region = (int *)w.region.p;
    o.region_ctr = (unsigned long long *)w.ctr.p + 1;
    o.region_cap = region_cap;
    o.first_cap = N;
    o.frag_src = (unsigned long long *)w.fsrc.p;
    o.frag_nf = (int *)w.fnf.p;
    o.frag_nb = (int *)w.fnb.p;
    o.err = err;
    // one thread per edge; short blocks, since a few threads trace long components
    const int nb128 = (int)((N + 127) / 128);
    k_trace_paths<<<nb128, 128, 0, s>>>(g, o);
    CVL_TRY(check_launch("k_trace_paths"));
    k_trace_cycles<<<nb128, 128, 0, s>>>(g, o);
    CVL_TRY(check_launch("k_trace_cycles"));
    k_frag_sizes<<<nb, 256, 0, s>>>(n, (const int *)w.fnf.p, (const int *)w.fnb.p, (unsigned *)w.isfrag.p,
                                    (unsigned long long *)w.flen.p);
    CVL_TRY(check_launch("k_frag_sizes"));
    CVL_TRY((scan<unsigned, unsigned>(e, (const unsigned *)w.isfrag.p, N, (unsigned *)w.fidx.p)));
    CVL_TRY((scan<unsigned long long, unsigned long long>(e, (const unsigned long long *)w.flen.p, N,
                                                           (unsigned long long *)w.idoff.p)));
    k_frag_write<<<nb, 256, 0, s>>>(n, (const int *)w.fnf.p, (const int *)w.fnb.p,
                                    (const unsigned long long *)w.fsrc.p, (const int *)w.region.p,
                                    (const unsigned *)w.fidx.p, (const unsigned long long *)w.idoff.p,
                                    (long long *)w.fragoff.p, (int *)w.fragids.p);
    CVL_TRY(check_launch("k_frag_write"));
    e->mark("contours");

    unsigned long long h_links = 0, h_ids = 0;
    unsigned h_frags = 0, h_err = 0;
    CVL_CUDA(cudaMemcpyAsync(&h_links, (unsigned long long *)w.loff.p + N, sizeof(h_links), cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(&h_ids, (unsigned long long *)w.idoff.p + N, sizeof(h_ids), cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(&h_frags, (unsigned *)w.fidx.p + N, sizeof(h_frags), cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaMemcpyAsync(&h_err, err, sizeof(h_err), cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaStreamSynchronize(s));
    if (h_err & ERR_ID) return fail(CVL_EINVAL, "a curvelet chain holds an edge id outside the map");
    if (h_err) return fail(CVL_EOVERFLOW, "contour kernels reported error bits " + std::to_string(h_err));

    c->pool = e->pinned;
    c->links_p = e->pinned->get(sizeof(int) * 3 * (h_links ? h_links : 1));
    c->offs_p = e->pinned->get(sizeof(long long) * (h_frags + 1));
    c->ids_p = e->pinned->get(sizeof(int) * (h_ids ? h_ids : 1));
    if (!c->links_p || !c->offs_p || !c->ids_p)
        return fail(CVL_ENOMEM, "page-locked result buffers could not be allocated");
    int *lp = (int *)c->links_p;
    if (h_links) {
        CVL_CUDA(cudaMemcpyAsync(lp, w.lpe.p, sizeof(int) * h_links, cudaMemcpyDeviceToHost, s));
        CVL_CUDA(cudaMemcpyAsync(lp + h_links, w.lce.p, sizeof(int) * h_links, cudaMemcpyDeviceToHost, s));
        CVL_CUDA(cudaMemcpyAsync(lp + 2 * h_links, w.lvotes.p, sizeof(int) * h_links, cudaMemcpyDeviceToHost, s));
    }
    CVL_CUDA(cudaMemcpyAsync(c->offs_p, w.fragoff.p, sizeof(long long) * (h_frags + 1), cudaMemcpyDeviceToHost, s));
    if (h_ids) CVL_CUDA(cudaMemcpyAsync(c->ids_p, w.fragids.p, sizeof(int) * h_ids, cudaMemcpyDeviceToHost, s));
    CVL_CUDA(cudaStreamSynchronize(s));
    if (h_frags == 0) ((long long *)c->offs_p)[0] = 0;
    cvl_contours_view &v = c->v;
    v.num_links = (int64_t)h_links;
    v.link_parent = lp;
    v.link_child = lp + h_links;
    v.link_votes = lp + 2 * h_links;
    v.num_fragments = (int64_t)h_frags;
    v.fragment_offsets = (const int64_t *)c->offs_p;
    v.fragment_ids = (const int32_t *)c->ids_p;
    int32_t mx = 0;
    for (unsigned f = 0; f < h_frags; ++f)
        mx = std::max<int32_t>(mx, (int32_t)(v.fragment_offsets[f + 1] - v.fragment_offsets[f]));
    v.max_fragment_length = mx;
    v.num_edges = n;
    v.num_polyarcs = 0;
    v.polyarc_offsets = nullptr;
    v.polyarc_ids = nullptr;
    v.polyarc_info = nullptr;
    if (cp.fit_polyarcs && h_frags > 0) {
        // the polyarc model: form_curvelet_process's dx, dt, max_k on CC_curve_model_3d's
        // fixed grid steps (0.1 px, 0.08 rad)
        cvl_params mp;
        cvl_params_default(&mp);
        mp.dx = cp.dx;
        mp.dt_rad = cp.dt_rad;
        mp.max_k = cp.max_k;
        mp.sx = 0.1;
        mp.st = 0.08;
        Model pm;
        int pcpl = 2;
        CVL_TRY(make_model(e, &mp, mp.nrad, 3u, mp.max_candidates, pm, pcpl));
        const unsigned long long slots = h_ids - h_frags;  // at most N - 1 per fragment of N edges
        CVL_TRY(e->alloc(w.pstart, sizeof(long long) * std::max<unsigned long long>(slots, 1)));
        CVL_TRY(e->alloc(w.psize, sizeof(int) * std::max<unsigned long long>(slots, 1)));
        CVL_TRY(e->alloc(w.pinfo, sizeof(double) * 12 * std::max<unsigned long long>(slots, 1)));
        CVL_TRY(e->alloc(w.pcount, sizeof(unsigned) * h_frags));
        CVL_TRY(e->alloc(w.poff, sizeof(unsigned long long) * (h_frags + 1)));
        PolyArgs pa;
        pa.md = pm;
        pa.edges = d_edges;
        pa.sz = sz;
        pa.nfrags = (int)h_frags;
        pa.frag_off = (const long long *)w.fragoff.p;
        pa.frag_ids = (const int *)w.fragids.p;
        pa.rad = cp.rad;
        pa.token_len = cp.token_len;
        pa.poly_start = (long long *)w.pstart.p;
        pa.poly_size = (int *)w.psize.p;
        pa.poly_info = (double *)w.pinfo.p;
        pa.poly_count = (unsigned *)w.pcount.p;
        const int pb = (int)std::max(1u, (h_frags + 3) / 4);
        switch (pcpl) {
            case 1: k_polyarcs<1><<<pb, 128, 0, s>>>(pa); break;
            case 3: k_polyarcs<3><<<pb, 128, 0, s>>>(pa); break;
            case 4: k_polyarcs<4><<<pb, 128, 0, s>>>(pa); break;
            default: k_polyarcs<2><<<pb, 128, 0, s>>>(pa); break;
        }
        CVL_TRY(check_launch("k_polyarcs"));
        CVL_TRY((scan<unsigned, unsigned long long>(e, (const unsigned *)w.pcount.p, h_frags,
                                                     (unsigned long long *)w.poff.p)));
        unsigned long long h_poly = 0;
        CVL_CUDA(cudaMemcpyAsync(&h_poly, (unsigned long long *)w.poff.p + h_frags, sizeof(h_poly),
                                 cudaMemcpyDeviceToHost, s));
        CVL_CUDA(cudaStreamSynchronize(s));
        CVL_TRY(e->alloc(w.pstart2, sizeof(long long) * std::max<unsigned long long>(h_poly, 1)));
        CVL_TRY(e->alloc(w.psize2, sizeof(int) * std::max<unsigned long long>(h_poly, 1)));
        CVL_TRY(e->alloc(w.pinfo2, sizeof(double) * 12 * std::max<unsigned long long>(h_poly, 1)));
        k_polyarcs_pack<<<(int)((h_frags + 255) / 256), 256, 0, s>>>(
            (int)h_frags, (const long long *)w.fragoff.p, (const unsigned *)w.pcount.p,
            (const unsigned long long *)w.poff.p, (const long long *)w.pstart.p, (const int *)w.psize.p,
            (const double *)w.pinfo.p, (long long *)w.pstart2.p, (int *)w.psize2.p, (double *)w.pinfo2.p);
        CVL_TRY(check_launch("k_polyarcs_pack"));
        e->mark("polyarcs");
        std::vector<long long> st(h_poly);
        std::vector<int> sizes(h_poly);
        c->poly_info.resize(12 * h_poly);
        if (h_poly) {
            CVL_CUDA(cudaMemcpyAsync(st.data(), w.pstart2.p, sizeof(long long) * h_poly, cudaMemcpyDeviceToHost, s));
            CVL_CUDA(cudaMemcpyAsync(sizes.data(), w.psize2.p, sizeof(int) * h_poly, cudaMemcpyDeviceToHost, s));
            CVL_CUDA(cudaMemcpyAsync(c->poly_info.data(), w.pinfo2.p, sizeof(double) * 12 * h_poly,
                                     cudaMemcpyDeviceToHost, s));
        }
        CVL_CUDA(cudaStreamSynchronize(s));
        c->poly_offsets.assign(h_poly + 1, 0);
        for (unsigned long long q = 0; q < h_poly; ++q) c->poly_offsets[q + 1] = c->poly_offsets[q] + sizes[q];
        c->poly_ids.resize((size_t)c->poly_offsets[h_poly] + 1);
        for (unsigned long long q = 0; q < h_poly; ++q)
            std::memcpy(c->poly_ids.data() + c->poly_offsets[q], v.fragment_ids + st[q], sizeof(int32_t) * sizes[q]);
        v.num_polyarcs = (int64_t)h_poly;
        v.polyarc_offsets = c->poly_offsets.data();
        v.polyarc_ids = c->poly_ids.data();
        v.polyarc_info = c->poly_info.data();
    } else if (cp.fit_polyarcs) {
        c->poly_offsets.assign(1, 0);
        v.polyarc_offsets = c->poly_offsets.data();
    }
    return CVL_OK;
}

// the caller's parameters, or the defaults with `gap` (CurveletParams::gap, the
// downstream stages' parameter, param_settings.hpp) when cp is NULL
int contour_params_of(const cvl_contour_params *cp, double gap, cvl_contour_params &out) {
    cvl_contour_params_default(&out);
    if (cp)
        out = *cp;
    else
        out.gap = gap;
    if (!(out.gap >= 0.0) || !std::isfinite(out.gap)) return fail(CVL_EINVAL, "gap must be finite and >= 0");
    if (out.fit_polyarcs && (!(out.dx > 0) || !(out.dt_rad > 0) || !std::isfinite(out.max_k) || !(out.rad > 0) ||
                             !(out.token_len > 0) || !std::isfinite(out.dx) || !std::isfinite(out.dt_rad)))
        return fail(CVL_EINVAL, "polyarc parameters: dx, dt_rad, rad and token_len must be finite and > 0");
    return CVL_OK;
}

}  // namespace

extern "C" {

void cvl_contour_params_default(cvl_contour_params *p) {
    if (!p) return;
    p->min_group_size = 4;
    p->gap = 1.5;
    p->fit_polyarcs = 0;
    p->dx = 0.4;
    p->dt_rad = (15.0 / 180.0) * CVL_PI;
    p->max_k = 0.3;
    p->rad = 3.5;
    p->token_len = 1.0;
}

int cvl_link_contours(cvl_engine *e, const double *edges, int32_t num_edges, int32_t edge_data_sz,
                      const uint32_t *chains, int64_t num_curvelets, int32_t chain_width,
                      const cvl_contour_params *cp, cvl_contours **out) {
    if (!e || !out) return fail(CVL_EINVAL, "engine/out is NULL");
    *out = nullptr;
    CVL_TRY(check_edges_args(edges, num_edges, edge_data_sz));
    if (num_curvelets < 0 || (num_curvelets > 0 && !chains)) return fail(CVL_EINVAL, "chains is NULL");
    if (chain_width < 2 || chain_width > 64) return fail(CVL_EINVAL, "chain_width must be in [2, 64]");
    cvl_contour_params p;
    CVL_TRY(contour_params_of(cp, 1.5, p));
    // the link graph visits anchors in ascending order (form_curvelet_process.cpp:479-491)
    for (int64_t r = 0; r < num_curvelets; ++r) {
        const uint32_t a = chains[(size_t)r * chain_width];
        if (a == 0 || a > (uint32_t)num_edges)
            return fail(CVL_EINVAL, "curvelet row " + std::to_string(r) + ": anchor id outside the map");
        if (r > 0 && a < chains[(size_t)(r - 1) * chain_width])
            return fail(CVL_EINVAL, "curvelet rows must be grouped by anchor in ascending order");
    }
    CVL_CUDA(cudaSetDevice(e->device));
    e->nmarks = 0;
    g_launches = 0;
    e->mark("start");
    std::vector<int32_t> mo = {0, num_edges};
    CVL_TRY(upload(e, edges, num_edges, edge_data_sz, mo));
    const size_t cbytes = sizeof(uint32_t) * (size_t)std::max<int64_t>(num_curvelets, 1) * chain_width;
    CVL_TRY(e->alloc(e->cw.chains_in, cbytes));
    if (num_curvelets > 0)
        CVL_CUDA(cudaMemcpyAsync(e->cw.chains_in.p, chains, sizeof(uint32_t) * (size_t)num_curvelets * chain_width,
                                 cudaMemcpyHostToDevice, e->stream));
    e->mark("upload");
    cvl_contours *c = new cvl_contours();
    int rc = contours_on_device(e, (const double *)e->edges.p, num_edges, edge_data_sz,
                                (const unsigned *)e->cw.chains_in.p, num_curvelets, chain_width, p, c);
    if (rc != CVL_OK) {
        delete c;
        return rc;
    }
    e->collect_marks();
    c->v.device_ms = (float)e->last_device_ms;
    *out = c;
    return CVL_OK;
}

int cvl_run_contours(cvl_engine *e, const double *edges, int32_t num_edges, int32_t edge_data_sz,
                     const cvl_params *p, const cvl_contour_params *cp, cvl_result **curvelets_out,
                     cvl_contours **out) {
    if (!e || !out) return fail(CVL_EINVAL, "engine/out is NULL");
    *out = nullptr;
    if (curvelets_out) *curvelets_out = nullptr;
    CVL_TRY(check_edges_args(edges, num_edges, edge_data_sz));
    cvl_contour_params q;
    CVL_TRY(contour_params_of(cp, p ? p->gap : 1.5, q));
    CVL_CUDA(cudaSetDevice(e->device));
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, p ? p->nrad : 0.0, 3u, p ? p->max_candidates : 0u, md, cpl));
    std::vector<int32_t> mo = {0, num_edges};
    CVL_TRY(upload(e, edges, num_edges, edge_data_sz, mo));
    RunOut ro;
    CVL_TRY(run_pipeline(e, (const double *)e->edges.p, num_edges, edge_data_sz, (const int *)e->map_off.p, mo, md,
                         cpl, 0, false, ro));
    cvl_contours *c = new cvl_contours();
    int rc = contours_on_device(e, (const double *)e->edges.p, num_edges, edge_data_sz, (const unsigned *)e->chains.p,
                                (long long)ro.total_curvelets, md.gms + 1, q, c);
    if (rc != CVL_OK) {
        delete c;
        return rc;
    }
    e->collect_marks();
    c->v.device_ms = (float)e->last_device_ms;
    if (curvelets_out) {
        cvl_result *r = new cvl_result();
        rc = fill_view_from_run(e, ro, num_edges, md.gms + 1, r);
        if (rc != CVL_OK) {
            delete r;
            delete c;
            return rc;
        }
        *curvelets_out = r;
    }
    *out = c;
    return CVL_OK;
}

int cvl_contours_get(const cvl_contours *c, cvl_contours_view *view) {
    if (!c || !view) return fail(CVL_EINVAL, "contours/view is NULL");
    *view = c->v;
    return CVL_OK;
}

void cvl_contours_free(cvl_contours *c) { delete c; }

}  // extern "C"


// =============================================================================
// Many maps, host to host, with the result copies behind the compute (by SM threads:
// copy_result_to_host)
// =============================================================================

extern "C" int cvl_run_maps(cvl_engine *e, const double *edges, const int32_t *counts, int32_t num_maps,
                            int32_t edge_data_sz, const cvl_params *p, int64_t group_edges, cvl_result **out) {
    if (!e || !edges || !counts || !out || num_maps <= 0 || edge_data_sz < 4)
        return fail(CVL_EINVAL, "invalid arguments");
    for (int32_t m = 0; m < num_maps; ++m) out[m] = nullptr;
    std::vector<long long> off(num_maps + 1, 0);
    for (int32_t m = 0; m < num_maps; ++m) {
        if (counts[m] <= 0) return fail(CVL_EINVAL, "map " + std::to_string(m) + ": num_edges must be > 0");
        off[m + 1] = off[m] + counts[m];
    }
    if (off[num_maps] > 0x7fffffffLL) return fail(CVL_EOVERFLOW, "more than 2^31 - 1 edges in one call");
    CVL_CUDA(cudaSetDevice(e->device));
    if (!e->copy_stream) {
        CVL_CUDA(cudaStreamCreateWithFlags(&e->copy_stream, cudaStreamNonBlocking));
        CVL_CUDA(cudaStreamCreateWithFlags(&e->upload_stream, cudaStreamNonBlocking));
        for (int k = 0; k < 2; ++k) {
            CVL_CUDA(cudaEventCreateWithFlags(&e->computed[k], cudaEventDisableTiming));
            CVL_CUDA(cudaEventCreateWithFlags(&e->copied[k], cudaEventDisableTiming));
            CVL_CUDA(cudaEventCreateWithFlags(&e->uploaded[k], cudaEventDisableTiming));
            CVL_CUDA(cudaEventCreateWithFlags(&e->consumed[k], cudaEventDisableTiming));
        }
    }

    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, p ? p->nrad : 0.0, 3u, p ? p->max_candidates : 0u, md, cpl));
    const int W = md.gms + 1;
    const long long total = off[num_maps];
    const bool default_groups = group_edges <= 0;
    if (default_groups) group_edges = std::min<long long>(std::max<long long>(total / 6, 1LL << 20), 8LL << 20);

    // The maps in the order they run: by default the smallest maps, about a sixteenth
    // of the edges (at least 256 Ki), are held back for a last group of their own, so
    // that the result copies left after the last compute are short.
    std::vector<int32_t> order;
    order.reserve(num_maps);
    std::vector<char> tail(num_maps, 0);
    if (default_groups && total > group_edges && num_maps > 1) {
        std::vector<int32_t> by_size(num_maps);
        for (int32_t m = 0; m < num_maps; ++m) by_size[m] = m;
        std::stable_sort(by_size.begin(), by_size.end(), [&](int32_t a, int32_t b) { return counts[a] < counts[b]; });
        const long long want = std::max<long long>(total / 16, 256LL << 10);
        long long got = 0;
        for (int32_t k = 0; k + 1 < num_maps && got < want; ++k) {
            tail[by_size[k]] = 1;
            got += counts[by_size[k]];
        }
    }
    for (int32_t m = 0; m < num_maps; ++m)
        if (!tail[m]) order.push_back(m);
    const size_t body = order.size();
    for (int32_t m = 0; m < num_maps; ++m)
        if (tail[m]) order.push_back(m);

    // groups of whole maps (positions in order), about group_edges edges each; the held
    // back maps form the last group
    std::vector<int32_t> gstart = {0};
    long long acc = 0;
    for (size_t k = 0; k < order.size(); ++k) {
        acc += counts[order[k]];
        const bool cut = (k + 1 == body) || (k + 1 < order.size() && acc >= group_edges && k + 1 < body);
        if (k + 1 < order.size() && cut) {
            gstart.push_back((int32_t)(k + 1));
            acc = 0;
        }
    }
    gstart.push_back(num_maps);
    const int G = (int)gstart.size() - 1;
    long long max_group = 0;
    for (int g = 0; g < G; ++g) {
        long long ng = 0;
        for (int k = gstart[g]; k < gstart[g + 1]; ++k) ng += counts[order[k]];
        max_group = std::max(max_group, ng);
    }

    // Two device edge buffers: a group's edges go up on the upload stream while the
    // group before computes (a host-to-device copy beside the path's kernels slows them
    // by 2% at most).
    DBuf *ebuf[2] = {&e->edges, &e->edges_alt};
    CVL_TRY(e->alloc(e->edges, sizeof(double) * (size_t)max_group * edge_data_sz));
    CVL_TRY(e->alloc(e->edges_alt, sizeof(double) * (size_t)max_group * edge_data_sz));
    for (int b = 0; b < 2; ++b) CVL_CUDA(cudaEventRecord(e->consumed[b], e->stream));
    auto upload_group = [&](int g) -> int {
        const int b = g & 1;
        CVL_CUDA(cudaStreamWaitEvent(e->upload_stream, e->consumed[b], 0));
        size_t at = 0;
        for (int k = gstart[g]; k < gstart[g + 1];) {
            // runs of maps that lie back to back in the host array go in one copy
            int k1 = k + 1;
            while (k1 < gstart[g + 1] && order[k1] == order[k1 - 1] + 1) ++k1;
            const size_t rows = (size_t)(off[order[k1 - 1] + 1] - off[order[k]]);
            CVL_CUDA(cudaMemcpyAsync((double *)ebuf[b]->p + at * edge_data_sz,
                                     edges + (size_t)off[order[k]] * edge_data_sz, sizeof(double) * rows * edge_data_sz,
                                     cudaMemcpyHostToDevice, e->upload_stream));
            at += rows;
            k = k1;
        }
        CVL_CUDA(cudaEventRecord(e->uploaded[b], e->upload_stream));
        return CVL_OK;
    };

    std::vector<cvl_result *> res(num_maps, nullptr);
    auto cleanup = [&](int rc) {
        cudaStreamSynchronize(e->copy_stream);
        cudaStreamSynchronize(e->upload_stream);
        for (cvl_result *r : res) delete r;
        return rc;
    };
    double device_ms = 0.0;
    bool copy_pending[2] = {false, false};
    if (int rc = upload_group(0)) return cleanup(rc);
    for (int g = 0; g < G; ++g) {
        const int m0 = gstart[g], m1 = gstart[g + 1], M = m1 - m0;
        const int buf = g & 1;
        if (g + 1 < G) {
            if (int rc = upload_group(g + 1)) return cleanup(rc);
        }
        // this group's outputs go to the buffer pair the group before last used:
        // its copies must be done before run_pipeline may overwrite or regrow it
        if (g > 0) {
            std::swap(e->chains, e->chains_alt);
            std::swap(e->info, e->info_alt);
        }
        if (copy_pending[buf]) CVL_CUDA(cudaStreamWaitEvent(e->stream, e->copied[buf], 0));
        std::vector<int32_t> mo(M + 1, 0);
        for (int k = 0; k < M; ++k) mo[k + 1] = mo[k] + counts[order[m0 + k]];
        const int n = mo[M];
        int rc = e->alloc(e->map_off, sizeof(int) * mo.size());
        if (rc != CVL_OK) return cleanup(rc);
        if (cudaMemcpyAsync(e->map_off.p, mo.data(), sizeof(int) * mo.size(), cudaMemcpyHostToDevice, e->stream) !=
                cudaSuccess ||
            cudaStreamWaitEvent(e->stream, e->uploaded[buf], 0) != cudaSuccess)
            return cleanup(fail(CVL_ECUDA, "map offsets upload failed"));
        RunOut ro;
        rc = run_pipeline(e, (const double *)ebuf[buf]->p, n, edge_data_sz, (const int *)e->map_off.p, mo, md, cpl, 0,
                          false, ro);
        if (rc != CVL_OK) return cleanup(rc);
        if (cudaEventRecord(e->consumed[buf], e->stream) != cudaSuccess)
            return cleanup(fail(CVL_ECUDA, "event record failed"));
        e->collect_marks();
        device_ms += e->last_device_ms;
        if (cudaEventRecord(e->computed[buf], e->stream) != cudaSuccess ||
            cudaStreamWaitEvent(e->copy_stream, e->computed[buf], 0) != cudaSuccess)
            return cleanup(fail(CVL_ECUDA, "event record/wait failed"));
        for (int k = 0; k < M; ++k) {
            const unsigned long long c0 = ro.cv_off[k], C = ro.cv_off[k + 1] - c0;
            cvl_result *r = new cvl_result();
            res[order[m0 + k]] = r;
            r->pool = e->pinned;
            r->chains_p = e->pinned->get(sizeof(unsigned) * (C ? C : 1) * W);
            r->info_p = e->pinned->get(sizeof(double) * (C ? C : 1) * 10);
            if (!r->chains_p || !r->info_p)
                return cleanup(fail(CVL_ENOMEM, "page-locked result buffers could not be allocated"));
            if (C) {  // by SM threads beside the next group's compute; the last group's alone
                const bool alone = g == G - 1;
                cudaError_t ce = copy_result_to_host(r->chains_p, (const unsigned *)e->chains.p + c0 * W,
                                                     sizeof(unsigned) * C * W, e->copy_stream, alone);
                if (ce == cudaSuccess)
                    ce = copy_result_to_host(r->info_p, (const double *)e->info.p + c0 * 10,
                                             sizeof(double) * C * 10, e->copy_stream, alone);
                if (ce != cudaSuccess) return cleanup(fail(CVL_ECUDA, std::string("result copy: ") + cudaGetErrorString(ce)));
            }
            const MapStats &st = ro.stats[k];
            cvl_result_view &v = r->v;
            v.num_curvelets = (uint32_t)C;
            v.chain_width = (uint32_t)W;
            v.chains = (const uint32_t *)r->chains_p;
            v.info = (const double *)r->info_p;
            v.valid_pairs = st.valid_pairs;
            v.total_neighbor_pairs = (int64_t)st.pairs;
            v.max_num_of_neighbors = st.max_deg;
            v.truncated_anchors = st.truncated;
            v.num_edges = (uint32_t)counts[order[m0 + k]];
            v.flags = v.truncated_anchors ? CVL_FLAG_TRUNCATED : 0u;
        }
        if (cudaEventRecord(e->copied[buf], e->copy_stream) != cudaSuccess)
            return cleanup(fail(CVL_ECUDA, "event record failed"));
        copy_pending[buf] = true;
    }
    CVL_CUDA(cudaStreamSynchronize(e->copy_stream));
    for (int32_t m = 0; m < num_maps; ++m) {
        res[m]->v.device_ms = device_ms;
        out[m] = res[m];
    }
    e->last_device_ms = device_ms;
    return CVL_OK;
}


// =============================================================================
// Edges already in device memory
// =============================================================================
extern "C" int cvl_run_device(cvl_engine *e, const double *d_edges, int32_t num_edges, int32_t edge_data_sz,
                              const cvl_params *p, void *ready_event, cvl_result **out) {
    if (!e) return fail(CVL_EINVAL, "engine is NULL");
    if (out) *out = nullptr;
    CVL_TRY(check_edges_args(d_edges, num_edges, edge_data_sz));
    CVL_CUDA(cudaSetDevice(e->device));
    cudaPointerAttributes pa{};
    if (cudaPointerGetAttributes(&pa, d_edges) != cudaSuccess) {
        cudaGetLastError();
        return fail(CVL_EINVAL, "d_edges is not a CUDA pointer");
    }
    if ((pa.type != cudaMemoryTypeDevice && pa.type != cudaMemoryTypeManaged) || pa.device != e->device)
        return fail(CVL_EINVAL, "d_edges must be device or managed memory on the engine's device");
    if (ready_event) CVL_CUDA(cudaStreamWaitEvent(e->stream, (cudaEvent_t)ready_event, 0));
    Model md;
    int cpl = 2;
    CVL_TRY(make_model(e, p, p ? p->nrad : 0.0, 3u, p ? p->max_candidates : 0u, md, cpl));
    std::vector<int32_t> mo = {0, num_edges};
    CVL_TRY(e->alloc(e->map_off, sizeof(int) * mo.size()));
    CVL_CUDA(cudaMemcpyAsync(e->map_off.p, mo.data(), sizeof(int) * mo.size(), cudaMemcpyHostToDevice, e->stream));
    RunOut ro;
    CVL_TRY(run_pipeline(e, d_edges, num_edges, edge_data_sz, (const int *)e->map_off.p, mo, md, cpl, 0, false, ro));
    e->collect_marks();
    if (!e->dev_done) CVL_CUDA(cudaEventCreateWithFlags(&e->dev_done, cudaEventDisableTiming));
    CVL_CUDA(cudaEventRecord(e->dev_done, e->stream));
    e->dev_curvelets = ro.total_curvelets;
    e->dev_width = md.gms + 1;
    e->dev_generation = e->generation;
    if (!out) return CVL_OK;
    cvl_result *r = new cvl_result();
    const int rc = fill_view_from_run(e, ro, num_edges, md.gms + 1, r);
    if (rc != CVL_OK) {
        delete r;
        return rc;
    }
    *out = r;
    return CVL_OK;
}

extern "C" int cvl_engine_device_results(cvl_engine *e, cvl_device_results *out) {
    if (!e || !out) return fail(CVL_EINVAL, "engine/out is NULL");
    if (e->dev_generation != e->generation)
        return fail(CVL_EINVAL, "no device-resident results: the engine's last run was not cvl_run_device");
    out->num_curvelets = (uint32_t)e->dev_curvelets;
    out->chain_width = (uint32_t)e->dev_width;
    out->chains = (const uint32_t *)e->chains.p;
    out->info = (const double *)e->info.p;
    out->done_event = (void *)e->dev_done;
    return CVL_OK;
}

void cvl_engine_growth(const cvl_engine *e, uint64_t *dev_grows, double *dev_ms, uint64_t *host_grows,
                       double *host_ms) {
    *dev_grows = e->dev_grows.load();
    *dev_ms = (double)e->dev_grow_ns.load() * 1e-6;
    *host_grows = e->pinned->grows();
    *host_ms = e->pinned->grow_ms();
}
