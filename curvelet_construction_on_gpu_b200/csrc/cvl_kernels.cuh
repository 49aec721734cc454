// cvl_kernels.cuh -- sm_100a kernels of the curvelet path, part 1: shared
// definitions, (a) spatial-hash binning and (b) the neighbour search.
//
// Pipeline over a ragged batch of M edge maps (M = 1 for the plain form):
//   (a) k_bin_keys / k_bin_scatter  counting sort of the edges into S x S
//       pixel-cell blocks (S a power of two >= the window half width + 1) of a
//       spatial hash; SoA FP64 edge arrays in bucket order; per-edge
//       sin/cos(theta +- dt) computed once;
//   (b) k_nb<COUNT> / k_nb<FILL>     warp per anchor: the window's bucket
//       ranges are loaded by all lanes at once, then the candidates are
//       enumerated 32 at a time with the reference's predicate (7x7 pixel
//       window, not self, not d^2 > r^2; preprocess.hpp:129-167). COUNT writes
//       the capped degree; FILL stages the candidates in shared memory, keeps
//       the first max_candidates in window-scan order when there are more
//       (:165-167), rank-sorts them by (d^2, scan position) (:172-176) and
//       writes the CSR row, each pair's direction-run class
//       (cpu_curvelet.hpp:454-462) and the anchor's sin/cos(T2 + delta_t2_j).
//   (c) + (d) + (e) are in cvl_path.cuh.
//
// Every FP64 expression keeps the reference's operand order; the library is
// compiled with -fmad=false so no multiply-add is contracted, and uses IEEE
// division and square root. sin/cos/atan2/fmod are CUDA's.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cvl {

constexpr unsigned FULL = 0xffffffffu;
constexpr int QMAX = 32;     // orientation samples supported (grid Q)
constexpr int GMS_MAX = 16;  // group_max_sz supported
constexpr int MAPS_SMEM = 256;  // per-block map statistics kept in shared memory up to this many maps
constexpr double CVL_PI = 3.14159265358979323846;  // curvelet_utils.hpp:10

// Error bits raised by kernels (checked by the host after a run).
constexpr unsigned ERR_NONFINITE = 1u;   // non-finite or out-of-range coordinate
constexpr unsigned ERR_CAPACITY = 2u;    // a device capacity was exceeded
constexpr unsigned ERR_INTERNAL = 4u;    // an internal invariant failed (bounds check)
constexpr unsigned ERR_ARENA = 8u;       // the record arena was too small (the host resizes and reruns)

// T is the path's scalar type: double (run_curvelet<double>) or float (the
// reference's --float mode, run_curvelet<float>, main.cpp:110). In float mode
// the reference's expressions keep their C++ types: a double literal in an
// expression (2.0, 1.0) promotes it to double and the result rounds to float
// on assignment; everything else is float arithmetic. The kernels restate
// each expression with those types (marked "float mode" where they differ from
// the all-T form).
template <typename T>
struct ModelT {
    T nrad, rad_sqr;        // neighbour radius and its square (preprocess.hpp:221)
    T dx, dx2, four_dx_dx;  // _dx, _dx*_dx, 4*_dx*_dx (cpu_curvelet.hpp:654,682)
    T dt, sx, st, max_k;    // dt in radians (main.cpp:24)
    int P, Q, cells;             // bundle grid (cpu_curvelet.hpp:73-74)
    int gms;                     // group_max_sz
    int max_cand;                // max_candidates
    int w;                       // pixel-window half width (3, main.cpp:48)
    int sbits;                   // hash block edge S = 1 << sbits pixel cells
    unsigned hash_mask;          // table size - 1
    int shared_quot;             // FP64 transport: the k_dx quotients on one reciprocal
                                 // (QUOT_SHARED) unless a run's operands fail certify_*
};

// Operands whose ranges give every nonzero e1 and k_dx numerator of the FP64
// transport a magnitude in [2^-500, 2^501), the range in which the transport's
// shared-reciprocal quotients round correctly (cvl_path.cuh). With x, y and the
// parameters dx, sx in {0} or [2^-40, 2^40] in magnitude (coordinates are below
// 1e9 < 2^30 in any case), and the anchor trig values sin/cos(T2t_j) in {0} or
// [2^-100, 1]: every value is a multiple of its lowest bit 2^(exponent - 52), sums
// keep the smallest of their operands' lowest bits, and products multiply them,
// so e1 = (((DX^2 - (2 d) tt) + DY^2) - dx^2) + d^2 is 0 or at least 2^-336 (DX
// from 2^-92, tt = sin DX - cos DY from 2^-244, 2 d from 2^-92) and at most 2^94,
// and the numerators (2 tt - 2 d) -+ 2 dx are 0 or in [2^-243, 2^48]. A run with
// an operand outside these ranges sets its flag, and its transport divides.
template <typename T>
__device__ __forceinline__ bool certify_coord(T v) {
    const T a = fabs(v);
    return a == T(0) || (a >= T(0x1p-40) && a <= T(0x1p40));
}
template <typename T>
__device__ __forceinline__ bool certify_trig(T v) {
    const T a = fabs(v);
    return a == T(0) || a >= T(0x1p-100);
}
using Model = ModelT<double>;

// SoA copy of the edges in hash-bucket order ("internal" index space).
template <typename T>
struct BinnedT {
    T *x, *y, *th;         // position, orientation
    T *sp, *cp, *sm, *cm;  // sin/cos(theta + dt), sin/cos(theta - dt)
    int2 *cell;                 // pixel cell (lrint(x), lrint(y))
    int *orig;                  // global input index
    int *map;                   // map of the edge
};

// The sizes of a run that a captured graph replays (one graph per size bucket
// serves every run within the bucket): the kernels launched for the bucket's
// capacity read the run's own sizes from device memory at their start. nullptr
// outside graphs, where the launch's arguments are the run's sizes.
struct RunDims {
    int N;  // edges of the run (all maps)
    int M;  // maps
};

// One chunk of a graph run's bundle/growth stages, computed on the device
// (k_chunk_dims): its anchors [a_begin, a_end) and their pairs [p_begin, p_end).
struct ChunkDims {
    int a_begin, a_end;
    unsigned long long p_begin, p_end;
};

struct MapStats {
    unsigned long long pairs;  // total_neighbor_pairs
    unsigned max_deg;          // max_num_of_neighbors
    unsigned truncated;        // anchors that reached max_candidates
    unsigned valid_pairs;      // pairs with a valid bundle
    unsigned close_pairs;      // pairs that keep the default bundle (no transport)
};

// Per-block map statistics: accumulated with shared-memory atomics and added to
// the global MapStats once per block (global atomics per anchor on the same few
// addresses would serialise in L2).
struct BlockStats {
    unsigned long long pairs[MAPS_SMEM];
    unsigned max_deg[MAPS_SMEM];
    unsigned truncated[MAPS_SMEM];
    unsigned valid[MAPS_SMEM];
    unsigned close[MAPS_SMEM];
};

__device__ __forceinline__ void block_stats_init(BlockStats &bs, int M) {
    for (int m = threadIdx.x; m < M && m < MAPS_SMEM; m += blockDim.x) {
        bs.pairs[m] = 0;
        bs.max_deg[m] = 0;
        bs.truncated[m] = 0;
        bs.valid[m] = 0;
        bs.close[m] = 0;
    }
}

__device__ __forceinline__ void stats_add(BlockStats &bs, MapStats *gs, int M, int m, unsigned pairs, unsigned deg,
                                          unsigned trunc, unsigned valid, unsigned close = 0u) {
    if (M <= MAPS_SMEM) {
        if (pairs) atomicAdd(&bs.pairs[m], (unsigned long long)pairs);
        if (deg) atomicMax(&bs.max_deg[m], deg);
        if (trunc) atomicAdd(&bs.truncated[m], trunc);
        if (valid) atomicAdd(&bs.valid[m], valid);
        if (close) atomicAdd(&bs.close[m], close);
    } else {
        if (pairs) atomicAdd(&gs[m].pairs, (unsigned long long)pairs);
        if (deg) atomicMax(&gs[m].max_deg, deg);
        if (trunc) atomicAdd(&gs[m].truncated, trunc);
        if (valid) atomicAdd(&gs[m].valid_pairs, valid);
        if (close) atomicAdd(&gs[m].close_pairs, close);
    }
}

__device__ __forceinline__ void block_stats_flush(BlockStats &bs, MapStats *gs, int M) {
    if (M > MAPS_SMEM) return;
    for (int m = threadIdx.x; m < M; m += blockDim.x) {
        if (bs.pairs[m]) atomicAdd(&gs[m].pairs, bs.pairs[m]);
        if (bs.max_deg[m]) atomicMax(&gs[m].max_deg, bs.max_deg[m]);
        if (bs.truncated[m]) atomicAdd(&gs[m].truncated, bs.truncated[m]);
        if (bs.valid[m]) atomicAdd(&gs[m].valid_pairs, bs.valid[m]);
        if (bs.close[m]) atomicAdd(&gs[m].close_pairs, bs.close[m]);
    }
}

// Spatial hash of a (map, block) key: XOR of products with large primes
// (Teschner et al., "Optimized Spatial Hashing for Collision Detection of
// Deformable Objects", VMV 2003) followed by a 32-bit avalanche mix.
__device__ __forceinline__ unsigned cell_hash(int m, int bx, int by) {
    unsigned h = ((unsigned)bx * 73856093u) ^ ((unsigned)by * 19349663u) ^ ((unsigned)m * 83492791u);
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h;
}

// sq_dist (curvelet_utils.hpp:13-17)
template <typename T>
__device__ __forceinline__ T sq_dist(T x1, T y1, T x2, T y2) {
    return (x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2);
}

// Out-of-line copies of the libm calls: one copy of each in a kernel instead of
// one per call site keeps the kernels' code within the instruction cache.
__device__ __noinline__ double cvl_sin(double x) { return sin(x); }
__device__ __noinline__ double cvl_cos(double x) { return cos(x); }
__device__ __noinline__ double cvl_atan2(double y, double x) { return atan2(y, x); }
__device__ __noinline__ double cvl_fmod(double x, double y) { return fmod(x, y); }
// the float functions of float mode (std::sin(float) etc.)
__device__ __noinline__ float cvl_sin(float x) { return sinf(x); }
__device__ __noinline__ float cvl_cos(float x) { return cosf(x); }
__device__ __noinline__ float cvl_atan2(float y, float x) { return atan2f(y, x); }
__device__ __noinline__ float cvl_fmod(float x, float y) { return fmodf(x, y); }

// T(2) * T(M_PI), To2Pi's bound (curvelet_utils.hpp:29)
template <typename T>
__device__ __forceinline__ T two_pi() {
    return T(2) * T(CVL_PI);
}

// lrint (preprocess.hpp:85-86): round half to even, of the scalar type's value
__device__ __forceinline__ int lrint_dev(double x) { return __double2int_rn(x); }
__device__ __forceinline__ int lrint_dev(float x) { return __float2int_rn(x); }

// delta = s * (k - (n - 1.0) / 2.0) with k, n small integers: evaluated in double
// (the 1.0 and 2.0 are double literals) and rounded to T (cpu_curvelet.hpp:697-698)
template <typename T>
__device__ __forceinline__ T grid_offset(T s, int k, int n) {
    return (T)((double)s * ((double)k - ((double)n - 1.0) / 2.0));
}

// fmod(x, 2pi) with its IEEE fast case inline: for |x| < |y|, fmod(x, y) == x exactly.
template <typename T>
__device__ __forceinline__ T fmod_2pi(T x) {
    return (fabs(x) < two_pi<T>()) ? x : cvl_fmod(x, two_pi<T>());
}

// To2Pi (curvelet_utils.hpp:25-46)
template <typename T>
__device__ __forceinline__ T to_2pi(T angle) {
    T a;
    if (angle >= two_pi<T>())
        a = fmod_2pi(angle);
    else if (angle < 0)
        a = (two_pi<T>() + fmod_2pi(angle));
    else
        a = angle;
    if (!(a >= 0 && a < two_pi<T>())) a = 0;
    return a;
}

__device__ __forceinline__ int map_of(const int *map_off, int M, int e) {
    int lo = 0, hi = M;  // map_off[lo] <= e < map_off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (map_off[mid] <= e) lo = mid; else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// (a) spatial-hash binning
// ---------------------------------------------------------------------------
template <typename T>
__global__ void k_bin_keys(const T *__restrict__ edges, int sz, int N, const int *__restrict__ map_off, int M,
                           ModelT<T> md, unsigned *__restrict__ ehash, unsigned *__restrict__ bcount,
                           unsigned *__restrict__ err, unsigned *__restrict__ uncertified,
                           const RunDims *__restrict__ dims) {
    if (dims) {
        N = dims->N;
        M = dims->M;
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N; e += gridDim.x * blockDim.x) {
        const T x = edges[(size_t)e * sz + 0];
        const T y = edges[(size_t)e * sz + 1];
        const T th = edges[(size_t)e * sz + 2];
        if (!isfinite(x) || !isfinite(y) || !isfinite(th) || fabs(x) >= T(1.0e9) || fabs(y) >= T(1.0e9)) {
            atomicOr(err, ERR_NONFINITE);
            ehash[e] = 0;
            atomicAdd(&bcount[0], 1u);
            continue;
        }
        if (uncertified && !(certify_coord(x) && certify_coord(y))) atomicOr(uncertified, 1u);
        const int m = map_of(map_off, M, e);
        const int cx = lrint_dev(x);  // lrint, round half to even (preprocess.hpp:85-86)
        const int cy = lrint_dev(y);
        const unsigned h = cell_hash(m, cx >> md.sbits, cy >> md.sbits) & md.hash_mask;
        ehash[e] = h;
        atomicAdd(&bcount[h], 1u);
    }
}

template <typename T>
__global__ void k_bin_scatter(const T *__restrict__ edges, int sz, int N, const int *__restrict__ map_off,
                              int M, ModelT<T> md, const unsigned *__restrict__ ehash,
                              const unsigned *__restrict__ bstart, unsigned *__restrict__ bfill, BinnedT<T> B,
                              int *__restrict__ pos_of, const RunDims *__restrict__ dims) {
    if (dims) {
        N = dims->N;
        M = dims->M;
    }
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N; e += gridDim.x * blockDim.x) {
        const unsigned h = ehash[e];
        const unsigned pos = bstart[h] + atomicAdd(&bfill[h], 1u);
        const T x = edges[(size_t)e * sz + 0];
        const T y = edges[(size_t)e * sz + 1];
        const T th = edges[(size_t)e * sz + 2];
        B.x[pos] = x;
        B.y[pos] = y;
        B.th[pos] = th;
        // T0 +- dt and their sin/cos (cpu_curvelet.hpp:655-656, 730-733), once per edge
        const T t_p = th + md.dt;
        const T t_m = th - md.dt;
        B.sp[pos] = sin(t_p);
        B.cp[pos] = cos(t_p);
        B.sm[pos] = sin(t_m);
        B.cm[pos] = cos(t_m);
        B.cell[pos] = make_int2(lrint_dev(x), lrint_dev(y));
        B.orig[pos] = e;
        B.map[pos] = map_of(map_off, M, e);
        pos_of[e] = (int)pos;
    }
}

// ---------------------------------------------------------------------------
// (b) neighbour search: warp per anchor
// ---------------------------------------------------------------------------
// Candidate key for ties and truncation: window-scan position (py outer, px
// inner, preprocess.hpp:141-142) then global edge index (within a cell).
__device__ __forceinline__ unsigned long long scan_key(int2 c, int cx, int cy, int w, int e) {
    const int side = 2 * w + 1;
    const unsigned r = (unsigned)((c.y - cy + w) * side + (c.x - cx + w));
    return ((unsigned long long)r << 32) | (unsigned)e;
}

template <typename T>
struct NbrSmemT {  // per-warp candidate staging, capacity max_cand (d2 slots are 8 bytes in both modes)
    T *d2;
    unsigned long long *key;
    int *idx;
};

enum { NB_COUNT = 0, NB_FILL = 1 };

// Per-warp candidate staging bytes: d2 (8) + key (8) + idx (4) per candidate,
// rounded up to 16 so every warp's arrays start 16-byte aligned.
__host__ __device__ inline size_t nbr_smem_per_warp(int max_cand) {
    return ((size_t)max_cand * 20 + 15) & ~(size_t)15;
}

// Visits every edge of the anchor's map in the hash blocks covering its window
// and calls f(ok, j, d2, key) warp-uniformly, 32 entries at a time; ok is the
// reference predicate. The window's bucket ranges (up to 32 per round) are
// loaded by the lanes at once; entries are enumerated over their prefix sums.
// WANT_KEY: compute the scan key (a counting pass needs none).
template <bool WANT_KEY = true, typename T, typename F>
__device__ __forceinline__ void for_window_candidates(const ModelT<T> &md, const BinnedT<T> &B, const unsigned *bstart,
                                                      int i, int m, int2 ac, T ax, T ay, int lane, F &&f) {
    const int bx0 = (ac.x - md.w) >> md.sbits, bx1 = (ac.x + md.w) >> md.sbits;
    const int by0 = (ac.y - md.w) >> md.sbits, by1 = (ac.y + md.w) >> md.sbits;
    const int nbx = bx1 - bx0 + 1;
    const int nb = nbx * (by1 - by0 + 1);
    for (int t0 = 0; t0 < nb; t0 += 32) {
        const int t = t0 + lane;
        int bx = 0, by = 0;
        unsigned s = 0, c = 0;
        if (t < nb) {
            by = by0 + t / nbx;
            bx = bx0 + t - (t / nbx) * nbx;
            const unsigned h = cell_hash(m, bx, by) & md.hash_mask;
            s = bstart[h];
            c = bstart[h + 1] - s;
        }
        // inclusive prefix of the bucket sizes
        unsigned incl = c;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned o = __shfl_up_sync(FULL, incl, d);
            if (lane >= d) incl += o;
        }
        const unsigned total = __shfl_sync(FULL, incl, 31);
        for (unsigned e0 = 0; e0 < total; e0 += 32) {
            const unsigned e = e0 + lane;
            // bucket of entry e: the first lane whose inclusive prefix exceeds e
            int lo = 0;
#pragma unroll
            for (int step = 16; step >= 1; step >>= 1) {
                const unsigned v = __shfl_sync(FULL, incl, lo + step - 1);
                if (v <= e) lo += step;
            }
            const unsigned pre = __shfl_sync(FULL, incl, lo) - __shfl_sync(FULL, c, lo);
            const unsigned sb = __shfl_sync(FULL, s, lo);
            const int vbx = __shfl_sync(FULL, bx, lo), vby = __shfl_sync(FULL, by, lo);
            bool ok = false;
            T d2 = 0;
            unsigned long long key = 0;
            const int j = (int)(sb + (e - pre));
            if (e < total && j != i) {
                const int2 cc = B.cell[j];
                // the entry's own block must be the visited one (a bucket can hold
                // several blocks, and two window blocks can share a bucket)
                if (B.map[j] == m && (cc.x >> md.sbits) == vbx && (cc.y >> md.sbits) == vby &&
                    abs(cc.x - ac.x) <= md.w && abs(cc.y - ac.y) <= md.w) {
                    d2 = sq_dist(ax, ay, B.x[j], B.y[j]);  // sq_dist(te, ne), preprocess.hpp:160
                    ok = !(d2 > md.rad_sqr);               // preprocess.hpp:161-163
                    if (WANT_KEY) key = scan_key(cc, ac.x, ac.y, md.w, B.orig[j]);
                }
            }
            f(ok, j, d2, key);
        }
    }
}

// Truncation (preprocess.hpp:165-167): keep the first max_cand candidates in
// window-scan order. Walks the window pixel cell by pixel cell; inside the cell
// where the cap is crossed keeps the lowest edge indices. Returns the count kept.
template <typename T>
__device__ __noinline__ unsigned gather_truncated(const ModelT<T> &md, const BinnedT<T> &B, const unsigned *bstart,
                                                  int i, int m, int2 ac, T ax, T ay, int lane, NbrSmemT<T> S,
                                                  unsigned *err) {
    const unsigned lt_mask = (1u << lane) - 1u;
    const int side = 2 * md.w + 1;
    unsigned n = 0;
    for (int r = 0; r < side * side && n < (unsigned)md.max_cand; ++r) {
        const int px = ac.x - md.w + r % side;
        const int py = ac.y - md.w + r / side;
        const unsigned h = cell_hash(m, px >> md.sbits, py >> md.sbits) & md.hash_mask;
        const int b0 = (int)bstart[h], b1 = (int)bstart[h + 1];
        // count this cell's candidates
        unsigned c = 0;
        for (int base = b0; base < b1; base += 32) {
            const int j = base + lane;
            bool ok = false;
            if (j < b1 && j != i) {
                const int2 cc = B.cell[j];
                ok = B.map[j] == m && cc.x == px && cc.y == py && !(sq_dist(ax, ay, B.x[j], B.y[j]) > md.rad_sqr);
            }
            c += __popc(__ballot_sync(FULL, ok));
        }
        const unsigned need = (unsigned)md.max_cand - n;
        for (int base = b0; base < b1; base += 32) {
            const int j = base + lane;
            bool ok = false;
            T d2 = 0;
            int oj = 0;
            if (j < b1 && j != i) {
                const int2 cc = B.cell[j];
                if (B.map[j] == m && cc.x == px && cc.y == py) {
                    d2 = sq_dist(ax, ay, B.x[j], B.y[j]);
                    ok = !(d2 > md.rad_sqr);
                    oj = B.orig[j];
                }
            }
            if (ok && c > need) {
                // rank by edge index among this cell's candidates
                unsigned rk = 0;
                for (int k = b0; k < b1; ++k) {
                    if (k == i) continue;
                    const int2 ck = B.cell[k];
                    if (B.map[k] == m && ck.x == px && ck.y == py && B.orig[k] < oj &&
                        !(sq_dist(ax, ay, B.x[k], B.y[k]) > md.rad_sqr))
                        ++rk;
                }
                ok = rk < need;
            }
            const unsigned bal = __ballot_sync(FULL, ok);
            if (ok) {
                const unsigned p = n + __popc(bal & lt_mask);
                if (p < (unsigned)md.max_cand) {
                    S.d2[p] = d2;
                    S.key[p] = ((unsigned long long)r << 32) | (unsigned)oj;
                    S.idx[p] = j;
                } else {
                    atomicOr(err, ERR_INTERNAL);
                }
            }
            n += __popc(bal);
        }
    }
    return n > (unsigned)md.max_cand ? (unsigned)md.max_cand : n;
}

template <typename T>
struct NbArgsT {
    ModelT<T> md;
    BinnedT<T> B;
    const unsigned *bstart;
    int N, M;
    unsigned *ncand;                     // COUNT: candidates in window (before the cap)
    MapStats *stats;
    const unsigned long long *pair_off;  // FILL: [N+1] internal order
    int *csr_ids;                        // FILL: internal neighbour indices, by pair
    T *csr_d2;                           // FILL (optional): squared distances
    unsigned char *pcls;                 // FILL (optional): run | close << 2 per pair
    int *pair_anchor;                    // FILL (optional): internal anchor of each pair
    T *atrig;                            // FILL (optional): [N][2Q + 2] sin/cos(T2 + delta_t2_j), cos/sin(T2)
    unsigned *err;
    unsigned *uncertified;               // FILL (optional): set when a trig value fails certify_trig
    const RunDims *dims;                 // graph runs: N and M from device memory
    unsigned long long pair_cap;         // graph runs: pairs the CSR buffers hold (0: sized to the run)
};

// COUNT: ncand[i], per-map pairs / max degree / truncated anchors.
// FILL:  the CSR row of anchor i at pair_off[i] sorted by (d2, scan key), and
//        optionally the pair classes, pair->anchor map and anchor trig table.
// The direction class of a neighbour (:454-462): the sign of
// dot(angle_from_pt_to_pt(te, le), te's orientation) (curvelet_utils.hpp:58-69),
// 0 ahead, 1 behind, 2 exactly perpendicular. That dot is the cosine of the angle
// between the neighbour's direction and the orientation, computed through atan2,
// To2Pi, cos and sin with an error of a few ulps: below 5e-15 in double and 2e-6 in
// float. v = dx cos(theta) + dy sin(theta) is that cosine times the vector's length,
// which is at most |dx| + |dy|, and is computed here to about 1e-15 of |dx| + |dy|.
// So when |v| exceeds 1e-12 (double) or 1e-4 (float) of |dx| + |dy|, the sign of v
// is the sign of the reference's dot, and the three transcendental calls are
// skipped; nearer to perpendicular, the reference's own expression decides.
template <typename T>
__device__ __forceinline__ unsigned direction_class(T ax, T ay, T lx, T ly, T cosT2, T sinT2) {
    const double dx = (double)lx - (double)ax, dy = (double)ly - (double)ay;
    const double v = dx * (double)cosT2 + dy * (double)sinT2;
    const double margin = (sizeof(T) == sizeof(double) ? 1e-12 : 1e-4) * (fabs(dx) + fabs(dy));
    if (v > margin) return 0u;
    if (v < -margin) return 1u;
    const T dir = to_2pi(cvl_atan2(ly - ay, lx - ax));      // angle_from_pt_to_pt(te, le)
    const T d = cvl_cos(dir) * cosT2 + cvl_sin(dir) * sinT2;  // dot(dir, te_orient)
    return (d > 0) ? 0u : ((d < 0) ? 1u : 2u);
}

// The parameter is a __grid_constant__: gather_truncated (not inlined) takes
// references to its model and binned arrays, and a plain by-value parameter would
// be copied to every thread's local stack for that (~300 bytes per thread, stored
// in the prologue of every launch whether or not any anchor is truncated).
template <typename T, int MODE>
// Register budgets: both passes are latency-bound gathers, which gain more from
// resident warps than their few spills cost. COUNT 8 blocks per SM (32 registers:
// 21.8 -> 18.2 ms on the 64-map batch); FILL 6 (40 registers: 48.1 -> 42.1 ms against
// 64 registers, 42.8 ms at 48; without a bound it took more and ran 78% slower).
__global__ void __launch_bounds__(256, MODE == NB_COUNT ? 8 : 6) k_nb(const __grid_constant__ NbArgsT<T> a) {
    extern __shared__ __align__(16) unsigned char nb_smem[];
    __shared__ BlockStats bstats;
    const ModelT<T> &md = a.md;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int N = a.dims ? a.dims->N : a.N;
    const int M = a.dims ? a.dims->M : a.M;
    if (MODE == NB_COUNT) {
        block_stats_init(bstats, M);
        __syncthreads();
    }
    NbrSmemT<T> S;
    {
        unsigned char *p = nb_smem + (size_t)wib * nbr_smem_per_warp(md.max_cand);
        S.d2 = (T *)p;
        S.key = (unsigned long long *)(p + (size_t)md.max_cand * 8);
        S.idx = (int *)(p + (size_t)md.max_cand * 16);
    }
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int i = blockIdx.x * wpb + wib; i < N; i += gridDim.x * wpb) {
        const int m = a.B.map[i];
        const int2 ac = a.B.cell[i];
        const T ax = a.B.x[i], ay = a.B.y[i];
        if (MODE == NB_COUNT) {
            unsigned cnt = 0;
            for_window_candidates<false>(md, a.B, a.bstart, i, m, ac, ax, ay, lane,
                                         [&](bool ok, int, T, unsigned long long) {
                                      cnt += __popc(__ballot_sync(FULL, ok));
                                  });
            if (lane == 0) {
                a.ncand[i] = cnt;
                const unsigned deg = cnt < (unsigned)md.max_cand ? cnt : (unsigned)md.max_cand;
                stats_add(bstats, a.stats, M, m, deg, deg, deg >= (unsigned)md.max_cand ? 1u : 0u, 0u);
            }
            continue;
        }
        const unsigned total = a.ncand[i];
        unsigned n = 0;
        if (total <= (unsigned)md.max_cand) {
            for_window_candidates(md, a.B, a.bstart, i, m, ac, ax, ay, lane,
                                  [&](bool ok, int j, T d2, unsigned long long key) {
                                      const unsigned bal = __ballot_sync(FULL, ok);
                                      if (ok) {
                                          const unsigned p = n + __popc(bal & lt_mask);
                                          if (p < (unsigned)md.max_cand) {
                                              S.d2[p] = d2;
                                              S.key[p] = key;
                                              S.idx[p] = j;
                                          } else {
                                              atomicOr(a.err, ERR_INTERNAL);
                                          }
                                      }
                                      n += __popc(bal);
                                  });
        } else {
            n = gather_truncated(md, a.B, a.bstart, i, m, ac, ax, ay, lane, S, a.err);
        }
        __syncwarp();
        const unsigned long long off = a.pair_off[i];
        if (a.pair_off[i + 1] - off != n) {  // the two passes must agree
            if (lane == 0) atomicOr(a.err, ERR_INTERNAL);
            __syncwarp();
            continue;
        }
        if (a.pair_cap && a.pair_off[i + 1] > a.pair_cap) {  // a graph run beyond its pair buffers
            if (lane == 0) atomicOr(a.err, ERR_CAPACITY);
            __syncwarp();
            continue;
        }
        // the anchor's trig row [2Q + 2]: sin(T2 + delta_t2_j), cos(T2 + delta_t2_j)
        // for j < Q (:702-705), then cos(T2), sin(T2) (:690 and the dot product). One
        // sincos per lane: lane j takes T2t_j, lane Q (mod 32) T2 itself, whose values
        // go to every lane by shuffle. sincos gives the values of sin and cos
        // (tests/probes/sincos_identity.cu compares them on the device, double and float).
        const T T2 = a.B.th[i];
        T cosT2 = T(0), sinT2 = T(0);
        if (a.pcls || a.atrig) {
            T sT2 = T(0), cT2 = T(0);
            T *row = a.atrig ? a.atrig + (size_t)i * (2 * md.Q + 2) : nullptr;
            for (int j = lane; j <= md.Q; j += 32) {
                if (j < md.Q && !row) continue;
                // T2t = T2 + delta_t2 (:698-702)
                const T t = (j < md.Q) ? T(T2 + grid_offset(md.st, j, md.Q)) : T2;
                T sv, cv;
                sincos(t, &sv, &cv);  // inline (measured 2% faster than the out-of-line call)
                if (j == md.Q) {
                    sT2 = sv;
                    cT2 = cv;
                    if (row) {
                        row[2 * md.Q] = cv;
                        row[2 * md.Q + 1] = sv;
                    }
                } else {
                    row[j] = sv;
                    row[md.Q + j] = cv;
                    if (a.uncertified && !(certify_trig(sv) && certify_trig(cv))) atomicOr(a.uncertified, 1u);
                }
            }
            cosT2 = __shfl_sync(FULL, cT2, md.Q & 31);
            sinT2 = __shfl_sync(FULL, sT2, md.Q & 31);
        }
        // rank sort by (d2, scan key) -- std::sort by distance, preprocess.hpp:172-176
        for (unsigned t = lane; t < n; t += 32) {
            const T dt_ = S.d2[t];
            const unsigned long long kt = S.key[t];
            unsigned rk = 0;
            for (unsigned u = 0; u < n; ++u) {
                const T du = S.d2[u];
                rk += (du < dt_) || (du == dt_ && S.key[u] < kt);
            }
            const int nn = S.idx[t];
            a.csr_ids[off + rk] = nn;
            if (a.csr_d2) a.csr_d2[off + rk] = dt_;
            if (a.pair_anchor) a.pair_anchor[off + rk] = i;
            if (a.pcls) {
                // direction filter (:454-462) and close pair (:682)
                const T lx = a.B.x[nn], ly = a.B.y[nn];
                const unsigned run = direction_class(ax, ay, lx, ly, cosT2, sinT2);
                const T DX = ax - lx, DY = ay - ly;
                const bool close = (DX * DX + DY * DY < md.four_dx_dx);
                a.pcls[off + rk] = (unsigned char)(run | (close ? 4u : 0u));
            }
        }
        __syncwarp();
    }
    if (MODE == NB_COUNT) {
        __syncthreads();
        block_stats_flush(bstats, a.stats, M);
    }
}

// deg[i] for i < N; with dims (a graph run launched for its bucket's N), deg of the
// run's anchors and 0 for the rest of the N entries, so that the scan over all N
// gives the run's pair offsets and, at [N], its total.
__global__ void k_deg_from_ncand(int N, int max_cand, const unsigned *__restrict__ ncand, unsigned *__restrict__ deg,
                                 const RunDims *__restrict__ dims) {
    const int n_run = dims ? dims->N : N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const unsigned c = i < n_run ? ncand[i] : 0u;
        deg[i] = c < (unsigned)max_cand ? c : (unsigned)max_cand;
    }
}

// Chunks of anchors for the bundle/growth stages: chunk k starts at the first
// anchor whose pair offset is >= k * per_chunk (anchor-aligned, <= per_chunk +
// max_deg pairs each). chunk_start[k] for k in [1, nchunks); [0] = 0.
__global__ void k_chunk_starts(int N, const unsigned long long *__restrict__ pair_off, unsigned long long per_chunk,
                               int nchunks, int *__restrict__ chunk_start, const RunDims *__restrict__ dims) {
    if (dims) N = dims->N;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const unsigned long long lo = (i == 0) ? 0ull : pair_off[i - 1];
        const unsigned long long hi = pair_off[i];
        // chunk boundaries k with lo < k * per_chunk <= hi start at anchor i
        for (unsigned long long k = lo / per_chunk + 1; k * per_chunk <= hi && k < (unsigned long long)nchunks; ++k)
            chunk_start[k] = i;
    }
}

// A graph run's chunks (ChunkDims[K]) from k_chunk_starts' boundaries: the run has
// ceil(P / per_chunk) chunks (at least one); chunks beyond those are empty. A run
// with more than K chunks does not fit the graph: ERR_CAPACITY (the host runs it
// without the graph). One thread.
__global__ void k_chunk_dims(const RunDims *__restrict__ dims, const unsigned long long *__restrict__ pair_off,
                             const int *__restrict__ chunk_start, unsigned long long per_chunk, int K,
                             ChunkDims *__restrict__ cd, unsigned *__restrict__ err) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int N = dims->N;
    const unsigned long long P = pair_off[N];
    unsigned long long nch = (P + per_chunk - 1) / per_chunk;
    if (nch < 1) nch = 1;
    // more chunks than the graph holds: every chunk stays empty (the host runs the
    // map again kernel by kernel)
    const bool over = nch > (unsigned long long)K;
    if (over) atomicOr(err, ERR_CAPACITY);
    for (int c = 0; c < K; ++c) {
        int a0 = N, a1 = N;
        if (!over && (unsigned long long)c < nch) {
            a0 = c == 0 ? 0 : chunk_start[c];
            a1 = ((unsigned long long)c + 1 < nch && c + 1 < K) ? chunk_start[c + 1] : N;
        }
        cd[c].a_begin = a0;
        cd[c].a_end = a1;
        cd[c].p_begin = pair_off[a0];
        cd[c].p_end = pair_off[a1];
    }
}

}  // namespace cvl
