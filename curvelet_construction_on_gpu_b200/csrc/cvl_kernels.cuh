// cvl_kernels.cuh -- sm_100a kernels of the curvelet path (FP64, no FMA contraction).
//
// Pipeline over a ragged batch of M edge maps (M = 1 for the plain form):
//   (a) k_bin_keys / k_bin_scatter  spatial-hash binning by counting sort into
//       S x S pixel-cell blocks ("cells sized to the neighbourhood"), SoA FP64
//       edge arrays, per-edge trig of theta +- dt precomputed once;
//   (b) k_neighbors<COUNT|FILL>     warp per anchor: the reference's 7x7
//       pixel-window + radius predicate (preprocess.hpp:129-167), candidates
//       staged in shared memory, truncation in window-scan order, rank sort by
//       (dist^2, scan position) (preprocess.hpp:172-176);
//   (c+d) k_curvelets               warp per anchor, persistent: pairwise
//       curve bundles (cpu_curvelet.hpp:637-819) with cells across lanes,
//       kept in shared memory, then lock-step chain growth of groups of seeds
//       with warp-vote bundle intersections (:479-545), first-wins dedup
//       (:876-916) and compact records (:258-280);
//   (e) k_finalize                  expands records into the chain rows and
//       the 10 info columns (fill_curvelet_info, :197-256) at anchor-major
//       output positions (compact_curvelet_output, :282-303).
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
constexpr double CVL_PI = 3.14159265358979323846;  // curvelet_utils.hpp:10

// Error bits raised by kernels (checked by the host after a run).
constexpr unsigned ERR_NONFINITE = 1u;   // non-finite or out-of-range coordinate
constexpr unsigned ERR_CAPACITY = 2u;    // a device capacity was exceeded
constexpr unsigned ERR_INTERNAL = 4u;    // an internal invariant failed (bounds check)

struct Model {
    double nrad, rad_sqr;      // neighbour radius and its square (preprocess.hpp:221)
    double dx, dx2, four_dx_dx;  // _dx, _dx*_dx, 4*_dx*_dx (cpu_curvelet.hpp:654,682)
    double dt, sx, st, max_k;  // dt in radians (main.cpp:24)
    int P, Q, cells;           // bundle grid (cpu_curvelet.hpp:73-74)
    int gms;                   // group_max_sz
    int max_cand;              // max_candidates
    int w;                     // pixel-window half width (3, main.cpp:48)
    int S;                     // hash block edge in pixel cells
    unsigned hash_mask;        // table size - 1
};

// SoA copy of the edges in hash-bucket order ("internal" index space).
struct Binned {
    double *x, *y, *th;        // position, orientation
    double *sp, *cp, *sm, *cm; // sin/cos(theta + dt), sin/cos(theta - dt)
    int2 *cell;                // pixel cell (lrint(x), lrint(y))
    int *orig;                 // global input index
    int *map;                  // map of the edge
};

struct MapStats {
    unsigned long long pairs;  // total_neighbor_pairs
    unsigned max_deg;          // max_num_of_neighbors
    unsigned truncated;        // anchors that reached max_candidates
    unsigned valid_pairs;      // pairs with a valid bundle
    unsigned pad;
};

// Compact curvelet record written by k_curvelets at the anchor's pair slots.
//   rec_ids  [slot][gms]  chain as global edge indices (anchor first)
//   rec_k    [slot][2]    k_max, k_min of the best cell of the final bundle
//   rec_meta [slot]       len | best_cell << 8 | forward << 24
struct Records {
    unsigned *ids;
    double *k;
    unsigned *meta;
};

__device__ __forceinline__ int floor_div(int a, int s) { return a >= 0 ? a / s : -((-a + s - 1) / s); }

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
__device__ __forceinline__ double sq_dist(double x1, double y1, double x2, double y2) {
    return (x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2);
}

// To2Pi (curvelet_utils.hpp:25-46)
__device__ __forceinline__ double to_2pi(double angle) {
    double a;
    if (angle >= 2.0 * CVL_PI)
        a = fmod(angle, 2.0 * CVL_PI);
    else if (angle < 0)
        a = (2.0 * CVL_PI + fmod(angle, 2.0 * CVL_PI));
    else
        a = angle;
    if (!(a >= 0 && a < 2.0 * CVL_PI)) a = 0;
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
__global__ void k_bin_keys(const double *__restrict__ edges, int sz, int N, const int *__restrict__ map_off, int M,
                           Model md, unsigned *__restrict__ ehash, unsigned *__restrict__ bcount,
                           unsigned *__restrict__ err) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N; e += gridDim.x * blockDim.x) {
        const double x = edges[(size_t)e * sz + 0];
        const double y = edges[(size_t)e * sz + 1];
        const double th = edges[(size_t)e * sz + 2];
        if (!isfinite(x) || !isfinite(y) || !isfinite(th) || fabs(x) >= 1.0e9 || fabs(y) >= 1.0e9) {
            atomicOr(err, ERR_NONFINITE);
            ehash[e] = 0;
            atomicAdd(&bcount[0], 1u);
            continue;
        }
        const int m = map_of(map_off, M, e);
        const int cx = __double2int_rn(x);  // lrint, round half to even (preprocess.hpp:85-86)
        const int cy = __double2int_rn(y);
        const unsigned h = cell_hash(m, floor_div(cx, md.S), floor_div(cy, md.S)) & md.hash_mask;
        ehash[e] = h;
        atomicAdd(&bcount[h], 1u);
    }
}

__global__ void k_bin_scatter(const double *__restrict__ edges, int sz, int N, const int *__restrict__ map_off,
                              int M, Model md, const unsigned *__restrict__ ehash,
                              const unsigned *__restrict__ bstart, unsigned *__restrict__ bfill, Binned B,
                              int *__restrict__ pos_of) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < N; e += gridDim.x * blockDim.x) {
        const unsigned h = ehash[e];
        const unsigned pos = bstart[h] + atomicAdd(&bfill[h], 1u);
        const double x = edges[(size_t)e * sz + 0];
        const double y = edges[(size_t)e * sz + 1];
        const double th = edges[(size_t)e * sz + 2];
        B.x[pos] = x;
        B.y[pos] = y;
        B.th[pos] = th;
        // T0 +- dt and their sin/cos (cpu_curvelet.hpp:655-656, 730-733), once per edge
        const double t_p = th + md.dt;
        const double t_m = th - md.dt;
        B.sp[pos] = sin(t_p);
        B.cp[pos] = cos(t_p);
        B.sm[pos] = sin(t_m);
        B.cm[pos] = cos(t_m);
        B.cell[pos] = make_int2(__double2int_rn(x), __double2int_rn(y));
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

struct NbrSmem {  // per-warp candidate staging, capacity max_cand
    double *d2;
    unsigned long long *key;
    int *idx;
};

enum { NB_COUNT = 0, NB_FILL = 1 };

// Per-warp candidate staging bytes: d2 (8) + key (8) + idx (4) per candidate,
// rounded up to 16 so every warp's arrays start 16-byte aligned.
__host__ __device__ inline size_t nbr_smem_per_warp(int max_cand) {
    return ((size_t)max_cand * 20 + 15) & ~(size_t)15;
}

// Visits every edge in the anchor's window that passes the reference's
// predicate; f(lane_ok, j, d2, key) is called warp-uniformly per chunk of 32.
template <typename F>
__device__ __forceinline__ void for_window_candidates(const Model &md, const Binned &B, const unsigned *bstart,
                                                      int i, int m, int2 ac, double ax, double ay, int lane, F &&f) {
    const int bx0 = floor_div(ac.x - md.w, md.S), bx1 = floor_div(ac.x + md.w, md.S);
    const int by0 = floor_div(ac.y - md.w, md.S), by1 = floor_div(ac.y + md.w, md.S);
    for (int by = by0; by <= by1; ++by) {
        for (int bx = bx0; bx <= bx1; ++bx) {
            const unsigned h = cell_hash(m, bx, by) & md.hash_mask;
            const int b0 = (int)bstart[h], b1 = (int)bstart[h + 1];
            for (int base = b0; base < b1; base += 32) {
                const int j = base + lane;
                bool ok = false;
                double d2 = 0.0;
                unsigned long long key = 0;
                if (j < b1 && j != i) {
                    const int2 c = B.cell[j];
                    if (B.map[j] == m && floor_div(c.x, md.S) == bx && floor_div(c.y, md.S) == by &&
                        abs(c.x - ac.x) <= md.w && abs(c.y - ac.y) <= md.w) {
                        d2 = sq_dist(ax, ay, B.x[j], B.y[j]);  // sq_dist(te, ne), preprocess.hpp:160
                        ok = !(d2 > md.rad_sqr);               // preprocess.hpp:161-163
                        key = scan_key(c, ac.x, ac.y, md.w, B.orig[j]);
                    }
                }
                f(ok, j, d2, key);
            }
        }
    }
}

// COUNT: ncand[i] = candidates in window (before the cap), per-map stats.
// FILL:  csr_ids/csr_d2 at pair_off[i], sorted by (d2, scan key), truncated
//        to max_cand in scan order when ncand[i] > max_cand.
template <int MODE>
__global__ void __launch_bounds__(256) k_neighbors(Model md, Binned B, const unsigned *__restrict__ bstart, int N,
                                                   unsigned *__restrict__ ncand, MapStats *__restrict__ stats,
                                                   const unsigned long long *__restrict__ pair_off,
                                                   int *__restrict__ csr_ids, double *__restrict__ csr_d2,
                                                   unsigned *__restrict__ err) {
    extern __shared__ __align__(16) unsigned char nb_smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    NbrSmem S;
    {
        unsigned char *p = nb_smem + (size_t)wib * nbr_smem_per_warp(md.max_cand);
        S.d2 = (double *)p;
        S.key = (unsigned long long *)(p + (size_t)md.max_cand * 8);
        S.idx = (int *)(p + (size_t)md.max_cand * 16);
        if (MODE == NB_FILL && (((uintptr_t)S.d2 | (uintptr_t)S.key) & 7u)) {  // layout self-check
            if ((threadIdx.x & 31) == 0) atomicOr(err, ERR_INTERNAL);
            return;
        }
    }
    const unsigned lt_mask = (1u << lane) - 1u;
    for (int i = blockIdx.x * wpb + wib; i < N; i += gridDim.x * wpb) {
        const int m = B.map[i];
        const int2 ac = B.cell[i];
        const double ax = B.x[i], ay = B.y[i];
        if (MODE == NB_COUNT) {
            unsigned cnt = 0;
            for_window_candidates(md, B, bstart, i, m, ac, ax, ay, lane,
                                  [&](bool ok, int, double, unsigned long long) {
                                      cnt += __popc(__ballot_sync(FULL, ok));
                                  });
            if (lane == 0) {
                ncand[i] = cnt;
                const unsigned deg = cnt < (unsigned)md.max_cand ? cnt : (unsigned)md.max_cand;
                atomicAdd(&stats[m].pairs, (unsigned long long)deg);
                atomicMax(&stats[m].max_deg, deg);
                if (deg >= (unsigned)md.max_cand) atomicAdd(&stats[m].truncated, 1u);
            }
            continue;
        }
        const unsigned total = ncand[i];
        unsigned n = 0;
        if (total <= (unsigned)md.max_cand) {
            for_window_candidates(md, B, bstart, i, m, ac, ax, ay, lane,
                                  [&](bool ok, int j, double d2, unsigned long long key) {
                                      const unsigned bal = __ballot_sync(FULL, ok);
                                      if (ok) {
                                          const unsigned p = n + __popc(bal & lt_mask);
                                          if (p < (unsigned)md.max_cand) {
                                              S.d2[p] = d2;
                                              S.key[p] = key;
                                              S.idx[p] = j;
                                          } else {
                                              atomicOr(err, ERR_INTERNAL);
                                          }
                                      }
                                      n += __popc(bal);
                                  });
        } else {
            // Truncation (preprocess.hpp:165-167): keep the first max_cand
            // candidates in window-scan order. Walk the window pixel cell by
            // pixel cell; inside the cell where the cap is crossed keep the
            // lowest edge indices.
            const int side = 2 * md.w + 1;
            for (int r = 0; r < side * side && n < (unsigned)md.max_cand; ++r) {
                const int px = ac.x - md.w + r % side;
                const int py = ac.y - md.w + r / side;
                const int bx = floor_div(px, md.S), by = floor_div(py, md.S);
                const unsigned h = cell_hash(m, bx, by) & md.hash_mask;
                const int b0 = (int)bstart[h], b1 = (int)bstart[h + 1];
                // count this cell's candidates
                unsigned c = 0;
                for (int base = b0; base < b1; base += 32) {
                    const int j = base + lane;
                    bool ok = false;
                    if (j < b1 && j != i) {
                        const int2 cc = B.cell[j];
                        ok = B.map[j] == m && cc.x == px && cc.y == py &&
                             !(sq_dist(ax, ay, B.x[j], B.y[j]) > md.rad_sqr);
                    }
                    c += __popc(__ballot_sync(FULL, ok));
                }
                const unsigned need = (unsigned)md.max_cand - n;
                for (int base = b0; base < b1; base += 32) {
                    const int j = base + lane;
                    bool ok = false;
                    double d2 = 0.0;
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
            if (n > (unsigned)md.max_cand) n = (unsigned)md.max_cand;
        }
        __syncwarp();
        // rank sort by (d2, scan key) -- std::sort by distance, preprocess.hpp:172-176
        const unsigned long long off = pair_off[i];
        for (unsigned t = lane; t < n; t += 32) {
            const double dt_ = S.d2[t];
            const unsigned long long kt = S.key[t];
            unsigned rk = 0;
            for (unsigned u = 0; u < n; ++u) {
                const double du = S.d2[u];
                rk += (du < dt_) || (du == dt_ && S.key[u] < kt);
            }
            csr_ids[off + rk] = S.idx[t];
            if (csr_d2) csr_d2[off + rk] = dt_;
        }
        __syncwarp();
    }
}

}  // namespace cvl
