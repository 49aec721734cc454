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
        unsigned char *p = nb_smem + (size_t)wib * (size_t)md.max_cand * 20;
        S.d2 = (double *)p;
        S.key = (unsigned long long *)(p + (size_t)md.max_cand * 8);
        S.idx = (int *)(p + (size_t)md.max_cand * 16);
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

// ---------------------------------------------------------------------------
// Pair geometry and the bundle transport (cpu_curvelet.hpp:637-819)
// ---------------------------------------------------------------------------
struct PairGeom {
    double DX, DY, DX2, DY2;
    double sin_p_DY, cos_p_DX, sin_m_DY, cos_m_DX;
    bool close;    // DX2 + DY2 < 4*_dx*_dx (:682)
    bool branch1;  // DX*cos(T2) + DY*sin(T2) < 0 (:690)
};

__device__ __forceinline__ PairGeom pair_geom(const Model &md, double te_x, double te_y, double cosT2, double sinT2,
                                              double le_x, double le_y, double sp, double cp, double sm, double cm) {
    PairGeom g;
    g.DX = te_x - le_x;
    g.DY = te_y - le_y;
    g.DX2 = g.DX * g.DX;
    g.DY2 = g.DY * g.DY;
    g.close = (g.DX2 + g.DY2 < md.four_dx_dx);
    g.branch1 = ((g.DX * cosT2 + g.DY * sinT2) < 0);
    g.sin_p_DY = g.DY * sp;
    g.cos_p_DX = g.DX * cp;
    g.sin_m_DY = g.DY * sm;
    g.cos_m_DX = g.DX * cm;
    return g;
}

// One cell of the transport. dx2c/dt-index of the cell, sT/cT = sin/cos(T2t_j),
// s_m/s_p = sin(T2t_j - (T0 -+ dt)). bmin/bmax enter as -max_k/+max_k.
__device__ __forceinline__ void bundle_cell(const Model &md, const PairGeom &g, double delta_x2, double sT, double cT,
                                            double s_m, double s_p, double &bmin, double &bmax) {
    const double tt = sT * g.DX - cT * g.DY;
    const double ttmdx2 = tt - delta_x2;
    if (g.branch1) {
        const double eq_denom = (-2.0 * delta_x2 * tt + g.DX2 + g.DY2 - md.dx2 + delta_x2 * delta_x2);
        const double k_dx_min = 2.0 * (ttmdx2 - md.dx) / eq_denom;
        const double k_dx_max = 2.0 * (ttmdx2 + md.dx) / eq_denom;
        if (bmin < k_dx_min) bmin = k_dx_min;
        if (bmax > k_dx_max) bmax = k_dx_max;
        const double k_dt_min = s_m / (-s_m * delta_x2 + g.cos_m_DX + g.sin_m_DY);
        const double k_dt_max = s_p / (-s_p * delta_x2 + g.cos_p_DX + g.sin_p_DY);
        if (bmin < k_dt_min) bmin = k_dt_min;
        if (bmax > k_dt_max) bmax = k_dt_max;
    } else {
        const double eq_denom = -(2.0 * delta_x2 * tt - g.DX2 - g.DY2 + md.dx2 - delta_x2 * delta_x2) / 2.0;
        const double k_dx_min = (ttmdx2 - md.dx) / eq_denom;
        const double k_dx_max = (ttmdx2 + md.dx) / eq_denom;
        if (bmin < k_dx_min) bmin = k_dx_min;
        if (bmax > k_dx_max) bmax = k_dx_max;
        const double k_dt_max = s_m / (-s_m * delta_x2 + g.cos_m_DX + g.sin_m_DY);
        if (bmax > k_dt_max) bmax = k_dt_max;
        const double k_dt_min = s_p / (-s_p * delta_x2 + g.cos_p_DX + g.sin_p_DY);
        if (bmin < k_dt_min) bmin = k_dt_min;
    }
}

// Per-lane constants of the cells this lane owns: c = lane + 32*u.
template <int CPL>
struct LaneCells {
    double dx2[CPL];  // delta_x2 of the cell (cpu_curvelet.hpp:697)
    int j[CPL];       // orientation index of the cell
    bool on[CPL];     // c < cells
    unsigned rank[CPL];  // best-cell order (fill_curvelet_info, :202-219); ~0u if never eligible
};

template <int CPL>
__device__ __forceinline__ void lane_cells_init(const Model &md, int lane, LaneCells<CPL> &L) {
#pragma unroll
    for (int u = 0; u < CPL; ++u) {
        const int c = lane + 32 * u;
        L.on[u] = c < md.cells;
        const int ci = L.on[u] ? c / md.Q : 0;
        const int cj = L.on[u] ? c % md.Q : 0;
        L.j[u] = cj;
        L.dx2[u] = md.sx * ((double)ci - ((double)md.P - 1.0) / 2.0);
        // best-cell rank: cells with d < 100 ordered by (d, row-major index)
        const double ddx = md.sx * ((double)ci - ((double)md.P - 1.0) / 2.0);
        const double ddt = md.st * ((double)cj - ((double)md.Q - 1.0) / 2.0);
        const double d = ddx * ddx + ddt * ddt;
        unsigned rk = ~0u;
        if (L.on[u] && d < 100.0) {
            rk = 0;
            for (int o = 0; o < md.cells; ++o) {
                const int oi = o / md.Q, oj = o % md.Q;
                const double ox = md.sx * ((double)oi - ((double)md.P - 1.0) / 2.0);
                const double ot = md.st * ((double)oj - ((double)md.Q - 1.0) / 2.0);
                const double od = ox * ox + ot * ot;
                rk += (od < d) || (od == d && o < c);
            }
        }
        L.rank[u] = rk;
    }
}

// ---------------------------------------------------------------------------
// (c+d) fused bundles + chain growth + dedup + record: persistent, warp/anchor
// ---------------------------------------------------------------------------
struct CurveletArgs {
    Model md;
    Binned B;
    int N;
    const unsigned long long *pair_off;  // [N+1] internal order
    const int *csr_ids;                  // internal neighbour indices
    Records rec;                         // slots at pair_off
    unsigned *count;                     // [N] curvelets per anchor, by ORIGINAL index
    MapStats *stats;
    unsigned *work;                      // persistent work counter
    double *scratch;                     // global overflow bundles: [warps][max_deg][2][32*CPL]
    unsigned short *scratch_chain;       // [warps][max_deg][gms]
    int scratch_deg;                     // bundles per warp slot in scratch
    int slots;                           // bundles per warp in shared memory
    int count_only;                      // 1: valid_pairs only (form_pairwise_bundles)
    unsigned *err;
};

// shared memory per warp (bytes), see k_curvelets
__host__ __device__ inline size_t curvelet_smem_per_warp(int max_cand, int slots, int gms, int cpl) {
    size_t b = 0;
    b += 3 * QMAX * 8;                        // sT, cT, T2t
    b += 64 * 8;                              // pair trig table
    b += (size_t)max_cand * 4;                // neighbour internal index
    b += (size_t)max_cand * 1;                // neighbour class
    b += (size_t)max_cand * 2;                // run's seed list (neighbour positions)
    b = (b + 15) & ~(size_t)15;
    b += (size_t)slots * (size_t)gms * 2;     // chains (smem part)
    b = (b + 15) & ~(size_t)15;
    b += (size_t)slots * 2 * 32 * cpl * 8;    // bundles
    return b;
}

// neighbour class byte: bits 0-1 run (0 fwd, 1 bwd, 2 none), bit 2 close, bit 3 branch1
template <int CPL, int K>
__global__ void __launch_bounds__(128) k_curvelets(CurveletArgs a) {
    extern __shared__ __align__(16) unsigned char cv_smem[];
    const Model &md = a.md;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int gwarp = blockIdx.x * (blockDim.x >> 5) + wib;
    const size_t per_warp = curvelet_smem_per_warp(md.max_cand, a.slots, md.gms, CPL);
    unsigned char *base = cv_smem + (size_t)wib * per_warp;
    double *sT = (double *)base;
    double *cT = sT + QMAX;
    double *T2t = cT + QMAX;
    double *ptab = T2t + QMAX;                       // [64]
    int *nb_idx = (int *)(ptab + 64);                // [max_cand]
    unsigned char *nb_cls = (unsigned char *)(nb_idx + md.max_cand);
    unsigned short *seed_pos = (unsigned short *)(((uintptr_t)(nb_cls + md.max_cand) + 1) & ~(uintptr_t)1);
    unsigned char *p2 = (unsigned char *)(seed_pos + md.max_cand);
    p2 = (unsigned char *)(((uintptr_t)p2 + 15) & ~(uintptr_t)15);
    unsigned short *chain_sm = (unsigned short *)p2;  // [slots][gms]
    p2 += (size_t)a.slots * md.gms * 2;
    p2 = (unsigned char *)(((uintptr_t)p2 + 15) & ~(uintptr_t)15);
    double *bund_sm = (double *)p2;                   // [slots][2][32*CPL]
    double *bund_gl = a.scratch + (size_t)gwarp * (size_t)a.scratch_deg * 2 * 32 * CPL;
    unsigned short *chain_gl = a.scratch_chain + (size_t)gwarp * (size_t)a.scratch_deg * md.gms;

    LaneCells<CPL> L;
    lane_cells_init<CPL>(md, lane, L);
    const int BW = 2 * 32 * CPL;  // doubles per bundle
    const int TP = md.Q * 2;      // trig values per pair

    for (;;) {
        int i = 0;
        if (lane == 0) i = (int)atomicAdd(a.work, 1u);
        i = __shfl_sync(FULL, i, 0);
        if (i >= a.N) break;

        const int m = a.B.map[i];
        const int orig = a.B.orig[i];
        const double ax = a.B.x[i], ay = a.B.y[i], T2 = a.B.th[i];
        const unsigned long long off = a.pair_off[i];
        const int deg = (int)(a.pair_off[i + 1] - off);

        // per-anchor trig: sin/cos(T2 + delta_t2_j) (:702-705) and cos/sin(T2) (:690, dot)
        if (lane < md.Q) {
            const double delta_t2 = md.st * ((double)lane - ((double)md.Q - 1.0) / 2.0);
            const double t = T2 + delta_t2;
            T2t[lane] = t;
            sT[lane] = sin(t);
            cT[lane] = cos(t);
        }
        const double cosT2 = cos(T2);
        const double sinT2 = sin(T2);

        // neighbour classes: direction filter (:454-462), close pair, branch
        for (int k = lane; k < deg; k += 32) {
            const int n = a.csr_ids[off + k];
            nb_idx[k] = n;
            const double lx = a.B.x[n], ly = a.B.y[n];
            const double dir = to_2pi(atan2(ly - ay, lx - ax));  // angle_from_pt_to_pt(te, le)
            const double d = cos(dir) * cosT2 + sin(dir) * sinT2; // dot(dir, te_orient)
            const unsigned run = (d > 0) ? 0u : ((d < 0) ? 1u : 2u);
            const double DX = ax - lx, DY = ay - ly;
            const bool close = (DX * DX + DY * DY < md.four_dx_dx);
            const bool br = ((DX * cosT2 + DY * sinT2) < 0);
            nb_cls[k] = (unsigned char)(run | (close ? 4u : 0u) | (br ? 8u : 0u));
        }
        __syncwarp();

        double sTl[CPL], cTl[CPL];
#pragma unroll
        for (int u = 0; u < CPL; ++u) {
            sTl[u] = sT[L.j[u]];
            cTl[u] = cT[L.j[u]];
        }
        unsigned n_out = 0;
        unsigned valid_cnt = 0;

        for (int f = 0; f < 2; ++f) {
            // ---- bundles of this run's neighbours (+ run-less ones, counted in run 0)
            int ns = 0;  // seeds stored
            for (int k0 = 0; k0 < deg; k0 += 32) {
                const int k = k0 + lane;
                bool take = false;
                if (k < deg) {
                    const unsigned run = nb_cls[k] & 3u;
                    take = (run == (unsigned)f) || (f == 0 && run == 2u);
                }
                unsigned bal = __ballot_sync(FULL, take);
                while (bal) {
                    // process up to PB pairs per trig batch
                    const int PB = (32 / TP) > 0 ? (32 / TP) : 1;
                    int kk[4];
                    int nb = 0;
                    while (bal && nb < PB && nb < 4) {
                        const int b = __ffs(bal) - 1;
                        bal &= bal - 1;
                        kk[nb++] = k0 + b;
                    }
                    // trig of the batch: sin(T2t_j - (T0 -+ dt)) (:728-729)
                    for (int t = lane; t < nb * TP; t += 32) {
                        const int pb = t / TP, q = t % TP;
                        int kq = kk[0];
#pragma unroll
                        for (int z = 1; z < 4; ++z)
                            if (pb == z) kq = kk[z];
                        const double T0 = a.B.th[nb_idx[kq]];
                        const int jj = q % md.Q;
                        const double arg = (q < md.Q) ? (T2t[jj] - (T0 - md.dt)) : (T2t[jj] - (T0 + md.dt));
                        ptab[pb * TP + q] = sin(arg);
                    }
                    __syncwarp();
                    for (int pb = 0; pb < nb; ++pb) {
                        int kq = kk[0];
#pragma unroll
                        for (int z = 1; z < 4; ++z)
                            if (pb == z) kq = kk[z];
                        const unsigned cls = nb_cls[kq];
                        const int n = nb_idx[kq];
                        double bmin[CPL], bmax[CPL];
#pragma unroll
                        for (int u = 0; u < CPL; ++u) {
                            bmin[u] = -md.max_k;
                            bmax[u] = md.max_k;
                        }
                        bool valid;
                        if (cls & 4u) {
                            valid = true;  // close pair: default bundle, hyp true (:682-687)
                        } else {
                            const PairGeom g = pair_geom(md, ax, ay, cosT2, sinT2, a.B.x[n], a.B.y[n], a.B.sp[n],
                                                         a.B.cp[n], a.B.sm[n], a.B.cm[n]);
                            bool lv = false;
#pragma unroll
                            for (int u = 0; u < CPL; ++u) {
                                if (L.on[u]) {
                                    const int jj = L.j[u];
                                    bundle_cell(md, g, L.dx2[u], sTl[u], cTl[u], ptab[pb * TP + jj],
                                                ptab[pb * TP + md.Q + jj], bmin[u], bmax[u]);
                                    lv = lv || (bmax[u] > bmin[u]);
                                }
                            }
                            valid = __any_sync(FULL, lv);  // bundle_valid_check (:821-830)
                        }
                        if (valid) {
                            ++valid_cnt;
                            if ((cls & 3u) == (unsigned)f && !a.count_only) {
                                double *dst = (ns < a.slots) ? bund_sm + (size_t)ns * BW
                                                             : bund_gl + (size_t)(ns - a.slots) * BW;
                                if (ns - a.slots >= a.scratch_deg) {
                                    if (lane == 0) atomicOr(a.err, ERR_CAPACITY);
                                } else {
#pragma unroll
                                    for (int u = 0; u < CPL; ++u) {
                                        dst[lane + 32 * u] = bmin[u];
                                        dst[32 * CPL + lane + 32 * u] = bmax[u];
                                    }
                                    if (lane == 0) seed_pos[ns] = (unsigned short)kq;
                                }
                                ++ns;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            __syncwarp();
            // With group_max_sz <= 2 a chain stops at length 2 and the len > 2 gate
            // (:549) never passes: no growth needed (and no chain slot is written).
            if (a.count_only || ns == 0 || md.gms <= 2) continue;
            if (ns - a.slots > a.scratch_deg) ns = a.slots + a.scratch_deg;  // capacity error already raised

            // ---- chain growth: seeds in groups of K walk the seed list in lock step
            for (int g0 = 0; g0 < ns; g0 += K) {
                double cmin[K][CPL], cmax[K][CPL];
                unsigned len[K];
                unsigned short *chain[K];
                unsigned done = 0;
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    const int s = g0 + q;
                    chain[q] = (s < a.slots) ? chain_sm + (size_t)s * md.gms
                                             : chain_gl + (size_t)(s - a.slots) * md.gms;
                    if (s < ns) {
                        const double *src = (s < a.slots) ? bund_sm + (size_t)s * BW
                                                          : bund_gl + (size_t)(s - a.slots) * BW;
#pragma unroll
                        for (int u = 0; u < CPL; ++u) {
                            cmin[q][u] = src[lane + 32 * u];
                            cmax[q][u] = src[32 * CPL + lane + 32 * u];
                        }
                        len[q] = 1;  // the anchor (:485)
                    } else {
                        len[q] = 0;
                        done |= 1u << q;
#pragma unroll
                        for (int u = 0; u < CPL; ++u) cmin[q][u] = cmax[q][u] = 0.0;
                    }
                }
                if (lane == 0) {
#pragma unroll
                    for (int q = 0; q < K; ++q)
                        if (g0 + q < ns) chain[q][0] = 0xffffu;  // anchor marker
                }
                for (int r = 0; r < ns && done != (1u << K) - 1u; ++r) {
                    const double *src = (r < a.slots) ? bund_sm + (size_t)r * BW
                                                      : bund_gl + (size_t)(r - a.slots) * BW;
                    double rmin[CPL], rmax[CPL];
#pragma unroll
                    for (int u = 0; u < CPL; ++u) {
                        rmin[u] = src[lane + 32 * u];
                        rmax[u] = src[32 * CPL + lane + 32 * u];
                    }
                    // per seed: lane-local "some cell stays open" bit
                    unsigned bits = 0;
#pragma unroll
                    for (int q = 0; q < K; ++q) {
                        bool lv = false;
#pragma unroll
                        for (int u = 0; u < CPL; ++u) {
                            // bundle_intersection (:832-843)
                            const double lo = (cmin[q][u] < rmin[u]) ? rmin[u] : cmin[q][u];
                            const double hi = (cmax[q][u] > rmax[u]) ? rmax[u] : cmax[q][u];
                            lv = lv || (L.on[u] && hi > lo);
                        }
                        bits |= lv ? (1u << q) : 0u;
                    }
                    bits = __reduce_or_sync(FULL, bits);  // bundle_intersection_valid_check (:845-854)
#pragma unroll
                    for (int q = 0; q < K; ++q) {
                        if (done & (1u << q)) continue;
                        const int s = g0 + q;
                        if (r == s) {
                            // the seed itself joins without intersection (:496-511)
                            if (lane == 0) chain[q][len[q]] = (unsigned short)r;
                            ++len[q];
                            if (len[q] >= (unsigned)md.gms) done |= 1u << q;
                            continue;
                        }
                        if (bits & (1u << q)) {
                            if (lane == 0) chain[q][len[q]] = (unsigned short)r;
                            ++len[q];
                            // move_to_cmp_bundle(0, ..., true): the running bundle becomes the intersection
#pragma unroll
                            for (int u = 0; u < CPL; ++u) {
                                cmin[q][u] = (cmin[q][u] < rmin[u]) ? rmin[u] : cmin[q][u];
                                cmax[q][u] = (cmax[q][u] > rmax[u]) ? rmax[u] : cmax[q][u];
                            }
                        }
                        if (len[q] >= (unsigned)md.gms) done |= 1u << q;
                    }
                }
                __syncwarp();
                // ---- dedup (first identical chain in seed order wins, :876-916) + record
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    const int s = g0 + q;
                    if (s >= ns || len[q] <= 2u) continue;  // len > 2 gate (:549)
                    if (lane == 0) chain[q][0] = (unsigned short)len[q] | 0x8000u;  // store length in slot 0
                    __syncwarp();
                    // compare with every earlier seed of this run whose chain has the same length
                    bool dup = false;
                    for (int p = lane; p < s; p += 32) {
                        const unsigned short *cp = (p < a.slots) ? chain_sm + (size_t)p * md.gms
                                                                 : chain_gl + (size_t)(p - a.slots) * md.gms;
                        if (cp[0] == chain[q][0]) {
                            bool same = true;
                            for (unsigned z = 1; z < len[q]; ++z) same = same && (cp[z] == chain[q][z]);
                            dup = dup || same;
                        }
                    }
                    if (__any_sync(FULL, dup)) continue;
                    // best cell of the final bundle: smallest rank among open cells
                    unsigned best = ~0u;
#pragma unroll
                    for (int u = 0; u < CPL; ++u)
                        if (L.on[u] && cmax[q][u] > cmin[q][u] && L.rank[u] < best) best = L.rank[u];
                    best = __reduce_min_sync(FULL, best);
                    // lane owning the best cell publishes (cell, k_max, k_min); none -> cell 0 (:202-204)
                    int bcell = 0;
                    double kmax = 0.0, kmin = 0.0;
                    {
                        int mycell = -1;
                        double mymax = 0.0, mymin = 0.0;
#pragma unroll
                        for (int u = 0; u < CPL; ++u) {
                            const bool hit = (best != ~0u) ? (L.on[u] && L.rank[u] == best && cmax[q][u] > cmin[q][u])
                                                           : (lane + 32 * u == 0);
                            if (hit) {
                                mycell = lane + 32 * u;
                                mymax = cmax[q][u];
                                mymin = cmin[q][u];
                            }
                        }
                        const unsigned who = __ballot_sync(FULL, mycell >= 0);
                        const int src = who ? (__ffs(who) - 1) : 0;
                        bcell = __shfl_sync(FULL, mycell, src);
                        kmax = __shfl_sync(FULL, mymax, src);
                        kmin = __shfl_sync(FULL, mymin, src);
                    }
                    if (lane == 0) {
                        const unsigned long long slot = off + n_out;
                        unsigned *ids = a.rec.ids + slot * (unsigned long long)md.gms;
                        ids[0] = (unsigned)orig;
                        for (unsigned z = 1; z < len[q]; ++z)
                            ids[z] = (unsigned)a.B.orig[nb_idx[seed_pos[chain[q][z]]]];
                        a.rec.k[slot * 2 + 0] = kmax;
                        a.rec.k[slot * 2 + 1] = kmin;
                        a.rec.meta[slot] = len[q] | ((unsigned)bcell << 8) | ((f == 0 ? 1u : 0u) << 24);
                    }
                    ++n_out;
                }
                __syncwarp();
            }
        }
        if (lane == 0) {
            if (!a.count_only) a.count[orig] = n_out;
            atomicAdd(&a.stats[m].valid_pairs, valid_cnt);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// (e) finalize: records -> chain rows + info rows at anchor-major positions
// ---------------------------------------------------------------------------
__global__ void k_finalize(Model md, const double *__restrict__ edges, int sz, int N, const int *__restrict__ map_off,
                           int M, const int *__restrict__ orig_of, const unsigned long long *__restrict__ pair_off,
                           Records rec, const unsigned *__restrict__ count,
                           const unsigned long long *__restrict__ out_off, unsigned *__restrict__ chains,
                           double *__restrict__ info) {
    const int W = md.gms + 1;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int a = orig_of[i];
        const unsigned n = count[a];
        if (n == 0) continue;
        const int m = map_of(map_off, M, a);
        const int moff = map_off[m];
        const unsigned long long src = pair_off[i];
        const unsigned long long dst = out_off[a];
        const double ref_x = edges[(size_t)a * sz + 0];
        const double ref_y = edges[(size_t)a * sz + 1];
        const double ref_theta = edges[(size_t)a * sz + 2];
        for (unsigned r = 0; r < n; ++r) {
            const unsigned long long s = src + r;
            const unsigned long long d = dst + r;
            const unsigned meta = rec.meta[s];
            const unsigned len = meta & 0xffu;
            const unsigned bcell = (meta >> 8) & 0xffffu;
            const bool forward = (meta >> 24) & 1u;
            const unsigned *ids = rec.ids + s * (unsigned long long)md.gms;
            // chain row (record_curvelet_chain, :269-276): [anchor+1, chain[0]+1, ...], zero padded
            unsigned *row = chains + d * (unsigned long long)W;
            row[0] = (unsigned)(a - moff) + 1u;
            for (int z = 0; z + 1 < W; ++z) row[z + 1] = (z < (int)len) ? (ids[z] - (unsigned)moff) + 1u : 0u;
            // fill_curvelet_info (:221-255)
            const int mini = (int)bcell / md.Q, minj = (int)bcell % md.Q;
            const double k_max = rec.k[s * 2 + 0];
            const double k_min = rec.k[s * 2 + 1];
            const double k = (k_max + k_min) / 2.0;
            const double dx = md.sx * ((double)mini - ((double)md.P - 1.0) / 2.0);
            const double dt = md.st * ((double)minj - ((double)md.Q - 1.0) / 2.0);
            const double theta = to_2pi(ref_theta + dt);
            const double pt_x = ref_x - dx * sin(theta);
            const double pt_y = ref_y + dx * cos(theta);
            double length = 0.0;
            for (unsigned z = 0; z + 1 < len; ++z) {
                const unsigned e1 = ids[z], e2 = ids[z + 1];
                length += sqrt(sq_dist(edges[(size_t)e1 * sz + 0], edges[(size_t)e1 * sz + 1],
                                       edges[(size_t)e2 * sz + 0], edges[(size_t)e2 * sz + 1]));
            }
            const double quality =
                (length > 0.0 && len > 0) ? 2.0 / (1.0 * md.nrad / length + 1.0 * length / (double)len) : 0.0;
            double *inf = info + d * 10ull;
            inf[0] = forward ? 1.0 : 0.0;
            inf[1] = k_max;
            inf[2] = k_min;
            inf[3] = ref_theta;
            inf[4] = pt_x;
            inf[5] = pt_y;
            inf[6] = theta;
            inf[7] = k;
            inf[8] = length;
            inf[9] = quality;
        }
    }
}

// ---------------------------------------------------------------------------
// Standalone transport for independent pairs (cvl_pair_bundles): warp per pair,
// the same bundle_cell as the fused kernel.
// pairs[p] = (te_x, te_y, te_theta, le_x, le_y, le_theta)
// ---------------------------------------------------------------------------
template <int CPL>
__global__ void __launch_bounds__(128) k_pair_bundles(Model md, const double *__restrict__ pairs, int n,
                                                      double *__restrict__ bmin_out, double *__restrict__ bmax_out,
                                                      unsigned char *__restrict__ valid_out) {
    __shared__ double tab[4][4 * QMAX];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *sT = tab[wib], *cT = sT + QMAX, *sM = cT + QMAX, *sP = sM + QMAX;
    LaneCells<CPL> L;
    lane_cells_init<CPL>(md, lane, L);
    for (int p = blockIdx.x * 4 + wib; p < n; p += gridDim.x * 4) {
        const double *q = pairs + (size_t)p * 6;
        const double te_x = q[0], te_y = q[1], T2 = q[2], le_x = q[3], le_y = q[4], T0 = q[5];
        for (int j = lane; j < md.Q; j += 32) {
            const double t = T2 + md.st * ((double)j - ((double)md.Q - 1.0) / 2.0);
            sT[j] = sin(t);
            cT[j] = cos(t);
            sM[j] = sin(t - (T0 - md.dt));
            sP[j] = sin(t - (T0 + md.dt));
        }
        __syncwarp();
        const double t_p = T0 + md.dt, t_m = T0 - md.dt;
        const PairGeom g = pair_geom(md, te_x, te_y, cos(T2), sin(T2), le_x, le_y, sin(t_p), cos(t_p), sin(t_m),
                                     cos(t_m));
        double bmin[CPL], bmax[CPL];
        bool lv = false;
#pragma unroll
        for (int u = 0; u < CPL; ++u) {
            bmin[u] = -md.max_k;
            bmax[u] = md.max_k;
            if (!g.close && L.on[u]) {
                const int jj = L.j[u];
                bundle_cell(md, g, L.dx2[u], sT[jj], cT[jj], sM[jj], sP[jj], bmin[u], bmax[u]);
            }
            lv = lv || (L.on[u] && bmax[u] > bmin[u]);
        }
        const bool valid = g.close ? true : (bool)__any_sync(FULL, lv);
#pragma unroll
        for (int u = 0; u < CPL; ++u) {
            if (L.on[u]) {
                bmin_out[(size_t)p * md.cells + lane + 32 * u] = bmin[u];
                bmax_out[(size_t)p * md.cells + lane + 32 * u] = bmax[u];
            }
        }
        if (lane == 0) valid_out[p] = valid ? 1 : 0;
        __syncwarp();
    }
}

// CSR in the reference's layout (anchor = input order, neighbour ids = input
// indices local to the map) from the internal CSR.
__global__ void k_graph_degrees(int N, const int *__restrict__ orig_of, const unsigned long long *__restrict__ pair_off,
                                unsigned *__restrict__ deg_orig) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        deg_orig[orig_of[i]] = (unsigned)(pair_off[i + 1] - pair_off[i]);
}

__global__ void k_graph_export(int N, const int *__restrict__ orig_of, const int *__restrict__ map_off, int M,
                               const unsigned long long *__restrict__ pair_off, const int *__restrict__ csr_ids,
                               const double *__restrict__ csr_d2, const unsigned long long *__restrict__ off_orig,
                               int *__restrict__ ids_out, double *__restrict__ d2_out) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const int a = orig_of[i];
        const int moff = map_off[map_of(map_off, M, a)];
        const unsigned long long s = pair_off[i], e = pair_off[i + 1], d = off_orig[a];
        for (unsigned long long k = s; k < e; ++k) {
            ids_out[d + (k - s)] = orig_of[csr_ids[k]] - moff;
            d2_out[d + (k - s)] = csr_d2[k];
        }
    }
}

__global__ void k_deg_from_ncand(int N, int max_cand, const unsigned *__restrict__ ncand, unsigned *__restrict__ deg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x) {
        const unsigned c = ncand[i];
        deg[i] = c < (unsigned)max_cand ? c : (unsigned)max_cand;
    }
}

// FP64 FMA throughput probe: independent dependent-chains per thread, all in registers.
__global__ void k_fp64_peak(double *out, int iters, double seed) {
    double a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
           a7 = a0 + 7;
    const double b = 0.999999, c = 1e-7;
    for (int k = 0; k < iters; ++k) {
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            a0 = fma(a0, b, c); a1 = fma(a1, b, c); a2 = fma(a2, b, c); a3 = fma(a3, b, c);
            a4 = fma(a4, b, c); a5 = fma(a5, b, c); a6 = fma(a6, b, c); a7 = fma(a7, b, c);
        }
    }
    const double s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == 12345.678) out[0] = s;  // keeps the chains live
}

// Writes a buffer larger than L2 (timing hygiene).
__global__ void k_flush(unsigned *buf, size_t n, unsigned v) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        buf[i] = v + (unsigned)i;
}

}  // namespace cvl
