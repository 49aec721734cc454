// cvl_curvelets.cuh -- (c+d) the fused curve-bundle / chain-growth kernel, (e) the
// output expansion, and the small utility kernels.
//
// k_curvelets: one warp per anchor (static round-robin over anchors). Per anchor:
//   1. classify its neighbours (lane per neighbour): direction run (dot of the
//      anchor orientation with the anchor->neighbour angle, cpu_curvelet.hpp:454-462),
//      close pair (:682), transport branch (:690);
//   2. per direction run, the run's pairs in chunks of PCH: stage each pair's
//      geometry and its 2Q sin(T2t_j - T0 -+ dt) values in shared memory, then
//      one compact task loop over (pair, cell) computes the bundle cells
//      (:693-810) into the pair's slot; a warp vote per pair gives validity
//      (bundle_valid_check, :821-830) and the run's seeds are compacted;
//   3. chain growth: seeds in groups of K walk the run's seed list in lock step;
//      each intersection (:832-854) is one __reduce_or_sync vote;
//   4. first-wins dedup (:876-916) and a compact record per accepted chain
//      (best cell, k_max, k_min, ids) at the anchor's pair slots.
// Seed bundles live in shared memory (slots per warp) and spill to a per-warp
// global scratch area when a run has more seeds than slots.
#pragma once

#include "cvl_kernels.cuh"

namespace cvl {

constexpr int PCH = 4;      // pairs per transport chunk
constexpr int GEO_N = 8;    // doubles of staged pair geometry
constexpr int CELLS_MAX = 128;
constexpr size_t CELL_TABLE_BYTES = CELLS_MAX * 8 + CELLS_MAX * 1 + CELLS_MAX * 2 + 128;  // dx2, j, rank (+pad)

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

// One cell of the transport, both branches in one branch-free body. Branch 1
// (:693-754): eq = -2 dx2 tt + DX2 + DY2 - dx^2 + dx2^2, k_dx = 2 (ttmdx2 -+ dx) / eq,
// k_dt_min = s_m / (...), k_dt_max = s_p / (...). Branch 2 (:758-809):
// eq = -(2 dx2 tt - DX2 - DY2 + dx^2 - dx2^2) / 2, k_dx = (ttmdx2 -+ dx) / eq,
// k_dt_max = s_m / (...), k_dt_min = s_p / (...). Each formula keeps the
// reference's operand order; the clamp order per bound is the reference's.
// (x / 2.0 and x * 0.5 are the same correctly rounded value.)
__device__ __forceinline__ void bundle_cell(const Model &md, double DX, double DY, double DX2, double DY2,
                                            double sin_p_DY, double cos_p_DX, double sin_m_DY, double cos_m_DX,
                                            bool branch1, double delta_x2, double sT, double cT, double s_m,
                                            double s_p, double &bmin, double &bmax) {
    const double tt = sT * DX - cT * DY;
    const double ttmdx2 = tt - delta_x2;
    const double e1 = (-2.0 * delta_x2 * tt + DX2 + DY2 - md.dx2 + delta_x2 * delta_x2);
    const double e2 = -(2.0 * delta_x2 * tt - DX2 - DY2 + md.dx2 - delta_x2 * delta_x2) * 0.5;
    const double lo = ttmdx2 - md.dx, hi = ttmdx2 + md.dx;
    const double den = branch1 ? e1 : e2;
    const double k_dx_min = (branch1 ? 2.0 * lo : lo) / den;
    const double k_dx_max = (branch1 ? 2.0 * hi : hi) / den;
    const double km = s_m / (-s_m * delta_x2 + cos_m_DX + sin_m_DY);
    const double kp = s_p / (-s_p * delta_x2 + cos_p_DX + sin_p_DY);
    if (bmin < k_dx_min) bmin = k_dx_min;
    if (bmax > k_dx_max) bmax = k_dx_max;
    const double k2min = branch1 ? km : kp;
    const double k2max = branch1 ? kp : km;
    if (bmin < k2min) bmin = k2min;
    if (bmax > k2max) bmax = k2max;
}

// Cell constants: delta_x2 (:697), orientation index j, and the best-cell rank of
// fill_curvelet_info (:202-219): cells with d < 100 ordered by (d, row-major index);
// 0xffff = never eligible.
__device__ __forceinline__ void cell_tables_init(const Model &md, double *dx2, unsigned char *cj,
                                                 unsigned short *rank) {
    for (int c = threadIdx.x; c < CELLS_MAX; c += blockDim.x) {
        if (c >= md.cells) {
            dx2[c] = 0.0;
            cj[c] = 0;
            rank[c] = 0xffffu;
            continue;
        }
        const int ci = c / md.Q, j = c % md.Q;
        dx2[c] = md.sx * ((double)ci - ((double)md.P - 1.0) / 2.0);
        cj[c] = (unsigned char)j;
        const double ddx = md.sx * ((double)ci - ((double)md.P - 1.0) / 2.0);
        const double ddt = md.st * ((double)j - ((double)md.Q - 1.0) / 2.0);
        const double d = ddx * ddx + ddt * ddt;
        unsigned rk = 0xffffu;
        if (d < 100.0) {
            rk = 0;
            for (int o = 0; o < md.cells; ++o) {
                const int oi = o / md.Q, oj = o % md.Q;
                const double ox = md.sx * ((double)oi - ((double)md.P - 1.0) / 2.0);
                const double ot = md.st * ((double)oj - ((double)md.Q - 1.0) / 2.0);
                const double od = ox * ox + ot * ot;
                rk += (od < d) || (od == d && o < c);
            }
        }
        rank[c] = (unsigned short)rk;
    }
}

// ---------------------------------------------------------------------------
// (c+d) the fused kernel
// ---------------------------------------------------------------------------
struct CurveletArgs {
    Model md;
    Binned B;
    int N;
    const unsigned long long *pair_off;  // [N+1] internal order
    const int *csr_ids;                  // internal neighbour indices
    Records rec;                         // slots at pair_off
    unsigned *count;                     // [N] curvelets per anchor, by input index
    MapStats *stats;
    double *scratch;                     // [warps][scratch_slots][2][32*CPL]
    unsigned short *scratch_chain;       // [warps][scratch_slots][gms]
    int scratch_slots;                   // bundle slots per warp in global scratch
    int slots;                           // bundle slots per warp in shared memory
    int count_only;                      // 1: valid_pairs only (form_pairwise_bundles)
    unsigned *err;
};

struct WarpLayout {
    size_t sT, cT, T2t, geo, gflag, tab, ck, nb_idx, nb_orig, seed_orig, nb_cls, chain, bund, total;
};

__host__ __device__ inline size_t lay_take(size_t &b, size_t bytes, size_t align) {
    b = (b + align - 1) & ~(align - 1);
    const size_t o = b;
    b += bytes;
    return o;
}

__host__ __device__ inline WarpLayout curvelet_warp_layout(int max_cand, int slots, int gms, int cpl, int Q) {
    WarpLayout L;
    size_t b = 0;
    L.sT = lay_take(b, QMAX * 8, 16);
    L.cT = lay_take(b, QMAX * 8, 8);
    L.T2t = lay_take(b, QMAX * 8, 8);
    L.geo = lay_take(b, (size_t)PCH * GEO_N * 8, 8);
    L.gflag = lay_take(b, (size_t)PCH * 4, 4);
    L.tab = lay_take(b, (size_t)PCH * 2 * Q * 8, 8);
    L.ck = lay_take(b, (size_t)PCH * 4, 4);
    L.nb_idx = lay_take(b, (size_t)max_cand * 4, 4);
    L.nb_orig = lay_take(b, (size_t)max_cand * 4, 4);
    L.seed_orig = lay_take(b, (size_t)max_cand * 4, 4);
    L.nb_cls = lay_take(b, (size_t)max_cand, 1);
    L.chain = lay_take(b, (size_t)slots * gms * 2, 16);
    L.bund = lay_take(b, (size_t)slots * 2 * 32 * cpl * 8, 16);
    L.total = (b + 15) & ~(size_t)15;
    return L;
}

__host__ __device__ inline size_t curvelet_smem_bytes(int warps, int max_cand, int slots, int gms, int cpl, int Q) {
    return CELL_TABLE_BYTES + (size_t)warps * curvelet_warp_layout(max_cand, slots, gms, cpl, Q).total;
}

// neighbour class byte: bits 0-1 run (0 fwd, 1 bwd, 2 none), bit 2 close
template <int CPL, int K>
__global__ void __launch_bounds__(128, 4) k_curvelets(CurveletArgs a) {
    extern __shared__ __align__(16) unsigned char cv_smem[];
    const Model &md = a.md;
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int wpb = blockDim.x >> 5;
    const int gwarp = blockIdx.x * wpb + wib;
    const int nwarps = gridDim.x * wpb;

    double *cell_dx2 = (double *)cv_smem;
    unsigned char *cell_j = cv_smem + CELLS_MAX * 8;
    unsigned short *cell_rank = (unsigned short *)(cv_smem + CELLS_MAX * 9);
    cell_tables_init(md, cell_dx2, cell_j, cell_rank);
    __syncthreads();

    const WarpLayout W = curvelet_warp_layout(md.max_cand, a.slots, md.gms, CPL, md.Q);
    unsigned char *base = cv_smem + CELL_TABLE_BYTES + (size_t)wib * W.total;
    double *sT = (double *)(base + W.sT);
    double *cT = (double *)(base + W.cT);
    double *T2t = (double *)(base + W.T2t);
    double *geo = (double *)(base + W.geo);
    int *gflag = (int *)(base + W.gflag);
    double *tab = (double *)(base + W.tab);
    int *ck = (int *)(base + W.ck);
    int *nb_idx = (int *)(base + W.nb_idx);
    int *nb_orig = (int *)(base + W.nb_orig);
    int *seed_orig = (int *)(base + W.seed_orig);
    unsigned char *nb_cls = base + W.nb_cls;
    unsigned short *chain_sm = (unsigned short *)(base + W.chain);
    double *bund_sm = (double *)(base + W.bund);
    double *bund_gl = a.scratch + (size_t)gwarp * (size_t)a.scratch_slots * 2 * 32 * CPL;
    unsigned short *chain_gl = a.scratch_chain + (size_t)gwarp * (size_t)a.scratch_slots * md.gms;

    constexpr int BW = 2 * 32 * CPL;  // doubles per bundle slot: mins then maxes, cell c at index c
    const int TP = 2 * md.Q;          // staged sin values per pair
    const int cells = md.cells;

    // this lane's cells for the growth phase: c = lane + 32u
    unsigned rank_l[CPL];
    bool on_l[CPL];
#pragma unroll
    for (int u = 0; u < CPL; ++u) {
        const int c = lane + 32 * u;
        on_l[u] = c < cells;
        rank_l[u] = on_l[u] ? (unsigned)cell_rank[c] : 0xffffu;
    }

    auto slot_ptr = [&](int s) -> double * {
        return (s < a.slots) ? bund_sm + (size_t)s * BW : bund_gl + (size_t)(s - a.slots) * BW;
    };
    auto chain_ptr = [&](int s) -> unsigned short * {
        return (s < a.slots) ? chain_sm + (size_t)s * md.gms : chain_gl + (size_t)(s - a.slots) * md.gms;
    };

    for (int i = gwarp; i < a.N; i += nwarps) {
        const int m = a.B.map[i];
        const int orig = a.B.orig[i];
        const double ax = a.B.x[i], ay = a.B.y[i], T2 = a.B.th[i];
        const unsigned long long off = a.pair_off[i];
        const int deg = (int)(a.pair_off[i + 1] - off);

        // anchor trig: sin/cos(T2 + delta_t2_j) (:702-705), cos/sin(T2) (:690 and dot)
        if (lane < md.Q) {
            const double delta_t2 = md.st * ((double)lane - ((double)md.Q - 1.0) / 2.0);
            const double t = T2 + delta_t2;
            T2t[lane] = t;
            sT[lane] = sin(t);
            cT[lane] = cos(t);
        }
        const double cosT2 = cos(T2);
        const double sinT2 = sin(T2);

        // 1. neighbour classes
        for (int k = lane; k < deg; k += 32) {
            const int n = a.csr_ids[off + k];
            nb_idx[k] = n;
            nb_orig[k] = a.B.orig[n];
            const double lx = a.B.x[n], ly = a.B.y[n];
            const double dir = to_2pi(atan2(ly - ay, lx - ax));   // angle_from_pt_to_pt(te, le)
            const double d = cos(dir) * cosT2 + sin(dir) * sinT2;  // dot(dir, te_orient)
            const unsigned run = (d > 0) ? 0u : ((d < 0) ? 1u : 2u);
            const double DX = ax - lx, DY = ay - ly;
            const bool close = (DX * DX + DY * DY < md.four_dx_dx);
            nb_cls[k] = (unsigned char)(run | (close ? 4u : 0u));
        }
        __syncwarp();

        unsigned n_out = 0;
        unsigned valid_cnt = 0;

        for (int f = 0; f < 2; ++f) {
            int ns = 0;  // this run's seeds, in slots 0..ns-1

            // 2. bundles of the chunk's pairs ck[0..nck) into tentative slots ns..ns+nck-1
            auto process_chunk = [&](int nck) {
                // 2a. staged trig and geometry
                for (int t = lane; t < nck * TP; t += 32) {
                    const int pb = t / TP, q = t - pb * TP;
                    const double T0 = a.B.th[nb_idx[ck[pb]]];
                    const int jj = (q < md.Q) ? q : q - md.Q;
                    const double arg = (q < md.Q) ? (T2t[jj] - (T0 - md.dt)) : (T2t[jj] - (T0 + md.dt));
                    tab[t] = sin(arg);  // sin(T2t - T0_m_dt), sin(T2t - T0_p_dt) (:728-729)
                }
                if (lane < nck) {
                    const int n = nb_idx[ck[lane]];
                    const PairGeom g = pair_geom(md, ax, ay, cosT2, sinT2, a.B.x[n], a.B.y[n], a.B.sp[n], a.B.cp[n],
                                                 a.B.sm[n], a.B.cm[n]);
                    double *gg = geo + lane * GEO_N;
                    gg[0] = g.DX;
                    gg[1] = g.DY;
                    gg[2] = g.DX2;
                    gg[3] = g.DY2;
                    gg[4] = g.sin_p_DY;
                    gg[5] = g.cos_p_DX;
                    gg[6] = g.sin_m_DY;
                    gg[7] = g.cos_m_DX;
                    gflag[lane] = (g.close ? 1 : 0) | (g.branch1 ? 2 : 0);
                }
                __syncwarp();
                // 2b. one task per (pair, cell)
                {
                    int pb = 0, c = lane;
                    while (c >= cells) {
                        c -= cells;
                        ++pb;
                    }
                    for (; pb < nck;) {
                        const double *gg = geo + pb * GEO_N;
                        const int fl = gflag[pb];
                        double bmin = -md.max_k, bmax = md.max_k;
                        if (!(fl & 1)) {
                            const int jj = cell_j[c];
                            bundle_cell(md, gg[0], gg[1], gg[2], gg[3], gg[4], gg[5], gg[6], gg[7], (fl & 2) != 0,
                                        cell_dx2[c], sT[jj], cT[jj], tab[pb * TP + jj], tab[pb * TP + md.Q + jj],
                                        bmin, bmax);
                        }
                        double *dst = slot_ptr(ns + pb);
                        dst[c] = bmin;
                        dst[32 * CPL + c] = bmax;
                        c += 32;
                        while (c >= cells) {
                            c -= cells;
                            ++pb;
                        }
                    }
                }
                __syncwarp();
                // 2c. validity (:821-830), seed compaction, valid_pairs (:346-350)
                const int ns0 = ns;
                for (int pb = 0; pb < nck; ++pb) {
                    const int k = ck[pb];
                    const unsigned cls = nb_cls[k];
                    const double *src = slot_ptr(ns0 + pb);
                    bool lv = false;
#pragma unroll
                    for (int u = 0; u < CPL; ++u) {
                        const int c = lane + 32 * u;
                        if (c < cells) lv = lv || (src[32 * CPL + c] > src[c]);
                    }
                    const bool valid = (cls & 4u) ? true : (bool)__any_sync(FULL, lv);
                    if (!valid) continue;
                    ++valid_cnt;
                    if ((cls & 3u) != (unsigned)f || a.count_only) continue;
                    if (ns != ns0 + pb) {
                        double *dst = slot_ptr(ns);
#pragma unroll
                        for (int v = 0; v < 2 * CPL; ++v) dst[lane + 32 * v] = src[lane + 32 * v];
                    }
                    if (lane == 0) seed_orig[ns] = nb_orig[k];
                    ++ns;
                    __syncwarp();
                }
                __syncwarp();
            };

            int nck = 0;
            for (int k0 = 0; k0 < deg; k0 += 32) {
                const int k = k0 + lane;
                bool take = false;
                if (k < deg) {
                    const unsigned run = nb_cls[k] & 3u;
                    take = (run == (unsigned)f) || (f == 0 && run == 2u);
                }
                unsigned bal = __ballot_sync(FULL, take);
                while (bal) {
                    const int b = __ffs(bal) - 1;
                    bal &= bal - 1;
                    if (lane == 0) ck[nck] = k0 + b;
                    ++nck;
                    if (nck == PCH) {
                        if (ns + PCH > a.slots + a.scratch_slots) {  // cannot happen when sized by max_deg
                            if (lane == 0) atomicOr(a.err, ERR_CAPACITY);
                            nck = 0;
                            continue;
                        }
                        __syncwarp();
                        process_chunk(nck);
                        nck = 0;
                    }
                }
            }
            if (nck > 0) {
                if (ns + nck > a.slots + a.scratch_slots) {
                    if (lane == 0) atomicOr(a.err, ERR_CAPACITY);
                } else {
                    __syncwarp();
                    process_chunk(nck);
                }
            }

            // With group_max_sz <= 2 a chain stops at length 2 and the len > 2 gate
            // (:549) never passes: no growth needed (and no chain slot is written).
            if (a.count_only || ns == 0 || md.gms <= 2) continue;

            // 3. chain growth: groups of K seeds walk the seed list in lock step
            for (int g0 = 0; g0 < ns; g0 += K) {
                double cmin[K][CPL], cmax[K][CPL];
                unsigned len[K];
                unsigned done = 0;
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    const int s = g0 + q;
                    if (s < ns) {
                        const double *src = slot_ptr(s);
#pragma unroll
                        for (int u = 0; u < CPL; ++u) {
                            cmin[q][u] = src[lane + 32 * u];
                            cmax[q][u] = src[32 * CPL + lane + 32 * u];
                        }
                        len[q] = 1;  // the anchor (:485)
                        if (lane == 0) chain_ptr(s)[0] = 0xffffu;
                    } else {
                        len[q] = 0;
                        done |= 1u << q;
#pragma unroll
                        for (int u = 0; u < CPL; ++u) cmin[q][u] = cmax[q][u] = 0.0;
                    }
                }
                for (int r = 0; r < ns && done != (1u << K) - 1u; ++r) {
                    const double *src = slot_ptr(r);
                    double rmin[CPL], rmax[CPL];
#pragma unroll
                    for (int u = 0; u < CPL; ++u) {
                        rmin[u] = src[lane + 32 * u];
                        rmax[u] = src[32 * CPL + lane + 32 * u];
                    }
                    unsigned bits = 0;
#pragma unroll
                    for (int q = 0; q < K; ++q) {
                        bool lv = false;
#pragma unroll
                        for (int u = 0; u < CPL; ++u) {
                            // bundle_intersection (:832-843)
                            const double lo = (cmin[q][u] < rmin[u]) ? rmin[u] : cmin[q][u];
                            const double hi = (cmax[q][u] > rmax[u]) ? rmax[u] : cmax[q][u];
                            lv = lv || (on_l[u] && hi > lo);
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
                            if (lane == 0) chain_ptr(s)[len[q]] = (unsigned short)r;
                            ++len[q];
                            if (len[q] >= (unsigned)md.gms) done |= 1u << q;
                            continue;
                        }
                        if (bits & (1u << q)) {
                            if (lane == 0) chain_ptr(s)[len[q]] = (unsigned short)r;
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
                // 4. dedup (first identical chain in seed order wins, :876-916) + record
#pragma unroll
                for (int q = 0; q < K; ++q) {
                    const int s = g0 + q;
                    if (s >= ns || len[q] <= 2u) continue;  // len > 2 gate (:549)
                    unsigned short *my = chain_ptr(s);
                    if (lane == 0) my[0] = (unsigned short)(len[q] | 0x8000u);  // length tag in slot 0
                    __syncwarp();
                    bool dup = false;
                    for (int p = lane; p < s; p += 32) {
                        const unsigned short *cp = chain_ptr(p);
                        if (cp[0] == my[0]) {
                            bool same = true;
                            for (unsigned z = 1; z < len[q]; ++z) same = same && (cp[z] == my[z]);
                            dup = dup || same;
                        }
                    }
                    if (__any_sync(FULL, dup)) continue;
                    // best cell of the final bundle: smallest rank among open cells;
                    // none -> cell 0 (mini = minj = 0, :202-204)
                    unsigned best = 0xffffu;
#pragma unroll
                    for (int u = 0; u < CPL; ++u)
                        if (on_l[u] && cmax[q][u] > cmin[q][u] && rank_l[u] < best) best = rank_l[u];
                    best = __reduce_min_sync(FULL, best);
                    int mycell = -1;
                    double mymax = 0.0, mymin = 0.0;
#pragma unroll
                    for (int u = 0; u < CPL; ++u) {
                        const bool hit = (best != 0xffffu)
                                             ? (on_l[u] && rank_l[u] == best && cmax[q][u] > cmin[q][u])
                                             : (lane + 32 * u == 0);
                        if (hit) {
                            mycell = lane + 32 * u;
                            mymax = cmax[q][u];
                            mymin = cmin[q][u];
                        }
                    }
                    const unsigned who = __ballot_sync(FULL, mycell >= 0);
                    const int srcl = who ? (__ffs(who) - 1) : 0;
                    const int bcell = __shfl_sync(FULL, mycell, srcl);
                    const double kmax = __shfl_sync(FULL, mymax, srcl);
                    const double kmin = __shfl_sync(FULL, mymin, srcl);
                    const unsigned long long slot = off + n_out;
                    if ((unsigned)lane < len[q]) {
                        a.rec.ids[slot * (unsigned long long)md.gms + lane] =
                            (lane == 0) ? (unsigned)orig : (unsigned)seed_orig[my[lane]];
                    }
                    if (lane == 0) {
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
__global__ void __launch_bounds__(128) k_pair_bundles(Model md, const double *__restrict__ pairs, int n,
                                                      double *__restrict__ bmin_out, double *__restrict__ bmax_out,
                                                      unsigned char *__restrict__ valid_out) {
    __shared__ double tab[4][4 * QMAX];
    __shared__ double cell_dx2[CELLS_MAX];
    __shared__ unsigned char cell_j[CELLS_MAX];
    __shared__ unsigned short cell_rank[CELLS_MAX];
    cell_tables_init(md, cell_dx2, cell_j, cell_rank);
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *sT = tab[wib], *cT = sT + QMAX, *sM = cT + QMAX, *sP = sM + QMAX;
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
        bool lv = false;
        for (int c = lane; c < md.cells; c += 32) {
            double bmin = -md.max_k, bmax = md.max_k;
            if (!g.close) {
                const int jj = cell_j[c];
                bundle_cell(md, g.DX, g.DY, g.DX2, g.DY2, g.sin_p_DY, g.cos_p_DX, g.sin_m_DY, g.cos_m_DX, g.branch1,
                            cell_dx2[c], sT[jj], cT[jj], sM[jj], sP[jj], bmin, bmax);
            }
            lv = lv || (bmax > bmin);
            bmin_out[(size_t)p * md.cells + c] = bmin;
            bmax_out[(size_t)p * md.cells + c] = bmax;
        }
        const bool valid = g.close ? true : (bool)__any_sync(FULL, lv);
        if (lane == 0) valid_out[p] = valid ? 1 : 0;
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// Utility kernels
// ---------------------------------------------------------------------------
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
