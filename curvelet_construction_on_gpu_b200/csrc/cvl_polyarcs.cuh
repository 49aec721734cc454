// cvl_polyarcs.cuh -- C^1 polyarcs along the contour fragments, as the reference's
// original_code fits them after the one-chains:
//   fit_polyarcs_to_all_edgel_chains / fit_polyarc_to_chain
//       (original_code/form_curvelet_process.cpp:661-796)
//   form_a_hypothesis (leading, forward: :388-444), CC_curve_model_3d's bundle,
//   intersection, compute_best_fit, update_best_fit (CC_curve_model_3d.cpp)
//   curvelet::compute_properties / update_length (curvelet.cpp:80-169)
//   polyarcmap::compute_best_fit_according_to_curvelets (polyarcmap.hpp:98-111)
//
// A warp per fragment, the bundle's cells across the lanes (CPL per lane), the
// fragment walked in order as fit_polyarc_to_chain walks it:
//   - from edge i, a polyarc starts when the next edge lies ahead of it (dot > 0)
//     and their bundle is valid; it grows over the following edges while each
//     one's bundle with the start edge is valid and the running intersection
//     stays valid; the next polyarc starts at its last edge;
//   - its best cell is the open cell of smallest rank (the rank table gives
//     compute_best_fit's order: nearest the grid centre, first in row-major order);
//   - the fit: a line or the circle through the start, middle and end edges, on
//     lane 0, with the reference's operand order (the library builds with
//     -fmad=false).
// compute_best_fit_according_to_curvelets runs at the end of every fragment over
// all polyarcs so far, so a polyarc fitted as an arc with |k| < k_th becomes a
// line at its next refit, keeping its centre, angle and length; every other fit
// repeats itself. A polyarc of any fragment but the last is refitted.
#pragma once

namespace cvl {

constexpr double POLY_K_TH = 1e-4;  // k_th, original_code/curvelet_utils.hpp:15

struct PolyArgs {
    Model md;                      // dx, dt, max_k; grid steps 0.1 px, 0.08 rad (CC_curve_model_3d.hpp:20-23)
    const double *edges;           // AoS [n][sz]
    int sz;
    int nfrags;
    const long long *frag_off;     // [nfrags + 1]
    const int *frag_ids;           // 0-based edge ids
    double rad, token_len;         // compute_properties' R and token_len
    long long *poly_start;         // [slots]: index into frag_ids of the polyarc's first edge
    int *poly_size;                // [slots]
    double *poly_info;             // [slots][12]
    unsigned *poly_count;          // [nfrags]
};

// The polyarc slots of fragment f start at frag_off[f] - f: a fragment of N edges
// gives at most N - 1 polyarcs (each spans at least two edges and the next one
// starts no earlier than the last edge of the one before).
template <int CPL>
__global__ void __launch_bounds__(128) k_polyarcs(PolyArgs a) {
    __shared__ double tab[4][4 * QMAX];
    __shared__ double cell_dx2[CELLS_MAX];
    __shared__ unsigned char cell_j[CELLS_MAX];
    __shared__ unsigned short cell_rank[CELLS_MAX];
    const Model &md = a.md;
    cell_tables_init(md, cell_dx2, cell_j, cell_rank);
    __syncthreads();
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    double *sT = tab[wib], *cT = sT + QMAX, *sM = cT + QMAX, *sP = sM + QMAX;
    bool on[CPL];
    int cj[CPL];
    double cdx2[CPL];
    unsigned rk[CPL];
#pragma unroll
    for (int u = 0; u < CPL; ++u) {
        const int c = lane + 32 * u;
        on[u] = c < md.cells;
        cj[u] = on[u] ? cell_j[c] : 0;
        cdx2[u] = on[u] ? cell_dx2[c] : 0.0;
        rk[u] = on[u] ? cell_rank[c] : 0xffffu;
    }
    for (int f = blockIdx.x * 4 + wib; f < a.nfrags; f += gridDim.x * 4) {
        const int *ids = a.frag_ids + a.frag_off[f];
        const int N = (int)(a.frag_off[f + 1] - a.frag_off[f]);
        const long long slot0 = a.frag_off[f] - f;
        unsigned count = 0;
        int i = 0;
        while (i < N - 1) {
            const int iA = i, ia = ids[i];
            ++i;
            const double *A = a.edges + (size_t)ia * a.sz;
            const double ax = A[0], ay = A[1], T2 = A[2];
            const double cosT2 = cvl_cos(T2), sinT2 = cvl_sin(T2);
            __syncwarp();  // the previous start's tables are read
            for (int j = lane; j < md.Q; j += 32) {
                const double t = T2 + grid_offset(md.st, j, md.Q);  // T2t = T2 + Dt(j)
                sT[j] = cvl_sin(t);
                cT[j] = cvl_cos(t);
            }
            // form_a_hypothesis(A, B) and its bundle: false when there is no model
            // (B not ahead of A) or the bundle is empty
            auto hypothesis = [&](int ib, double *bmin, double *bmax) -> bool {
                const double *B = a.edges + (size_t)ib * a.sz;
                const double bx = B[0], by = B[1], T0 = B[2];
                // dot(vPointPoint(A, B), A's orientation) > 0: B ahead of A
                if (direction_class(ax, ay, bx, by, cosT2, sinT2) != 0u) return false;
                __syncwarp();  // sM / sP of the previous pair are read
                for (int j = lane; j < md.Q; j += 32) {
                    const double t = T2 + grid_offset(md.st, j, md.Q);
                    sM[j] = cvl_sin(t - (T0 - md.dt));
                    sP[j] = cvl_sin(t - (T0 + md.dt));
                }
                __syncwarp();
                const double t_p = T0 + md.dt, t_m = T0 - md.dt;
                const PairGeom g = pair_geom(md, ax, ay, cosT2, sinT2, bx, by, cvl_sin(t_p), cvl_cos(t_p),
                                             cvl_sin(t_m), cvl_cos(t_m));
                bool lv = false;
#pragma unroll
                for (int u = 0; u < CPL; ++u) {
                    bmin[u] = -md.max_k;
                    bmax[u] = md.max_k;
                    if (on[u] && !g.close) {
                        const double tt = sT[cj[u]] * g.DX - cT[cj[u]] * g.DY;
                        bundle_cell_tt(md, g.DX2, g.DY2, g.sin_p_DY, g.cos_p_DX, g.sin_m_DY, g.cos_m_DX, g.branch1,
                                       cdx2[u], tt, sM[cj[u]], sP[cj[u]], bmin[u], bmax[u]);
                    }
                    lv = lv || (on[u] && bmax[u] > bmin[u]);
                }
                return g.close || __any_sync(FULL, lv);
            };
            double cmin[CPL], cmax[CPL];
            if (!hypothesis(ids[i], cmin, cmax)) continue;
            int j = i;
            while (j < N - 1) {
                double rmin[CPL], rmax[CPL];
                if (!hypothesis(ids[j + 1], rmin, rmax)) break;
                // CC_curve_model_3d(cm1, cm2): Kmin = std::max, Kmax = std::min
                bool lv = false;
#pragma unroll
                for (int u = 0; u < CPL; ++u) {
                    rmin[u] = (cmin[u] < rmin[u]) ? rmin[u] : cmin[u];
                    rmax[u] = (rmax[u] < cmax[u]) ? rmax[u] : cmax[u];
                    lv = lv || (on[u] && rmax[u] > rmin[u]);
                }
                if (!__any_sync(FULL, lv)) break;
#pragma unroll
                for (int u = 0; u < CPL; ++u) {
                    cmin[u] = rmin[u];
                    cmax[u] = rmax[u];
                }
                ++j;
            }
            // compute_best_fit: the open cell of smallest rank
            unsigned best = 0xffffu;
#pragma unroll
            for (int u = 0; u < CPL; ++u)
                if (on[u] && cmax[u] > cmin[u] && rk[u] < best) best = rk[u];
            best = __reduce_min_sync(FULL, best);
            double mymax = 0.0, mymin = 0.0;
            bool mine = false;
#pragma unroll
            for (int u = 0; u < CPL; ++u)
                if (on[u] && rk[u] == best && cmax[u] > cmin[u]) {
                    mine = true;
                    mymax = cmax[u];
                    mymin = cmin[u];
                }
            const unsigned who = __ballot_sync(FULL, mine);
            const int src = who ? __ffs(who) - 1 : 0;
            const double kmax = __shfl_sync(FULL, mymax, src);
            const double kmin = __shfl_sync(FULL, mymin, src);
            if (lane == 0) {
                const int size = j - iA + 1;
                double k = (kmax + kmin) / 2;  // set_best_fit's _k
                // curvelet::compute_properties: every step counts (the anchor is the front)
                double L = 0;
                for (int q = iA; q < j; ++q) {
                    const double *P0 = a.edges + (size_t)ids[q] * a.sz, *P1q = a.edges + (size_t)ids[q + 1] * a.sz;
                    L += sqrt((P0[0] - P1q[0]) * (P0[0] - P1q[0]) + (P0[1] - P1q[1]) * (P0[1] - P1q[1]));
                }
                const double quality = 2 / (1.0 * a.rad / L + 1.0 * L / a.token_len / size);
                // update_best_fit(middle, end) with _pt = the start edge
                const double *P1 = a.edges + (size_t)ids[iA + size / 2] * a.sz;
                const double *P2 = a.edges + (size_t)ids[j] * a.sz;
                double theta, angle = 0.0, cx = 0.0, cy = 0.0;
                bool arc = false;
                if (fabs(k) < POLY_K_TH) {
                    k = 0.0;
                    theta = cvl_atan2(P2[1] - ay, P2[0] - ax);
                } else {
                    const double d1 = ax * ax + ay * ay, d2 = P1[0] * P1[0] + P1[1] * P1[1],
                                 d3 = P2[0] * P2[0] + P2[1] * P2[1];
                    const double a11 = 2.0 * (ax - P1[0]), a12 = 2.0 * (ay - P1[1]), a21 = 2.0 * (P2[0] - P1[0]),
                                 a22 = 2.0 * (P2[1] - P1[1]);
                    const double b1 = d1 - d2, b2 = d3 - d2;
                    const double det = a11 * a22 - a21 * a12;
                    if (fabs(det) < POLY_K_TH) {
                        k = 0.0;
                        theta = cvl_atan2(P2[1] - ay, P2[0] - ax);
                    } else {
                        cx = (b1 * a22 - b2 * a12) / det;
                        cy = (b2 * a11 - b1 * a21) / det;
                        const double v1x = ax - cx, v1y = ay - cy, v2x = P2[0] - cx, v2y = P2[1] - cy;
                        const double c = v1x * v2y - v1y * v2x, d = v1x * v2x + v1y * v2y;
                        angle = cvl_atan2(fabs(c), d);
                        theta = cvl_atan2(c * v1x, -c * v1y);
                        k = 1.0 / sqrt(v2x * v2x + v2y * v2y);
                        arc = true;
                    }
                }
                if (fabs(angle) > 0 && fabs(k) > POLY_K_TH && arc) L = angle / fabs(k);  // update_length
                if (arc && fabs(k) < POLY_K_TH && f < a.nfrags - 1) {  // the refit of a later fragment
                    k = 0.0;
                    theta = cvl_atan2(P2[1] - ay, P2[0] - ax);
                }
                const long long s = slot0 + count;
                a.poly_start[s] = a.frag_off[f] + iA;
                a.poly_size[s] = size;
                double *row = a.poly_info + (size_t)s * 12;
                row[0] = 1.0;   // forward
                row[1] = kmax;  // _ref_pt after compute_best_fit: the best cell's k range
                row[2] = kmin;
                row[3] = T2;    // _ref_theta
                row[4] = ax;    // _pt: the start edge
                row[5] = ay;
                row[6] = theta;
                row[7] = k;
                row[8] = L;
                row[9] = quality;
                row[10] = arc ? cx : 0.0;
                row[11] = arc ? cy : 0.0;
            }
            ++count;
            i = j;
        }
        if (lane == 0) a.poly_count[f] = count;
    }
}

// polyarcs of all fragments packed in order (fragment, then start)
__global__ void k_polyarcs_pack(int nfrags, const long long *__restrict__ frag_off,
                                const unsigned *__restrict__ poly_count, const unsigned long long *__restrict__ poly_off,
                                const long long *__restrict__ start_in, const int *__restrict__ size_in,
                                const double *__restrict__ info_in, long long *__restrict__ start_out,
                                int *__restrict__ size_out, double *__restrict__ info_out) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nfrags) return;
    const long long s0 = frag_off[f] - f;
    const unsigned long long d0 = poly_off[f];
    for (unsigned q = 0; q < poly_count[f]; ++q) {
        start_out[d0 + q] = start_in[s0 + q];
        size_out[d0 + q] = size_in[s0 + q];
        for (int c = 0; c < 12; ++c) info_out[(d0 + q) * 12 + c] = info_in[(s0 + q) * 12 + c];
    }
}

}  // namespace cvl
