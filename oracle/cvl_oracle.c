/* cvl_oracle.c -- TEST INFRASTRUCTURE ONLY: a plain-C restatement of the
 * reference cpu_curvelet path (preprocess -> pairwise curve bundles -> greedy
 * chain growth, dedup, record), used as the CPU checker for the CUDA engine.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * legs load this library. The product (libcvl.so) never links or calls it.
 *
 * Pinning: tests/test_oracle_pinned.py checks this restatement bit for bit
 * against the reference's own code (oracle/ref_harness.cpp built from
 * cpu_curvelet headers) on the reference's sample edge files and on seeded
 * synthetic maps, and against the committed fixtures in tests/golden/.
 *
 * Arithmetic: FP64 throughout, glibc libm (sin, cos, atan2, fmod, sqrt, lrint),
 * the reference's operation order, and no FMA contraction (oracle/Makefile
 * passes -ffp-contract=off; the reference itself is built without -march, so
 * on x86-64 it has no FMA either).
 *
 * Citations are path:line within the reference project.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846 /* curvelet_utils.hpp:10 */

/* ---------------------------------------------------------------------- */
/* Math helpers: curvelet_utils.hpp:13-69                                  */
/* ---------------------------------------------------------------------- */

/* sq_dist, curvelet_utils.hpp:13-17 */
static double orc_sq_dist(double x1, double y1, double x2, double y2)
{
    return (x1 - x2) * (x1 - x2) + (y1 - y2) * (y1 - y2);
}

/* To2Pi, curvelet_utils.hpp:25-46 */
static double orc_to_2pi(double angle)
{
    double a;
    if (angle >= 2.0 * ORC_PI)
        a = fmod(angle, 2.0 * ORC_PI);
    else if (angle < 0)
        a = (2.0 * ORC_PI + fmod(angle, 2.0 * ORC_PI));
    else
        a = angle;
    if (!(a >= 0 && a < 2.0 * ORC_PI))
        a = 0;
    return a;
}

/* angle_from_pt_to_pt, curvelet_utils.hpp:58-62 */
static double orc_angle_pt_pt(double x1, double y1, double x2, double y2)
{
    return orc_to_2pi(atan2(y2 - y1, x2 - x1));
}

/* dot, curvelet_utils.hpp:65-69 */
static double orc_dot(double v1, double v2)
{
    return cos(v1) * cos(v2) + sin(v1) * sin(v2);
}

/* ---------------------------------------------------------------------- */
/* Neighbour graph: preprocess.hpp:41-274                                  */
/* ---------------------------------------------------------------------- */

typedef struct {
    int64_t key; /* pack_cell_key, preprocess.hpp:41-45 */
    int id;
} orc_cell_ent;

static int orc_cmp_cell_ent(const void *a, const void *b)
{
    const orc_cell_ent *x = (const orc_cell_ent *)a, *y = (const orc_cell_ent *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    return (x->id > y->id) - (x->id < y->id); /* within-cell order: edge index */
}

typedef struct {
    double d2;
    int scan; /* position in the window scan (py outer, px inner, cell order) */
    int id;
} orc_cand;

static int orc_cmp_cand(const void *a, const void *b)
{
    const orc_cand *x = (const orc_cand *)a, *y = (const orc_cand *)b;
    if (x->d2 < y->d2) return -1;
    if (x->d2 > y->d2) return 1;
    return (x->scan > y->scan) - (x->scan < y->scan);
}

static int64_t orc_pack_key(int x, int y)
{
    return (int64_t)(((uint64_t)(int64_t)y << 32) | (uint64_t)(uint32_t)x);
}

static int orc_lower_bound(const int64_t *keys, int n, int64_t key)
{
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = lo + ((hi - lo) >> 1);
        if (keys[mid] < key) lo = mid + 1; else hi = mid;
    }
    return lo;
}

typedef struct {
    int num_edges;
    int total_neighbor_pairs;
    unsigned max_num_of_neighbors;
    unsigned truncated_anchors; /* anchors whose list reached max_candidates (preprocess.hpp:224) */
    unsigned tie_anchors;       /* anchors with an exact dist^2 tie inside their kept list */
    int *neighbor_offsets;      /* [num_edges + 1] */
    int *neighbor_ids;          /* [total_neighbor_pairs] */
    double *neighbor_dist2;     /* [total_neighbor_pairs] */
} orc_csr;

void orc_csr_free(orc_csr *g)
{
    free(g->neighbor_offsets);
    free(g->neighbor_ids);
    free(g->neighbor_dist2);
    memset(g, 0, sizeof(*g));
}

/* build_neighbor_csr_graph + build_spatial_index_cpu + discover_neighbors_csr,
 * preprocess.hpp:62-274. Candidates are the edges whose pixel cell
 * (lrint(x), lrint(y)) lies in the (2w+1)^2 window around the anchor's cell and
 * whose squared distance is <= rad^2 (preprocess.hpp:141-163); the first
 * max_candidates in window-scan order are kept (:165-167), then sorted by
 * squared distance (:172-176). Where the reference's std::sort leaves the order
 * of equal keys to libstdc++, this restatement uses edge index (within a cell)
 * and scan position (within equal distances); tie_anchors counts the anchors
 * where the latter could matter. Returns 0 on success, -1 on invalid input
 * (preprocess.hpp:197-199). */
int orc_build_csr(const double *edges, int num_edges, int sz, double rad, unsigned neighbor_radius,
                  unsigned max_candidates, int nthreads, orc_csr *g)
{
    memset(g, 0, sizeof(*g));
    if (num_edges <= 0 || sz < 4 || edges == NULL) return -1;
    (void)nthreads;

    orc_cell_ent *ent = (orc_cell_ent *)malloc(sizeof(orc_cell_ent) * (size_t)num_edges);
    for (int i = 0; i < num_edges; ++i) {
        const int cx = (int)lrint(edges[(size_t)i * sz + 0]);
        const int cy = (int)lrint(edges[(size_t)i * sz + 1]);
        ent[i].key = orc_pack_key(cx, cy);
        ent[i].id = i;
    }
    qsort(ent, (size_t)num_edges, sizeof(orc_cell_ent), orc_cmp_cell_ent);

    /* run-length unique cells, preprocess.hpp:99-111 */
    int64_t *ukeys = (int64_t *)malloc(sizeof(int64_t) * (size_t)num_edges);
    int *ustart = (int *)malloc(sizeof(int) * (size_t)num_edges);
    int *ucount = (int *)malloc(sizeof(int) * (size_t)num_edges);
    int ncell = 0;
    for (int p = 0; p < num_edges;) {
        const int64_t key = ent[p].key;
        const int start = p;
        while (p < num_edges && ent[p].key == key) ++p;
        ukeys[ncell] = key;
        ustart[ncell] = start;
        ucount[ncell] = p - start;
        ++ncell;
    }

    const double rad_sqr = rad * rad;
    const int w = (int)neighbor_radius;
    int *deg = (int *)calloc((size_t)num_edges, sizeof(int));
    int **st_ids = (int **)calloc((size_t)num_edges, sizeof(int *));
    double **st_d2 = (double **)calloc((size_t)num_edges, sizeof(double *));
    unsigned truncated = 0, ties = 0;

#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : truncated, ties) num_threads(nthreads > 0 ? nthreads : 1)
#endif
    for (int te = 0; te < num_edges; ++te) {
        const double tx = edges[(size_t)te * sz + 0];
        const double ty = edges[(size_t)te * sz + 1];
        const int cx = (int)lrint(tx);
        const int cy = (int)lrint(ty);
        size_t cap = 64, n = 0;
        orc_cand *c = (orc_cand *)malloc(sizeof(orc_cand) * cap);
        int scan = 0;
        for (int py = cy - w; py <= cy + w; ++py) {
            for (int px = cx - w; px <= cx + w; ++px) {
                const int64_t key = orc_pack_key(px, py);
                const int ci = orc_lower_bound(ukeys, ncell, key);
                if (ci >= ncell || ukeys[ci] != key) continue;
                for (int k = ustart[ci]; k < ustart[ci] + ucount[ci]; ++k) {
                    const int ne = ent[k].id;
                    if (ne == te) continue;
                    const double d = orc_sq_dist(tx, ty, edges[(size_t)ne * sz + 0], edges[(size_t)ne * sz + 1]);
                    if (d > rad_sqr) continue;
                    if (n < (size_t)max_candidates) {
                        if (n == cap) {
                            cap *= 2;
                            c = (orc_cand *)realloc(c, sizeof(orc_cand) * cap);
                        }
                        c[n].d2 = d;
                        c[n].scan = scan;
                        c[n].id = ne;
                        ++n;
                    }
                    ++scan;
                }
            }
        }
        qsort(c, n, sizeof(orc_cand), orc_cmp_cand);
        for (size_t i = 1; i < n; ++i) {
            if (c[i].d2 == c[i - 1].d2) { ++ties; break; }
        }
        if (n >= (size_t)max_candidates) ++truncated;
        deg[te] = (int)n;
        st_ids[te] = (int *)malloc(sizeof(int) * (n ? n : 1));
        st_d2[te] = (double *)malloc(sizeof(double) * (n ? n : 1));
        for (size_t i = 0; i < n; ++i) { st_ids[te][i] = c[i].id; st_d2[te][i] = c[i].d2; }
        free(c);
    }

    g->num_edges = num_edges;
    g->neighbor_offsets = (int *)malloc(sizeof(int) * ((size_t)num_edges + 1));
    g->neighbor_offsets[0] = 0;
    unsigned maxdeg = 0;
    for (int te = 0; te < num_edges; ++te) {
        g->neighbor_offsets[te + 1] = g->neighbor_offsets[te] + deg[te];
        if ((unsigned)deg[te] > maxdeg) maxdeg = (unsigned)deg[te];
    }
    g->total_neighbor_pairs = g->neighbor_offsets[num_edges];
    g->max_num_of_neighbors = maxdeg;
    g->truncated_anchors = truncated;
    g->tie_anchors = ties;
    const size_t np = (size_t)g->total_neighbor_pairs;
    g->neighbor_ids = (int *)malloc(sizeof(int) * (np ? np : 1));
    g->neighbor_dist2 = (double *)malloc(sizeof(double) * (np ? np : 1));
    for (int te = 0; te < num_edges; ++te) {
        memcpy(g->neighbor_ids + g->neighbor_offsets[te], st_ids[te], sizeof(int) * (size_t)deg[te]);
        memcpy(g->neighbor_dist2 + g->neighbor_offsets[te], st_d2[te], sizeof(double) * (size_t)deg[te]);
        free(st_ids[te]);
        free(st_d2[te]);
    }
    free(st_ids); free(st_d2); free(deg);
    free(ukeys); free(ustart); free(ucount); free(ent);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Curve bundles: cpu_curvelet.hpp:636-830                                 */
/* ---------------------------------------------------------------------- */

typedef struct {
    double dx, dt, sx, st, max_k, nrad; /* dt in radians (main.cpp:24) */
    unsigned P, Q;                      /* bundle grid: pixel x theta (cpu_curvelet.hpp:73-74) */
    unsigned gms;                       /* group_max_sz */
} orc_model;

static void orc_model_init(orc_model *m, double nrad, double dx, double dt_deg, double max_k,
                           double sx, double st, unsigned gms)
{
    m->nrad = nrad;
    m->dx = dx;
    m->dt = (double)(dt_deg / 180.0) * (double)ORC_PI; /* main.cpp:24 */
    m->max_k = max_k;
    m->sx = sx;
    m->st = st;
    m->P = (unsigned)(2 * floor(dx / sx + 0.5) + 1); /* cpu_curvelet.hpp:73 */
    m->Q = (unsigned)(2 * floor(m->dt / st + 0.5) + 1); /* cpu_curvelet.hpp:74 */
    m->gms = gms;
}

/* compute_curve_bundle, cpu_curvelet.hpp:637-819 (Proposition 4: circular arc
 * bundle transport). bmin/bmax hold P*Q cells, pre-set to -max_k / +max_k by the
 * caller (cpu_curvelet.hpp:330-336, :577-583). Returns 1 when the bundle is
 * valid (close pair, or some cell with max > min). */
static int orc_curve_bundle(const orc_model *m, double te_x, double te_y, double le_x, double le_y,
                            double te_o, double le_o, double *bmin, double *bmax)
{
    const double DX = te_x - le_x;
    const double DY = te_y - le_y;
    const double DX2 = DX * DX;
    const double DY2 = DY * DY;
    const double T0 = le_o;
    const double T2 = te_o;
    const double _dx = m->dx;
    const double _dx2 = _dx * _dx;
    const double T0_p_dt = T0 + m->dt;
    const double T0_m_dt = T0 - m->dt;
    unsigned bk = 0;

    if (DX2 + DY2 < 4 * _dx * _dx) /* :682-687 */
        return 1;

    if ((DX * cos(T2) + DY * sin(T2)) < 0) { /* :690 */
        for (unsigned i = 0; i < m->P; i++) {
            for (unsigned j = 0; j < m->Q; j++) {
                const double delta_x2 = m->sx * ((double)i - ((double)m->P - 1.0) / 2.0);
                const double delta_t2 = m->st * ((double)j - ((double)m->Q - 1.0) / 2.0);
                const double T2t = T2 + delta_t2;
                const double tt = sin(T2t) * DX - cos(T2t) * DY;
                const double ttmdx2 = tt - delta_x2;
                const double eq_denom = (-2.0 * delta_x2 * tt + DX2 + DY2 - _dx2 + delta_x2 * delta_x2);
                const double k_dx_min = 2.0 * (ttmdx2 - _dx) / eq_denom;
                const double k_dx_max = 2.0 * (ttmdx2 + _dx) / eq_denom;
                if (bmin[bk] < k_dx_min) bmin[bk] = k_dx_min;
                if (bmax[bk] > k_dx_max) bmax[bk] = k_dx_max;
                const double s_m = sin(T2t - T0_m_dt);
                const double s_p = sin(T2t - T0_p_dt);
                const double sin_p_DY = DY * sin(T0_p_dt);
                const double cos_p_DX = DX * cos(T0_p_dt);
                const double sin_m_DY = DY * sin(T0_m_dt);
                const double cos_m_DX = DX * cos(T0_m_dt);
                const double k_dt_min = s_m / (-s_m * delta_x2 + cos_m_DX + sin_m_DY);
                const double k_dt_max = s_p / (-s_p * delta_x2 + cos_p_DX + sin_p_DY);
                if (bmin[bk] < k_dt_min) bmin[bk] = k_dt_min;
                if (bmax[bk] > k_dt_max) bmax[bk] = k_dt_max;
                bk++;
            }
        }
    } else { /* :756-810 */
        for (unsigned i = 0; i < m->P; i++) {
            for (unsigned j = 0; j < m->Q; j++) {
                const double delta_x2 = m->sx * ((double)i - ((double)m->P - 1.0) / 2.0);
                const double delta_t2 = m->st * ((double)j - ((double)m->Q - 1.0) / 2.0);
                const double T2t = T2 + delta_t2;
                const double tt = sin(T2t) * DX - cos(T2t) * DY;
                const double ttmdx2 = tt - delta_x2;
                const double eq_denom = -(2.0 * delta_x2 * tt - DX2 - DY2 + _dx2 - delta_x2 * delta_x2) / 2.0;
                const double k_dx_min = (ttmdx2 - _dx) / eq_denom;
                const double k_dx_max = (ttmdx2 + _dx) / eq_denom;
                if (bmin[bk] < k_dx_min) bmin[bk] = k_dx_min;
                if (bmax[bk] > k_dx_max) bmax[bk] = k_dx_max;
                const double s_m = sin(T2t - T0_m_dt);
                const double s_p = sin(T2t - T0_p_dt);
                const double sin_p_DY = DY * sin(T0_p_dt);
                const double cos_p_DX = DX * cos(T0_p_dt);
                const double sin_m_DY = DY * sin(T0_m_dt);
                const double cos_m_DX = DX * cos(T0_m_dt);
                const double k_dt_max = s_m / (-s_m * delta_x2 + cos_m_DX + sin_m_DY);
                if (bmax[bk] > k_dt_max) bmax[bk] = k_dt_max;
                const double k_dt_min = s_p / (-s_p * delta_x2 + cos_p_DX + sin_p_DY);
                if (bmin[bk] < k_dt_min) bmin[bk] = k_dt_min;
                bk++;
            }
        }
    }
    /* bundle_valid_check, :821-830 */
    for (unsigned c = 0; c < m->P * m->Q; ++c)
        if (bmax[c] > bmin[c]) return 1;
    return 0;
}

/* One pair's bundle with the grid pre-set to +-max_k. Returns validity. */
int orc_pair_bundle(double te_x, double te_y, double te_o, double le_x, double le_y, double le_o,
                    double nrad, double dx, double dt_deg, double max_k, double sx, double st,
                    double *bmin, double *bmax, int *ncells)
{
    orc_model m;
    orc_model_init(&m, nrad, dx, dt_deg, max_k, sx, st, 4);
    const unsigned cells = m.P * m.Q;
    for (unsigned c = 0; c < cells; ++c) { bmin[c] = -max_k; bmax[c] = max_k; }
    *ncells = (int)cells;
    return orc_curve_bundle(&m, te_x, te_y, le_x, le_y, te_o, le_o, bmin, bmax);
}

/* ---------------------------------------------------------------------- */
/* Greedy growth, dedup and record: cpu_curvelet.hpp:197-303, :363-634     */
/* ---------------------------------------------------------------------- */

typedef struct {
    int num_edges;
    int total_neighbor_pairs;
    unsigned max_num_of_neighbors;
    unsigned truncated_anchors;
    unsigned tie_anchors;
    unsigned valid_pairs;   /* form_pairwise_bundles count, cpu_curvelet.hpp:305-361 */
    unsigned num_curvelets;
    unsigned chain_width;   /* group_max_sz + 1 */
    unsigned *chains;       /* [num_curvelets * chain_width], 1-based ids, zero padded */
    double *info;           /* [num_curvelets * 10], row-major */
    unsigned *anchor_count; /* [num_edges] curvelets per anchor */
} orc_result;

void orc_result_free(orc_result *r)
{
    free(r->chains);
    free(r->info);
    free(r->anchor_count);
    memset(r, 0, sizeof(*r));
}

/* fill_curvelet_info, cpu_curvelet.hpp:197-256 (10 columns). */
static void orc_fill_info(const orc_model *m, const double *edges, int sz, int forward,
                          double ref_x, double ref_y, double ref_theta,
                          const double *cmin, const double *cmax, const unsigned *chain, unsigned chain_sz,
                          double *info)
{
    double mind = 100.0;
    unsigned mini = 0, minj = 0;
    for (unsigned ii = 0; ii < m->P; ii++) {
        for (unsigned jj = 0; jj < m->Q; jj++) {
            const unsigned b = ii * m->Q + jj;
            if (cmax[b] > cmin[b]) {
                const double ddx = m->sx * ((double)ii - ((double)m->P - 1.0) / 2.0);
                const double ddt = m->st * ((double)jj - ((double)m->Q - 1.0) / 2.0);
                const double d = ddx * ddx + ddt * ddt;
                if (d < mind) { mind = d; mini = ii; minj = jj; }
            }
        }
    }
    const unsigned best = mini * m->Q + minj;
    const double k_max = cmax[best];
    const double k_min = cmin[best];
    const double k = (k_max + k_min) / 2.0;
    const double dx = m->sx * ((double)mini - ((double)m->P - 1.0) / 2.0);
    const double dt = m->st * ((double)minj - ((double)m->Q - 1.0) / 2.0);
    const double theta = orc_to_2pi(ref_theta + dt);
    const double pt_x = ref_x - dx * sin(theta);
    const double pt_y = ref_y + dx * cos(theta);
    double length = 0.0;
    for (unsigned i = 0; i + 1 < chain_sz; i++) {
        const unsigned e1 = chain[i], e2 = chain[i + 1];
        length += sqrt(orc_sq_dist(edges[(size_t)e1 * sz + 0], edges[(size_t)e1 * sz + 1],
                                   edges[(size_t)e2 * sz + 0], edges[(size_t)e2 * sz + 1]));
    }
    const double quality = (length > 0.0 && chain_sz > 0)
                               ? 2.0 / (1.0 * m->nrad / length + 1.0 * length / (double)chain_sz)
                               : 0.0;
    info[0] = forward ? 1.0 : 0.0;
    info[1] = k_max;
    info[2] = k_min;
    info[3] = ref_theta;
    info[4] = pt_x;
    info[5] = pt_y;
    info[6] = theta;
    info[7] = k;
    info[8] = length;
    info[9] = quality;
}

/* All curvelets of one anchor, in the reference's record order (run 0 then
 * run 1, seeds in neighbour order). Writes at most deg rows into chains/info,
 * returns the count. Also accumulates the anchor's valid_pairs. */
static unsigned orc_anchor(const orc_model *m, const double *edges, int sz, const orc_csr *g, int te,
                           unsigned *chains, double *info, unsigned *valid_pairs_out, double *scratch)
{
    const unsigned cells = m->P * m->Q;
    const unsigned W = m->gms + 1;
    const int beg = g->neighbor_offsets[te];
    const unsigned deg = (unsigned)(g->neighbor_offsets[te + 1] - beg);
    const double tx = edges[(size_t)te * sz + 0], ty = edges[(size_t)te * sz + 1], to = edges[(size_t)te * sz + 2];
    double *bmin = scratch;                         /* [deg][cells] */
    double *bmax = bmin + (size_t)deg * cells;      /* [deg][cells] */
    double *cmin = bmax + (size_t)deg * cells;      /* [cells] running intersection */
    double *cmax = cmin + cells;
    double *imin = cmax + cells;
    double *imax = imin + cells;
    unsigned *accepted = (unsigned *)(imax + cells);         /* [deg + 1][W] */
    unsigned char *valid = (unsigned char *)(accepted + (size_t)(deg + 1) * W); /* [deg] */
    unsigned char *run = valid + deg;                        /* [deg]: 0 fwd, 1 bwd, 2 neither */
    unsigned n_out = 0, vp = 0;

    for (unsigned k = 0; k < deg; ++k) {
        const int ne = g->neighbor_ids[beg + k];
        const double lx = edges[(size_t)ne * sz + 0], ly = edges[(size_t)ne * sz + 1], lo = edges[(size_t)ne * sz + 2];
        double *mn = bmin + (size_t)k * cells, *mx = bmax + (size_t)k * cells;
        for (unsigned c = 0; c < cells; ++c) { mn[c] = -m->max_k; mx[c] = m->max_k; }
        valid[k] = (unsigned char)orc_curve_bundle(m, tx, ty, lx, ly, to, lo, mn, mx);
        vp += valid[k];
        /* direction filter, cpu_curvelet.hpp:459-461 */
        const double dir = orc_angle_pt_pt(tx, ty, lx, ly);
        const double d = orc_dot(dir, to);
        run[k] = (d > 0) ? 0 : ((d < 0) ? 1 : 2);
    }

    for (unsigned f = 0; f < 2; ++f) {
        unsigned n_acc = 0;
        for (unsigned s = 0; s < deg; ++s) {
            if (!(valid[s] && run[s] == f)) continue;
            unsigned chain[64];
            unsigned len = 0;
            chain[len++] = (unsigned)te;
            memcpy(cmin, bmin + (size_t)s * cells, sizeof(double) * cells);
            memcpy(cmax, bmax + (size_t)s * cells, sizeof(double) * cells);
            for (unsigned r = 0; r < deg; ++r) {
                if (!(valid[r] && run[r] == f)) continue;
                const unsigned rid = (unsigned)g->neighbor_ids[beg + r];
                if (r == s) { /* :496-511 */
                    chain[len++] = rid;
                    if (len >= m->gms) break;
                    continue;
                }
                /* bundle_intersection + valid check, :832-854 */
                int ok = 0;
                const double *rmn = bmin + (size_t)r * cells, *rmx = bmax + (size_t)r * cells;
                for (unsigned c = 0; c < cells; ++c) {
                    imin[c] = (cmin[c] < rmn[c]) ? rmn[c] : cmin[c];
                    imax[c] = (cmax[c] > rmx[c]) ? rmx[c] : cmax[c];
                }
                for (unsigned c = 0; c < cells; ++c)
                    if (imax[c] > imin[c]) { ok = 1; break; }
                if (ok) {
                    chain[len++] = rid;
                    memcpy(cmin, imin, sizeof(double) * cells);
                    memcpy(cmax, imax, sizeof(double) * cells);
                }
                if (len >= m->gms) break;
            }
            if (len <= 2) continue; /* :549 */
            /* check_curvelet_exist, :876-916 */
            int exists = 0;
            for (unsigned a = 0; a < n_acc && !exists; ++a) {
                const unsigned *row = accepted + (size_t)a * W;
                if (row[m->gms] != len) continue;
                int same = 1;
                for (unsigned q = 0; q < len; ++q) same = same && (row[q] == chain[q]);
                exists = same;
            }
            if (exists) continue;
            unsigned *row = accepted + (size_t)n_acc * W;
            for (unsigned q = 0; q < W; ++q) row[q] = 0;
            for (unsigned q = 0; q < len; ++q) row[q] = chain[q];
            row[m->gms] = len;
            ++n_acc;
            /* record_curvelet_chain, :258-280 */
            unsigned *out = chains + (size_t)n_out * W;
            for (unsigned q = 0; q < W; ++q) out[q] = 0;
            out[0] = (unsigned)te + 1;
            for (unsigned q = 0; q < len && q + 1 < W; ++q) out[q + 1] = chain[q] + 1;
            orc_fill_info(m, edges, sz, f == 0, tx, ty, to, cmin, cmax, chain, len, info + (size_t)n_out * 10);
            ++n_out;
        }
    }
    *valid_pairs_out = vp;
    return n_out;
}

/* The whole path: run_curvelet<double> without the file I/O (main.cpp:20-96).
 * Returns 0, or -1 on invalid input, -2 on unsupported parameters. */
int orc_run(const double *edges, int num_edges, int sz, double nrad, double dx, double dt_deg,
            double max_k, double sx, double st, unsigned group_max_sz, unsigned max_candidates,
            int nthreads, orc_result *res)
{
    memset(res, 0, sizeof(*res));
    if (group_max_sz < 1 || group_max_sz > 63) return -2;
    orc_csr g;
    if (orc_build_csr(edges, num_edges, sz, nrad, 3u, max_candidates, nthreads, &g) != 0) return -1;
    orc_model m;
    orc_model_init(&m, nrad, dx, dt_deg, max_k, sx, st, group_max_sz);
    const unsigned cells = m.P * m.Q;
    const unsigned W = group_max_sz + 1;
    const size_t np = (size_t)g.total_neighbor_pairs;

    unsigned *st_chains = (unsigned *)malloc(sizeof(unsigned) * (np ? np : 1) * W);
    double *st_info = (double *)malloc(sizeof(double) * (np ? np : 1) * 10);
    unsigned *cnt = (unsigned *)calloc((size_t)num_edges, sizeof(unsigned));
    unsigned vp_total = 0;
    const size_t scratch_bytes = sizeof(double) * ((size_t)2 * g.max_num_of_neighbors * cells + 4 * cells) +
                                 sizeof(unsigned) * (size_t)(g.max_num_of_neighbors + 1) * W +
                                 2 * (size_t)g.max_num_of_neighbors;

#ifdef _OPENMP
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : 1) reduction(+ : vp_total)
#endif
    {
        double *scratch = (double *)malloc(scratch_bytes + 64);
#ifdef _OPENMP
#pragma omp for schedule(dynamic, 64)
#endif
        for (int te = 0; te < num_edges; ++te) {
            unsigned vp = 0;
            const size_t base = (size_t)g.neighbor_offsets[te];
            cnt[te] = orc_anchor(&m, edges, sz, &g, te, st_chains + base * W, st_info + base * 10, &vp, scratch);
            vp_total += vp;
        }
        free(scratch);
    }

    /* compact_curvelet_output, cpu_curvelet.hpp:282-303 */
    size_t total = 0;
    for (int te = 0; te < num_edges; ++te) total += cnt[te];
    res->chains = (unsigned *)malloc(sizeof(unsigned) * (total ? total : 1) * W);
    res->info = (double *)malloc(sizeof(double) * (total ? total : 1) * 10);
    size_t dst = 0;
    for (int te = 0; te < num_edges; ++te) {
        const size_t base = (size_t)g.neighbor_offsets[te];
        memcpy(res->chains + dst * W, st_chains + base * W, sizeof(unsigned) * cnt[te] * W);
        memcpy(res->info + dst * 10, st_info + base * 10, sizeof(double) * cnt[te] * 10);
        dst += cnt[te];
    }
    res->num_edges = num_edges;
    res->total_neighbor_pairs = g.total_neighbor_pairs;
    res->max_num_of_neighbors = g.max_num_of_neighbors;
    res->truncated_anchors = g.truncated_anchors;
    res->tie_anchors = g.tie_anchors;
    res->valid_pairs = vp_total;
    res->num_curvelets = (unsigned)total;
    res->chain_width = W;
    res->anchor_count = cnt;
    free(st_chains);
    free(st_info);
    orc_csr_free(&g);
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Downstream: curvelets -> edgel link graph -> contour fragments           */
/* (original_code/form_curvelet_process.cpp:453-654, edgel_link_graph.hpp,  */
/*  curve_fragment_graph.hpp)                                                */
/* ---------------------------------------------------------------------- */

typedef struct {
    int pe, ce, votes;
} orc_link;

typedef struct {
    int *v;
    int n, cap;
} orc_ivec;

static void orc_ivec_push(orc_ivec *a, int x)
{
    if (a->n == a->cap) {
        a->cap = a->cap ? 2 * a->cap : 4;
        a->v = (int *)realloc(a->v, sizeof(int) * (size_t)a->cap);
    }
    a->v[a->n++] = x;
}

typedef struct {
    int num_links;
    int *link_pe, *link_ce, *link_votes; /* _cLinks order: parent id ascending, creation order */
    int num_frags;
    int64_t *frag_offsets;               /* [num_frags + 1] */
    int *frag_ids;                       /* 0-based edge ids, fragment order */
} orc_contours;

void orc_contours_free(orc_contours *c)
{
    free(c->link_pe);
    free(c->link_ce);
    free(c->link_votes);
    free(c->frag_offsets);
    free(c->frag_ids);
    memset(c, 0, sizeof(*c));
}

/* sq_distance of two edgel points, original_code/curvelet_utils.hpp:17-20 */
static double orc_pt_sqd(const double *edges, int sz, int a, int b)
{
    const double *A = edges + (size_t)a * sz, *B = edges + (size_t)b * sz;
    return (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]);
}

/* chains: row-major [num_curvelets][W] as the curvelet path writes them (column 0 =
 * anchor + 1, then the ordered chain, 1-based, zero-padded), rows grouped by anchor
 * in ascending anchor order. Returns 0, -1 on bad input. */
int orc_link_contours(const double *edges, int num_edges, int sz, const unsigned *chains, int num_curvelets,
                      int W, unsigned min_group_size, double gap, orc_contours *out)
{
    memset(out, 0, sizeof(*out));
    if (num_edges <= 0 || sz < 4 || W < 2) return -1;
    orc_ivec *clinks = (orc_ivec *)calloc((size_t)num_edges, sizeof(orc_ivec)); /* link indices */
    orc_ivec *plinks = (orc_ivec *)calloc((size_t)num_edges, sizeof(orc_ivec));
    orc_link *links = NULL;
    int nl = 0, capl = 0;
    /* construct_the_link_graph (form_curvelet_process.cpp:453-506): every curvelet
     * of order >= min_group_size, anchors ascending, links each consecutive pair of
     * its chain (form_links_from_a_curvelet, :509-520) */
    int prev_anchor = -1;
    for (int r = 0; r < num_curvelets; ++r) {
        const unsigned *row = chains + (size_t)r * W;
        const int a = (int)row[0] - 1;
        if (a < 0 || a >= num_edges || a < prev_anchor) goto bad;
        prev_anchor = a;
        int len = 0;
        while (len < W - 1 && row[1 + len]) {
            if ((int)row[1 + len] > num_edges) goto bad;
            ++len;
        }
        if ((unsigned)len < min_group_size) continue;
        for (int k = 0; k + 1 < len; ++k) {
            const int e1 = (int)row[1 + k] - 1, e2 = (int)row[2 + k] - 1;
            /* link_edgels / are_linked (edgel_link_graph.hpp:228-265): a link between
             * the two edgels in either direction takes the vote */
            int found = -1;
            for (int q = 0; q < clinks[e1].n && found < 0; ++q)
                if (links[clinks[e1].v[q]].ce == e2) found = clinks[e1].v[q];
            for (int q = 0; q < clinks[e2].n && found < 0; ++q)
                if (links[clinks[e2].v[q]].ce == e1) found = clinks[e2].v[q];
            if (found >= 0) {
                links[found].votes += 1;
                continue;
            }
            if (nl == capl) {
                capl = capl ? 2 * capl : 1024;
                links = (orc_link *)realloc(links, sizeof(orc_link) * (size_t)capl);
            }
            links[nl].pe = e1;
            links[nl].ce = e2;
            links[nl].votes = 1;
            orc_ivec_push(&clinks[e1], nl);
            orc_ivec_push(&plinks[e2], nl);
            ++nl;
        }
    }
    {
        /* extract_one_chains_from_the_link_graph (form_curvelet_process.cpp:563-654) */
        const double thres = gap * gap;
        unsigned char *linked = (unsigned char *)calloc((size_t)num_edges, 1);
        int *fwd = (int *)malloc(sizeof(int) * ((size_t)num_edges + 2));
        int *bwd = (int *)malloc(sizeof(int) * ((size_t)num_edges + 2));
        orc_ivec ids = {0};
        int64_t total = 0;
        out->frag_offsets = (int64_t *)malloc(sizeof(int64_t) * ((size_t)num_edges + 1));
        out->frag_offsets[0] = 0;
#define ORC_LEGAL(e) (!linked[e] && plinks[e].n <= 1 && clinks[e].n <= 1) /* edgel_link_graph.hpp:218-224 */
        for (int i = 0; i < num_edges; ++i) {
            if (linked[i]) continue;
            /* edgel_is_legal_first_edgel, edgel_link_graph.hpp:208-215 */
            if (!(plinks[i].n == 1 && clinks[i].n == 1 &&
                  links[plinks[i].v[0]].pe != links[clinks[i].v[0]].ce))
                continue;
            int nf = 0, nb = 0;
            linked[i] = 1;
            int eA = links[clinks[i].v[0]].ce, eB;
            if (orc_pt_sqd(edges, sz, i, eA) < thres) fwd[nf++] = eA;
            while (ORC_LEGAL(eA)) {
                linked[eA] = 1;
                if (clinks[eA].n == 0) break;
                eB = eA;
                eA = links[clinks[eA].v[0]].ce;
                if (orc_pt_sqd(edges, sz, eB, eA) < thres)
                    fwd[nf++] = eA;
                else
                    break;
            }
            if (eA != i) {
                eA = links[plinks[i].v[0]].pe;
                if (orc_pt_sqd(edges, sz, i, eA) < thres) bwd[nb++] = eA;
            }
            while (ORC_LEGAL(eA)) {
                linked[eA] = 1;
                if (plinks[eA].n == 0) break;
                eB = eA;
                eA = links[plinks[eA].v[0]].pe;
                if (orc_pt_sqd(edges, sz, eB, eA) < thres)
                    bwd[nb++] = eA;
                else
                    break;
            }
            if (nb + 1 + nf > 2) { /* prune the short ones, :648-651 */
                for (int q = nb - 1; q >= 0; --q) orc_ivec_push(&ids, bwd[q]);
                orc_ivec_push(&ids, i);
                for (int q = 0; q < nf; ++q) orc_ivec_push(&ids, fwd[q]);
                total += nb + 1 + nf;
                out->frag_offsets[++out->num_frags] = total;
            }
        }
#undef ORC_LEGAL
        out->frag_ids = ids.v ? ids.v : (int *)malloc(sizeof(int));
        free(linked);
        free(fwd);
        free(bwd);
    }
    /* the link list in _cLinks order (parent ascending, creation order) */
    out->num_links = nl;
    out->link_pe = (int *)malloc(sizeof(int) * ((size_t)nl + 1));
    out->link_ce = (int *)malloc(sizeof(int) * ((size_t)nl + 1));
    out->link_votes = (int *)malloc(sizeof(int) * ((size_t)nl + 1));
    {
        int k = 0;
        for (int e = 0; e < num_edges; ++e)
            for (int q = 0; q < clinks[e].n; ++q) {
                const orc_link *l = &links[clinks[e].v[q]];
                out->link_pe[k] = l->pe;
                out->link_ce[k] = l->ce;
                out->link_votes[k] = l->votes;
                ++k;
            }
    }
    for (int e = 0; e < num_edges; ++e) {
        free(clinks[e].v);
        free(plinks[e].v);
    }
    free(clinks);
    free(plinks);
    free(links);
    return 0;
bad:
    for (int e = 0; e < num_edges; ++e) {
        free(clinks[e].v);
        free(plinks[e].v);
    }
    free(clinks);
    free(plinks);
    free(links);
    return -1;
}

/* ---------------------------------------------------------------------- */
/* Downstream: C^1 polyarcs along the contour fragments                     */
/* (original_code/form_curvelet_process.cpp:661-796, CC_curve_model_3d.cpp, */
/*  curvelet.cpp, polyarcmap.hpp)                                            */
/* ---------------------------------------------------------------------- */

#define ORC_K_TH 1e-4 /* k_th, original_code/curvelet_utils.hpp:15 */

typedef struct {
    int num;
    int64_t *offsets; /* [num + 1] into ids */
    int *ids;         /* 0-based edge ids */
    double *info;     /* [num][12]: curvelet::set_output's columns, unset ones 0 */
} orc_polyarcs;

void orc_polyarcs_free(orc_polyarcs *p)
{
    free(p->offsets);
    free(p->ids);
    free(p->info);
    memset(p, 0, sizeof(*p));
}

/* form_a_hypothesis(ref, e2, max_k, ref_first, forward = true, centered = false,
 * leading = true) (form_curvelet_process.cpp:388-444): a model only when e2 lies
 * ahead of ref (dot > 0), with the CC_curve_model_3d bundle
 * (CC_curve_model_3d.cpp:181-335, the same transport as compute_curve_bundle of
 * cpu_curvelet). Returns 1 for a valid bundle, 0 for none or an empty one. */
static int orc_hypothesis(const orc_model *m, const double *edges, int sz, int a, int b, double *bmin,
                          double *bmax)
{
    const double *A = edges + (size_t)a * sz, *B = edges + (size_t)b * sz;
    if (!(orc_dot(orc_angle_pt_pt(A[0], A[1], B[0], B[1]), A[2]) > 0)) return 0;
    for (unsigned c = 0; c < m->P * m->Q; ++c) {
        bmin[c] = -m->max_k;
        bmax[c] = m->max_k;
    }
    return orc_curve_bundle(m, A[0], A[1], B[0], B[1], A[2], B[2], bmin, bmax);
}

/* fit_polyarc_to_chain over every fragment, then
 * compute_best_fit_according_to_curvelets (polyarcmap.hpp:98-111). dx, dt (rad),
 * max_k, rad and token_len are form_curvelet_process's; the bundle grid steps are
 * CC_curve_model_3d's fixed _dx_ = 0.1 and _dt_ = 0.08. */
int orc_polyarcs_fit(const double *edges, int num_edges, int sz, const int64_t *frag_off, const int *frag_ids,
                     int nfrags, double dx, double dt, double max_k, double rad, double token_len,
                     orc_polyarcs *out)
{
    memset(out, 0, sizeof(*out));
    if (num_edges <= 0 || sz < 4 || nfrags < 0) return -1;
    orc_model m;
    m.nrad = rad;
    m.dx = dx;
    m.dt = dt;
    m.max_k = max_k;
    m.sx = 0.1;
    m.st = 0.08;
    m.P = (unsigned)(2 * floor(dx / 0.1 + 0.5) + 1);  /* CC_curve_model_3d.cpp:196-200 */
    m.Q = (unsigned)(2 * floor(dt / 0.08 + 0.5) + 1);
    m.gms = 0;
    const unsigned cells = m.P * m.Q;
    double *cmin = (double *)malloc(sizeof(double) * cells * 4);
    double *cmax = cmin + cells, *rmin = cmax + cells, *rmax = rmin + cells;
    const int64_t total = nfrags ? frag_off[nfrags] : 0;
    out->offsets = (int64_t *)malloc(sizeof(int64_t) * ((size_t)total + 1));
    out->ids = (int *)malloc(sizeof(int) * ((size_t)total * 2 + 1));
    out->info = (double *)calloc((size_t)total * 12 + 1, sizeof(double));
    out->offsets[0] = 0;
    int64_t nid = 0;
    for (int f = 0; f < nfrags; ++f) {
        const int *ids = frag_ids + frag_off[f];
        const int N = (int)(frag_off[f + 1] - frag_off[f]);
        int i = 0;
        while (i < N - 1) { /* fit_polyarc_to_chain, form_curvelet_process.cpp:683-769 */
            const int iA = i, a = ids[i];
            ++i;
            if (!orc_hypothesis(&m, edges, sz, a, ids[i], cmin, cmax)) continue;
            int j = i;
            while (j < N - 1) {
                if (!orc_hypothesis(&m, edges, sz, a, ids[j + 1], rmin, rmax)) break;
                /* CC_curve_model_3d(cm1, cm2): Kmin = std::max, Kmax = std::min (hpp:70-84) */
                int ok = 0;
                for (unsigned c = 0; c < cells; ++c) {
                    rmin[c] = (cmin[c] < rmin[c]) ? rmin[c] : cmin[c];
                    rmax[c] = (rmax[c] < cmax[c]) ? rmax[c] : cmax[c];
                    ok = ok || (rmax[c] > rmin[c]);
                }
                if (!ok) break;
                memcpy(cmin, rmin, sizeof(double) * cells);
                memcpy(cmax, rmax, sizeof(double) * cells);
                ++j;
            }
            /* the polyarc is ids[iA .. j]; curve_fit_is_reasonable -> compute_best_fit
             * (CC_curve_model_3d.cpp:338-383, :444-451): the open cell nearest the grid
             * centre, first in row-major order */
            unsigned best = cells;
            double mind = 100;
            for (unsigned ci = 0; ci < m.P; ci++)
                for (unsigned cj = 0; cj < m.Q; cj++) {
                    const unsigned c = ci * m.Q + cj;
                    if (cmax[c] > cmin[c]) {
                        const double ddx = 0.1 * ((double)ci - ((double)m.P - 1.0) / 2.0);
                        const double ddt = 0.08 * ((double)cj - ((double)m.Q - 1.0) / 2.0);
                        const double d = ddx * ddx + ddt * ddt;
                        if (d < mind) {
                            mind = d;
                            best = c;
                        }
                    }
                }
            if (best == cells) best = 0; /* not reached: the bundle is valid */
            double k = (cmax[best] + cmin[best]) / 2;
            const double kmax = cmax[best], kmin = cmin[best];
            const int size = j - iA + 1;
            /* curvelet::compute_properties (curvelet.cpp:80-104): the anchor is the
             * chain's front, so every step counts before it */
            double L = 0;
            for (int q = iA; q < j; ++q) L += sqrt(orc_pt_sqd(edges, sz, ids[q], ids[q + 1]));
            const double quality = 2 / (1.0 * rad / L + 1.0 * L / token_len / size);
            /* compute_best_fit_according_to_curvelets -> update_best_fit
             * (CC_curve_model_3d.cpp:400-441) with _pt = the front edge */
            const double *PT = edges + (size_t)a * sz;
            const double *P1 = edges + (size_t)ids[iA + size / 2] * sz;
            const double *P2 = edges + (size_t)ids[j] * sz;
            double theta, angle = 0.0, cx = 0.0, cy = 0.0;
            int arc = 0;
            if (fabs(k) < ORC_K_TH) {
                k = 0.0;
                theta = atan2(P2[1] - PT[1], P2[0] - PT[0]);
            } else {
                const double d1 = PT[0] * PT[0] + PT[1] * PT[1], d2 = P1[0] * P1[0] + P1[1] * P1[1],
                             d3 = P2[0] * P2[0] + P2[1] * P2[1];
                const double a11 = 2.0 * (PT[0] - P1[0]), a12 = 2.0 * (PT[1] - P1[1]), a21 = 2.0 * (P2[0] - P1[0]),
                             a22 = 2.0 * (P2[1] - P1[1]);
                const double b1 = d1 - d2, b2 = d3 - d2;
                const double det = a11 * a22 - a21 * a12;
                if (fabs(det) < ORC_K_TH) {
                    k = 0.0;
                    theta = atan2(P2[1] - PT[1], P2[0] - PT[0]);
                } else {
                    cx = (b1 * a22 - b2 * a12) / det;
                    cy = (b2 * a11 - b1 * a21) / det;
                    const double v1x = PT[0] - cx, v1y = PT[1] - cy, v2x = P2[0] - cx, v2y = P2[1] - cy;
                    const double c = v1x * v2y - v1y * v2x, d = v1x * v2x + v1y * v2y;
                    angle = atan2(fabs(c), d);
                    theta = atan2(c * v1x, -c * v1y);
                    k = 1.0 / sqrt(v2x * v2x + v2y * v2y);
                    arc = 1;
                }
            }
            /* curvelet::update_length (curvelet.cpp:162-169) */
            if (fabs(angle) > 0 && fabs(k) > ORC_K_TH && arc) L = angle / fabs(k);
            /* fit_polyarc_to_chain ends with compute_best_fit_according_to_curvelets over
             * every polyarc so far (form_curvelet_process.cpp:772), so a polyarc of
             * fragment f is fitted again at the end of each later fragment. A refit
             * repeats a line and an arc with |k| >= k_th exactly; an arc with |k| < k_th
             * becomes a line (k = 0, theta along the chord), keeping its centre, angle and
             * length, and stays one. */
            if (arc && fabs(k) < ORC_K_TH && f < nfrags - 1) {
                k = 0.0;
                theta = atan2(P2[1] - PT[1], P2[0] - PT[0]);
            }
            double *row = out->info + (size_t)out->num * 12;
            row[0] = 1.0; /* forward */
            row[1] = kmax; /* _ref_pt, overwritten by compute_best_fit (:378-379) */
            row[2] = kmin;
            row[3] = PT[2]; /* _ref_theta */
            row[4] = PT[0];
            row[5] = PT[1];
            row[6] = theta;
            row[7] = k;
            row[8] = L;
            row[9] = quality;
            row[10] = arc ? cx : 0.0;
            row[11] = arc ? cy : 0.0;
            for (int q = iA; q <= j; ++q) out->ids[nid++] = ids[q];
            out->offsets[++out->num] = nid;
            i = j;
        }
    }
    free(cmin);
    return 0;
}
