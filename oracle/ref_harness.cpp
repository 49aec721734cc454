// ref_harness.cpp -- TEST INFRASTRUCTURE ONLY (the oracle's "reference" leg).
//
// This file is compiled against the reference's own header-only cpu_curvelet
// sources, where they lie (cpu_curvelet/preprocess.hpp, cpu_curvelet/cpu_curvelet.hpp,
// included by path through -I by oracle/Makefile), into oracle/_ref/libcvlref.so.
// It exposes the reference templates through a C ABI so that the tests and
// bench.py's reference arm can run the reference's exact code in-process and
// read its results at full precision (the reference's own info file is written
// with 6 significant digits, cpu_curvelet/data_io.hpp:109-134).
//
// The call sequence restates run_curvelet<double> (cpu_curvelet/main.cpp:20-96):
//   build_neighbor_csr_graph (preprocess.hpp:186)  -> CurveletCPU ctor (cpu_curvelet.hpp:82)
//   -> form_pairwise_bundles (cpu_curvelet.hpp:305) -> build_curvelets_greedy (:363)
// and then copies _edge_chain_final (row-major) and _curvelet_info (column-major,
// stride _max_curvelets, transposed to row-major as main.cpp:81-88 does).
//
// Nothing in the product (libcvl) links or loads this file.

// The headers come in main.cpp's order (main.cpp:1-11): <math.h> before the
// reference headers puts the float overloads of sin/cos in the global namespace,
// so that an unqualified sin(float) inside the templates resolves to the float
// function there, as it does in the reference program (T = float).
#include <iostream>
#include <cmath>
#include <math.h>
#include <string>
#include <vector>

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "preprocess.hpp"
#include "cpu_curvelet.hpp"

extern "C" {

typedef struct cvlref_out {
    int num_edges;
    int total_neighbor_pairs;
    unsigned max_num_of_neighbors;
    unsigned valid_pairs;
    unsigned num_curvelets;
    unsigned chain_width;
    int *neighbor_offsets;      // [num_edges + 1]
    int *neighbor_ids;          // [total_neighbor_pairs]
    double *neighbor_dist2;     // [total_neighbor_pairs]
    unsigned *chains;           // [num_curvelets * chain_width], 1-based ids
    double *info;               // [num_curvelets * 10], row-major
    double ms_csr;              // wall time of the three timed phases (main.cpp:43-66)
    double ms_pairwise;
    double ms_greedy;
} cvlref_out;

// Silences the reference's std::cout/std::cerr prints for the duration of a call.
struct quiet_scope {
    std::streambuf *o = nullptr, *e = nullptr;
    std::ostringstream sink;
    explicit quiet_scope(bool on) {
        if (on) {
            o = std::cout.rdbuf(sink.rdbuf());
            e = std::cerr.rdbuf(sink.rdbuf());
        }
    }
    ~quiet_scope() {
        if (o) std::cout.rdbuf(o);
        if (e) std::cerr.rdbuf(e);
    }
};

static double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

}  // extern "C"

// run_curvelet<T> without the file I/O (main.cpp:20-96), for T = double and float.
// With nb_offsets/nb_ids given, the neighbour lists that build_neighbor_csr_graph
// made are replaced by those before the CurveletCPU stage runs (the graph's edge
// table stays the reference's own): the reference's bundles, growth and record
// code then run on a caller-chosen CSR, e.g. one whose truncated anchors keep the
// lowest edge indices of a pixel cell.
template <typename T>
static int run_impl(const T *edges, int num_edges, int edge_data_sz, double nrad, double dx, double dt_deg,
                    double max_k, double sx, double st, unsigned group_max_sz, unsigned max_candidates, int nthreads,
                    int quiet, int want_outputs, cvlref_out *out, const int *nb_offsets = nullptr,
                    const int *nb_ids = nullptr)
{
    std::memset(out, 0, sizeof(*out));
    quiet_scope q(quiet != 0);

    // main.cpp:21-29 parameter conversions
    const T t_nrad = T(nrad);
    const T t_dx = T(dx);
    const T t_dt = T(dt_deg / 180.0) * T(M_PI);
    const T t_max_k = T(max_k);
    const T t_sx = T(sx);
    const T t_st = T(st);

    std::vector<T> toed(edges, edges + (size_t)num_edges * (size_t)edge_data_sz);
    int edge_num = num_edges;
    int sz = edge_data_sz;

    auto t0 = std::chrono::steady_clock::now();
    CPUNeighborGraph<T> csr;
    if (!build_neighbor_csr_graph(edge_num, sz, toed.data(), t_nrad, 3u, max_candidates, nthreads, csr)) {
        return -1;
    }
    out->ms_csr = ms_since(t0);
    if (nb_offsets != nullptr) {
        if (nb_offsets[0] != 0) return -3;
        unsigned maxdeg = 0;
        for (int a = 0; a < num_edges; ++a) {
            const int d = nb_offsets[a + 1] - nb_offsets[a];
            if (d < 0) return -3;
            if ((unsigned)d > maxdeg) maxdeg = (unsigned)d;
        }
        const int np = nb_offsets[num_edges];
        csr.neighbor_offsets.assign(nb_offsets, nb_offsets + num_edges + 1);
        csr.neighbor_ids.assign(nb_ids, nb_ids + np);
        csr.neighbor_dist2.assign((size_t)np, T(0));
        for (int a = 0; a < num_edges; ++a) {
            for (int k = nb_offsets[a]; k < nb_offsets[a + 1]; ++k) {
                const int b = nb_ids[k];
                if (b < 0 || b >= num_edges || b == a) return -3;
                csr.neighbor_dist2[(size_t)k] = sq_dist<T>(toed[(size_t)a * sz], toed[(size_t)a * sz + 1],
                                                           toed[(size_t)b * sz], toed[(size_t)b * sz + 1]);
            }
        }
        csr.total_neighbor_pairs = np;
        csr.max_num_of_neighbors = maxdeg;
    }

    t0 = std::chrono::steady_clock::now();
    CurveletCPU<T> obj(edge_num, sz, csr, t_dx, t_dt, t_sx, t_st, t_max_k, group_max_sz, nthreads, toed.data(),
                       t_nrad);
    CPUCurveletFormationResult br;
    if (!obj.form_pairwise_bundles(br)) {
        return -2;
    }
    out->ms_pairwise = ms_since(t0);

    t0 = std::chrono::steady_clock::now();
    obj.build_curvelets_greedy();
    out->ms_greedy = ms_since(t0);

    out->num_edges = num_edges;
    out->total_neighbor_pairs = csr.total_neighbor_pairs;
    out->max_num_of_neighbors = csr.max_num_of_neighbors;
    out->valid_pairs = br.valid_pairs;
    out->num_curvelets = obj.num_curvelets();
    out->chain_width = obj.chain_width();
    if (!want_outputs) {
        return 0;
    }

    const size_t np = (size_t)csr.total_neighbor_pairs;
    out->neighbor_offsets = (int *)std::malloc(sizeof(int) * ((size_t)num_edges + 1));
    out->neighbor_ids = (int *)std::malloc(sizeof(int) * (np ? np : 1));
    out->neighbor_dist2 = (double *)std::malloc(sizeof(double) * (np ? np : 1));
    std::memcpy(out->neighbor_offsets, csr.neighbor_offsets.data(), sizeof(int) * ((size_t)num_edges + 1));
    if (np) {
        std::memcpy(out->neighbor_ids, csr.neighbor_ids.data(), sizeof(int) * np);
        for (size_t k = 0; k < np; ++k) out->neighbor_dist2[k] = (double)csr.neighbor_dist2[k];
    }

    const size_t nc = out->num_curvelets;
    const size_t w = out->chain_width;
    out->chains = (unsigned *)std::malloc(sizeof(unsigned) * (nc * w ? nc * w : 1));
    out->info = (double *)std::malloc(sizeof(double) * (nc * 10 ? nc * 10 : 1));
    for (size_t i = 0; i < nc * w; ++i) out->chains[i] = obj._edge_chain_final[i];
    const size_t stride = obj._max_curvelets;
    for (size_t row = 0; row < nc; ++row)
        for (size_t col = 0; col < 10; ++col)
            out->info[row * 10 + col] = obj._curvelet_info[col * stride + row];
    return 0;
}

extern "C" {

int cvlref_run(const double *edges, int num_edges, int edge_data_sz,
               double nrad, double dx, double dt_deg, double max_k,
               double sx, double st, unsigned group_max_sz, unsigned max_candidates,
               int nthreads, int quiet, int want_outputs, cvlref_out *out)
{
    return run_impl<double>(edges, num_edges, edge_data_sz, nrad, dx, dt_deg, max_k, sx, st, group_max_sz,
                            max_candidates, nthreads, quiet, want_outputs, out);
}

// run_curvelet<float> (the --float mode, main.cpp:110), on edges already in float.
int cvlref_run_f32(const float *edges, int num_edges, int edge_data_sz,
                   double nrad, double dx, double dt_deg, double max_k,
                   double sx, double st, unsigned group_max_sz, unsigned max_candidates,
                   int nthreads, int quiet, int want_outputs, cvlref_out *out)
{
    return run_impl<float>(edges, num_edges, edge_data_sz, nrad, dx, dt_deg, max_k, sx, st, group_max_sz,
                           max_candidates, nthreads, quiet, want_outputs, out);
}

// The CurveletCPU stage of run_curvelet<double> / <float> on the given neighbour
// lists (offsets [num_edges + 1], ids [offsets[num_edges]], input edge indices).
// Returns -3 on lists that are not a CSR over the map's edges.
int cvlref_run_csr(const double *edges, int num_edges, int edge_data_sz,
                   double nrad, double dx, double dt_deg, double max_k,
                   double sx, double st, unsigned group_max_sz, unsigned max_candidates,
                   const int *nb_offsets, const int *nb_ids, cvlref_out *out)
{
    return run_impl<double>(edges, num_edges, edge_data_sz, nrad, dx, dt_deg, max_k, sx, st, group_max_sz,
                            max_candidates, 1, 1, 1, out, nb_offsets, nb_ids);
}

int cvlref_run_csr_f32(const float *edges, int num_edges, int edge_data_sz,
                       double nrad, double dx, double dt_deg, double max_k,
                       double sx, double st, unsigned group_max_sz, unsigned max_candidates,
                       const int *nb_offsets, const int *nb_ids, cvlref_out *out)
{
    return run_impl<float>(edges, num_edges, edge_data_sz, nrad, dx, dt_deg, max_k, sx, st, group_max_sz,
                           max_candidates, 1, 1, 1, out, nb_offsets, nb_ids);
}

void cvlref_free(cvlref_out *out)
{
    std::free(out->neighbor_offsets);
    std::free(out->neighbor_ids);
    std::free(out->neighbor_dist2);
    std::free(out->chains);
    std::free(out->info);
    std::memset(out, 0, sizeof(*out));
}

// One pair's 63-cell bundle through CurveletCPU::compute_curve_bundle
// (cpu_curvelet.hpp:637-819). Builds a two-edge object so the member is
// reachable; te/le are the anchor and neighbour (x, y, orientation).
int cvlref_pair_bundle(double te_x, double te_y, double te_o, double le_x, double le_y, double le_o,
                       double nrad, double dx, double dt_deg, double max_k, double sx, double st,
                       double *bmin, double *bmax, int *ncells)
{
    quiet_scope q(true);
    double e[8] = {te_x, te_y, te_o, 1.0, le_x, le_y, le_o, 1.0};
    CPUNeighborGraph<double> csr;
    csr.num_edges = 2;
    csr.total_neighbor_pairs = 1;
    csr.max_num_of_neighbors = 1;
    csr.edges.assign(e, e + 8);
    csr.neighbor_offsets = {0, 1, 1};
    csr.neighbor_ids = {1};
    csr.neighbor_dist2 = {0.0};
    int n = 2, sz = 4;
    const double t_dt = double(dt_deg / 180.0) * double(M_PI);
    CurveletCPU<double> obj(n, sz, csr, dx, t_dt, sx, st, max_k, 4u, 1, e, nrad);
    const int P = (int)(2 * std::floor(dx / sx + 0.5) + 1);
    const int Q = (int)(2 * std::floor(t_dt / st + 0.5) + 1);
    const int cells = P * Q;
    std::vector<double> mn((size_t)cells, -max_k), mx((size_t)cells, max_k);
    bool hyp[1] = {false};
    const bool ok = obj.compute_curve_bundle(0u, 0u, mn.data(), mx.data(), hyp, te_x, te_y, le_x, le_y, te_o, le_o);
    for (int c = 0; c < cells; ++c) { bmin[c] = mn[(size_t)c]; bmax[c] = mx[(size_t)c]; }
    *ncells = cells;
    return (ok && hyp[0]) ? 1 : 0;
}

}  // extern "C"
