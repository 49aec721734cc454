// orig_harness.cpp -- TEST INFRASTRUCTURE ONLY (the oracle's "reference" leg for
// the downstream stage: curvelets -> edgel link graph -> contour fragments).
//
// The reference implements this stage only in its original_code/ tree:
//   form_curvelet_process::construct_the_link_graph      (form_curvelet_process.cpp:453-506)
//   form_curvelet_process::form_links_from_a_curvelet     (form_curvelet_process.cpp:509-520)
//   form_curvelet_process::extract_regular_contours_from_the_link_graph
//                                                         (form_curvelet_process.cpp:529-547)
//   form_curvelet_process::extract_one_chains_from_the_link_graph
//                                                         (form_curvelet_process.cpp:563-654)
//   edgel_link_graph::link_edgels / edgel_is_legal*       (edgel_link_graph.hpp:207-265)
//   curve_fragment_graph::insert_fragment / get_output_array (curve_fragment_graph.hpp)
// Those are private members of form_curvelet_process and its execute() has the
// calls commented out, so no public entry reaches them. This file compiles the
// original sources where they lie (a single translation unit: oracle/Makefile
// passes -I to original_code/) with the access specifiers opened, fills the
// process's curvelet map with the curvelets given, runs the two stages and
// returns the link graph and the fragments through a C ABI.
//
// Nothing in the product (libcvl) links or loads this file.

// every standard header the original sources use comes first, so that the
// access override below touches only the original classes
#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <ctime>
#include <deque>
#include <filesystem>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <list>
#include <map>
#include <set>
#include <utility>
#include <vector>
#include <assert.h>
#include <math.h>
#include <string.h>

#define private public
#define protected public
#include "form_curvelet_process.cpp"
#include "curvelet.cpp"
#include "curveletmap.cpp"
#include "CC_curve_model_3d.cpp"
// the definition of k_th (declared extern by polyarcmap.hpp), which the original
// program gets from its main.cpp
#include "curvelet_utils.hpp"
#undef private
#undef protected

extern "C" {

typedef struct origref_contours_out {
    int32_t num_links;
    int32_t *link_pe;      // [num_links] parent edge id (0-based), in (_cLinks[i] order, i ascending)
    int32_t *link_ce;      // [num_links] child edge id
    int32_t *link_votes;   // [num_links] votes (number of curvelets giving the link)
    int32_t num_frags;
    int64_t *frag_offsets; // [num_frags + 1]
    int32_t *frag_ids;     // [frag_offsets[num_frags]] 0-based edge ids, fragment order
    double seconds;        // link graph + extraction, wall clock
} origref_contours_out;

// edges: row-major [num_edges][edge_data_sz]; chains: row-major [num_curvelets][chain_width],
// column 0 = anchor id + 1, then the ordered chain (1-based ids), zero-padded
int origref_link_contours(const double *edges, int num_edges, int edge_data_sz, const uint32_t *chains,
                          int num_curvelets, int chain_width, const uint8_t *forward, unsigned min_group_size,
                          double gap, origref_contours_out *out) {
    std::memset(out, 0, sizeof(*out));
    if (num_edges <= 0 || edge_data_sz < 4 || chain_width < 2) return -1;
    // form_curvelet_mex gets column-major edge info (original_code/main.cpp:168-178)
    std::vector<double> cm((size_t)num_edges * 4);
    for (int i = 0; i < num_edges; ++i)
        for (int j = 0; j < 4; ++j) cm[(size_t)j * num_edges + i] = edges[(size_t)i * edge_data_sz + j];
    arrayd edgeinfo;
    edgeinfo._data = cm.data();
    edgeinfo.set_h(num_edges);
    edgeinfo.set_w(4);
    // parameters besides gap do not enter the two stages; these are main.cpp's
    form_curvelet_process proc(edgeinfo, 1u, 1u, 3.5, gap, 0.4, (15.0 / 180.0) * M_PI, 1.0, 0.3,
                               (unsigned)(chain_width - 1), false, true);
    proc._curveletmap.resize(num_edges);
    for (int r = 0; r < num_curvelets; ++r) {
        const uint32_t *row = chains + (size_t)r * chain_width;
        const unsigned a = row[0];
        if (a == 0 || (int)a > num_edges) return -2;
        edgel_chain ch;
        for (int k = 1; k < chain_width && row[k]; ++k) {
            if ((int)row[k] > num_edges) return -2;
            ch.push_back(proc._edgemap._list[row[k] - 1]);
        }
        proc._curveletmap.add_curvelet(
            new curvelet(proc._edgemap._list[a - 1], nullptr, ch, forward ? forward[r] != 0 : true));
    }
    const auto t0 = std::chrono::steady_clock::now();
    proc.construct_the_link_graph(min_group_size, false);
    proc.extract_regular_contours_from_the_link_graph(false);
    out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    std::vector<int32_t> pe, ce, votes;
    for (size_t i = 0; i < proc._linkgraph._cLinks.size(); ++i)
        for (edgel_link *l : proc._linkgraph._cLinks[i]) {
            pe.push_back((int32_t)l->_pe->_id);
            ce.push_back((int32_t)l->_ce->_id);
            votes.push_back((int32_t)l->_vote);
        }
    out->num_links = (int32_t)pe.size();
    out->link_pe = (int32_t *)std::malloc(sizeof(int32_t) * (pe.size() + 1));
    out->link_ce = (int32_t *)std::malloc(sizeof(int32_t) * (pe.size() + 1));
    out->link_votes = (int32_t *)std::malloc(sizeof(int32_t) * (pe.size() + 1));
    std::copy(pe.begin(), pe.end(), out->link_pe);
    std::copy(ce.begin(), ce.end(), out->link_ce);
    std::copy(votes.begin(), votes.end(), out->link_votes);

    out->num_frags = (int32_t)proc._fragraph._frags.size();
    out->frag_offsets = (int64_t *)std::malloc(sizeof(int64_t) * (out->num_frags + 1));
    size_t total = 0;
    for (edgel_chain *c : proc._fragraph._frags) total += c->size();
    out->frag_ids = (int32_t *)std::malloc(sizeof(int32_t) * (total + 1));
    size_t k = 0, f = 0;
    out->frag_offsets[0] = 0;
    for (edgel_chain *c : proc._fragraph._frags) {
        for (edgel *e : *c) out->frag_ids[k++] = (int32_t)e->_id;
        out->frag_offsets[++f] = (int64_t)k;
    }
    return 0;
}

typedef struct origref_polyarcs_out {
    int32_t num_polyarcs;
    int64_t *offsets;  // [num_polyarcs + 1] into ids
    int32_t *ids;      // 0-based edge ids of each polyarc's chain
    double *info;      // [num_polyarcs][12], curvelet::set_output's columns (form_curvelet_process.cpp:847-851)
    double seconds;    // fit_polyarcs_to_all_edgel_chains, wall clock
} origref_polyarcs_out;

// The same curvelets through the link graph, the one-chains, and then
// fit_polyarcs_to_all_edgel_chains (form_curvelet_process.cpp:661-796), read out
// as output type 2 (get_output_arrary, :847-851). The process gets dx, dt,
// max_k, rad and token_len as form_curvelet_mex would.
int origref_polyarcs(const double *edges, int num_edges, int edge_data_sz, const uint32_t *chains, int num_curvelets,
                     int chain_width, unsigned min_group_size, double gap, double dx, double dt, double max_k,
                     double rad, double token_len, origref_polyarcs_out *out) {
    std::memset(out, 0, sizeof(*out));
    if (num_edges <= 0 || edge_data_sz < 4 || chain_width < 2) return -1;
    std::vector<double> cm((size_t)num_edges * 4);
    for (int i = 0; i < num_edges; ++i)
        for (int j = 0; j < 4; ++j) cm[(size_t)j * num_edges + i] = edges[(size_t)i * edge_data_sz + j];
    arrayd edgeinfo;
    edgeinfo._data = cm.data();
    edgeinfo.set_h(num_edges);
    edgeinfo.set_w(4);
    form_curvelet_process proc(edgeinfo, 1u, 1u, rad, gap, dx, dt, token_len, max_k, (unsigned)(chain_width - 1),
                               false, true);
    for (int r = 0; r < num_curvelets; ++r) {
        const uint32_t *row = chains + (size_t)r * chain_width;
        const unsigned a = row[0];
        if (a == 0 || (int)a > num_edges) return -2;
        edgel_chain ch;
        for (int k = 1; k < chain_width && row[k]; ++k) {
            if ((int)row[k] > num_edges) return -2;
            ch.push_back(proc._edgemap._list[row[k] - 1]);
        }
        proc._curveletmap.add_curvelet(new curvelet(proc._edgemap._list[a - 1], nullptr, ch, true));
    }
    proc.construct_the_link_graph(min_group_size, false);
    proc.extract_regular_contours_from_the_link_graph(false);
    const auto t0 = std::chrono::steady_clock::now();
    proc.fit_polyarcs_to_all_edgel_chains(false);
    out->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    unsigned h = 0, w = 0;
    proc.get_output_size(h, w, 2);
    out->num_polyarcs = (int32_t)h;
    // curvelet::set_output asserts size < width, so the id array is one column wider
    // than get_output_size's; Array::init zero-fills, so unset info columns read 0
    arrayi id_chain;
    id_chain.init(h ? h : 1, w + 1);
    arrayd info;
    info.init(h ? h : 1, 12);
    // get_output_arrary (type 2) insists on the exact width, so the polyarc map
    // fills the arrays itself, as get_output_arrary would (polyarcmap::get_output_array)
    if (h) proc._polyarcmap.get_output_array(id_chain, info);
    out->offsets = (int64_t *)std::malloc(sizeof(int64_t) * (h + 1));
    out->info = (double *)std::malloc(sizeof(double) * 12 * (h ? h : 1));
    size_t total = 0;
    for (curvelet *c : proc._polyarcmap._list) total += c->_edgel_chain.size();
    out->ids = (int32_t *)std::malloc(sizeof(int32_t) * (total + 1));
    size_t k = 0;
    out->offsets[0] = 0;
    for (unsigned r = 0; r < h; ++r) {
        for (unsigned c = 0; c <= w && id_chain.val(r, c) != 0; ++c) out->ids[k++] = id_chain.val(r, c) - 1;
        out->offsets[r + 1] = (int64_t)k;
        for (int c = 0; c < 12; ++c) out->info[(size_t)r * 12 + c] = info.val(r, c);
    }
    return 0;
}

void origref_polyarcs_free(origref_polyarcs_out *out) {
    std::free(out->offsets);
    std::free(out->ids);
    std::free(out->info);
    std::memset(out, 0, sizeof(*out));
}

void origref_contours_free(origref_contours_out *out) {
    std::free(out->link_pe);
    std::free(out->link_ce);
    std::free(out->link_votes);
    std::free(out->frag_offsets);
    std::free(out->frag_ids);
    std::memset(out, 0, sizeof(*out));
}

}  // extern "C"
