// cvl_cli.cpp -- drop-in replacement for the reference CURVELET program
// (cpu_curvelet/main.cpp), running the path on the GPU through libcvl.
//
// Same flags and defaults (cpu_curvelet/param_settings.hpp:26-155), same input
// location and format (../test_files/<edge-file>, data_io.hpp:11-79), same
// outputs (../outputs/<output> and its info file, data_io.hpp:81-145, written
// with the default ostream formatting), same summary lines on stdout.
#include <cerrno>
#include <cmath>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/cvl.h"

namespace {

struct CliParams {
    cvl_params p;
    std::string edge_file = "eth3d_cables2.txt";  // param_settings.hpp:21
};

void print_usage(const char *prog) {
    std::cerr << "Usage: " << prog << " [options]\n"
              << "\n"
              << "Options:\n"
              << "  --float, --double          Scalar type (default: double)\n"
              << "  --output <file>            Output chain file (default: chain_cpu.txt)\n"
              << "  --nthreads <N>             Host thread count (accepted; the path runs on the GPU)\n"
              << "  --edge-file <file>         Input edge file in ../test_files/ (default: eth3d_cables2.txt)\n"
              << "  --nrad <val>               Neighbor search radius (default: 3.5)\n"
              << "  --dx <val>                 Edge position tolerance in pixels (default: 0.4)\n"
              << "  --dt-deg <val>             Edge angle tolerance in degrees (default: 15)\n"
              << "  --max-k <val>              Maximum curvature (default: 0.3)\n"
              << "  --curvelet-style <N>       Curvelet style (default: 2)\n"
              << "  --group-max-sz <N>         Maximum group size (default: 4)\n"
              << "  --out-type <N>             Output type (default: 0)\n"
              << "  --sx <val>                 Position sampling step (default: 0.1)\n"
              << "  --st <val>                 Angle sampling step in radians (default: 0.08)\n"
              << "  --edge-data-sz <N>         Values per edge in input file (default: 4)\n"
              << "  --max-candidates <N>       Max neighbors per anchor in CSR build (default: 128)\n"
              << "  --fragments <file>         Also write the contour fragments (edgel link graph one-chains)\n"
              << "                             to ../outputs/<file>, one fragment per row, 1-based ids\n"
              << "  --gap <val>                Fragment gap: consecutive edges closer than this (default: 1.5)\n"
              << "  --link-min-group <N>       Curvelets with at least N edges form links (default: 4)\n"
              << "  --polyarcs <file>          Also fit C^1 polyarcs along the fragments and write them to\n"
              << "                             ../outputs/<file> (1-based ids) and its info file (12 columns)\n"
              << "  --help                     Show this help message\n";
}

bool parse_num(const char *arg, const char *name, double &v) {
    char *end = nullptr;
    const double x = std::strtod(arg, &end);
    if (end == arg || *end != '\0') {
        std::cerr << "Error: invalid value for " << name << ": " << arg << std::endl;
        return false;
    }
    v = x;
    return true;
}

bool parse_uns(const char *arg, const char *name, unsigned &v) {
    char *end = nullptr;
    const unsigned long x = std::strtoul(arg, &end, 10);
    if (end == arg || *end != '\0') {
        std::cerr << "Error: invalid value for " << name << ": " << arg << std::endl;
        return false;
    }
    v = (unsigned)x;
    return true;
}

bool parse_int(const char *arg, const char *name, int &v) {
    char *end = nullptr;
    const long x = std::strtol(arg, &end, 10);
    if (end == arg || *end != '\0') {
        std::cerr << "Error: invalid value for " << name << ": " << arg << std::endl;
        return false;
    }
    v = (int)x;
    return true;
}

// Flag table of param_settings.hpp:86-155.
bool parse_args(int argc, char **argv, CliParams &cp, bool &use_double, std::string &out_file, int &nthreads,
                bool &show_help, std::string &frag_file, std::string &poly_file, cvl_contour_params &lp) {
    show_help = false;
    for (int i = 1; i < argc; i++) {
        const char *a = argv[i];
        auto next = [&](void) -> const char * { return argv[++i]; };
        const bool has = (i + 1 < argc);
        if (!std::strcmp(a, "--help") || !std::strcmp(a, "-h")) {
            print_usage(argv[0]);
            show_help = true;
            return false;
        }
        if (!std::strcmp(a, "--float")) {
            use_double = false;
            out_file = "chain_cpu_float.txt";
        } else if (!std::strcmp(a, "--double")) {
            use_double = true;
            out_file = "chain_cpu_double.txt";
        } else if (!std::strcmp(a, "--output") && has) {
            out_file = next();
        } else if (!std::strcmp(a, "--nthreads") && has) {
            nthreads = std::atoi(next());
        } else if ((!std::strcmp(a, "--input") || !std::strcmp(a, "--edge-file")) && has) {
            cp.edge_file = next();
        } else if (!std::strcmp(a, "--nrad") && has) {
            if (!parse_num(next(), "--nrad", cp.p.nrad)) return false;
        } else if (!std::strcmp(a, "--dx") && has) {
            if (!parse_num(next(), "--dx", cp.p.dx)) return false;
        } else if (!std::strcmp(a, "--dt-deg") && has) {
            if (!parse_num(next(), "--dt-deg", cp.p.dt_deg)) return false;
        } else if (!std::strcmp(a, "--max-k") && has) {
            if (!parse_num(next(), "--max-k", cp.p.max_k)) return false;
        } else if (!std::strcmp(a, "--curvelet-style") && has) {
            if (!parse_uns(next(), "--curvelet-style", cp.p.curvelet_style)) return false;
        } else if (!std::strcmp(a, "--group-max-sz") && has) {
            if (!parse_uns(next(), "--group-max-sz", cp.p.group_max_sz)) return false;
        } else if (!std::strcmp(a, "--out-type") && has) {
            if (!parse_uns(next(), "--out-type", cp.p.out_type)) return false;
        } else if (!std::strcmp(a, "--sx") && has) {
            if (!parse_num(next(), "--sx", cp.p.sx)) return false;
        } else if (!std::strcmp(a, "--st") && has) {
            if (!parse_num(next(), "--st", cp.p.st)) return false;
        } else if (!std::strcmp(a, "--edge-data-sz") && has) {
            if (!parse_int(next(), "--edge-data-sz", cp.p.edge_data_sz)) return false;
        } else if (!std::strcmp(a, "--max-candidates") && has) {
            if (!parse_uns(next(), "--max-candidates", cp.p.max_candidates)) return false;
        } else if (!std::strcmp(a, "--fragments") && has) {  // the downstream stage, not in cpu_curvelet
            frag_file = next();
        } else if (!std::strcmp(a, "--gap") && has) {
            if (!parse_num(next(), "--gap", cp.p.gap)) return false;
            lp.gap = cp.p.gap;
        } else if (!std::strcmp(a, "--polyarcs") && has) {
            poly_file = next();
        } else if (!std::strcmp(a, "--link-min-group") && has) {
            if (!parse_uns(next(), "--link-min-group", lp.min_group_size)) return false;
        } else {
            std::cerr << "Unknown argument: " << a << std::endl;
            print_usage(argv[0]);
            return false;
        }
    }
    return true;
}

// Edge-file reader with the reference's acceptance rules and messages
// (data_io.hpp:22-79), multi-threaded in libcvl (cvl_read_edges /
// cvl_read_edges_f32, into the run's scalar type); a name ending in ".cvle" is
// the binary edge format.
template <typename T>
bool read_edges(const std::string &filename, int per_edge, std::vector<T> &out) {
    const std::string path = "../test_files/" + filename;
    if (!std::ifstream(path)) {
        std::cerr << "Error: input file does not exist: " << path << std::endl;
        return false;
    }
    std::cout << "reading data from file " << filename << std::endl;
    out.clear();
    T *buf = nullptr;
    int64_t n = 0;
    int rc;
    if constexpr (std::is_same<T, float>::value)
        rc = cvl_read_edges_f32(path.c_str(), per_edge, 0, &buf, &n);
    else
        rc = cvl_read_edges(path.c_str(), per_edge, 0, &buf, &n);
    if (rc != CVL_OK) {
        std::cerr << cvl_last_error() << std::endl;
        return false;
    }
    out.assign(buf, buf + (size_t)n * per_edge);
    cvl_free_edges(buf);
    std::cout << "read " << n << " edges from " << filename << std::endl;
    return true;
}

bool open_out(const std::string &name, std::ofstream &f) {
    std::cout << "writing data to a file " << name << " ..." << std::endl;
    const std::filesystem::path dir = "../outputs";
    std::error_code ec;
    std::filesystem::create_directories(dir, ec);
    if (ec) {
        std::cerr << "Failed to create output directory " << dir << ": " << ec.message() << std::endl;
        return false;
    }
    f.open(dir.string() + "/" + name);
    if (!f.is_open()) std::cout << "write data file cannot be opened!" << std::endl;
    return true;
}

std::string info_name(const std::string &chain_file) {  // data_io.hpp:136-145
    const std::size_t pos = chain_file.find("chain");
    if (pos != std::string::npos) {
        std::string s = chain_file;
        s.replace(pos, 5, "info");
        return s;
    }
    return "info_" + chain_file;
}

}  // namespace

int main(int argc, char **argv) {
    int nthreads = 1;
    bool use_double = true;
    std::string out_file = "chain_cpu.txt";
    CliParams cp;
    cvl_params_default(&cp.p);
    bool help = false;
    std::string frag_file, poly_file;
    cvl_contour_params lp;
    cvl_contour_params_default(&lp);
    if (!parse_args(argc, argv, cp, use_double, out_file, nthreads, help, frag_file, poly_file, lp))
        return help ? 0 : 1;
    if ((!frag_file.empty() || !poly_file.empty()) && !use_double) {
        std::cerr << "Error: --fragments and --polyarcs run in double only" << std::endl;
        return 1;
    }
    if (!poly_file.empty()) {
        // form_curvelet_mex's model parameters (original_code/main.cpp:145-151) from the flags
        lp.fit_polyarcs = 1;
        lp.dx = cp.p.dx;
        lp.dt_rad = (cp.p.dt_deg / 180.0) * 3.14159265358979323846;
        lp.max_k = cp.p.max_k;
        lp.rad = cp.p.nrad;
    }
    const bool downstream = !frag_file.empty() || !poly_file.empty();
    (void)nthreads;
    std::cout << "Using scalar type: " << (use_double ? "double" : "float") << std::endl;
    // run_curvelet<double> or run_curvelet<float> (main.cpp:110)
    std::vector<double> edges;
    std::vector<float> edges_f;
    if (use_double ? !read_edges(cp.edge_file, cp.p.edge_data_sz, edges)
                   : !read_edges(cp.edge_file, cp.p.edge_data_sz, edges_f))
        return 1;
    const int n = (int)((use_double ? edges.size() : edges_f.size()) / (size_t)cp.p.edge_data_sz);

    cvl_engine *eng = nullptr;
    if (cvl_engine_create(nullptr, &eng) != CVL_OK) {
        std::cerr << "Error: " << cvl_last_error() << std::endl;
        return 1;
    }
    cvl_result *res = nullptr;
    cvl_contours *frags = nullptr;
    const int rc = downstream
                       ? cvl_run_contours(eng, edges.data(), n, cp.p.edge_data_sz, &cp.p, &lp, &res, &frags)
                   : use_double ? cvl_run(eng, edges.data(), n, cp.p.edge_data_sz, &cp.p, &res)
                                : cvl_run_f32(eng, edges_f.data(), n, cp.p.edge_data_sz, &cp.p, &res);
    if (rc != CVL_OK) {
        std::cerr << "Error: " << cvl_last_error() << std::endl;
        cvl_engine_destroy(eng);
        return 1;
    }
    cvl_result_view v;
    cvl_result_get(res, &v);
    if (v.truncated_anchors)
        std::cerr << "Warning: " << v.truncated_anchors << " anchors hit max_candidates=" << cp.p.max_candidates
                  << "; neighbor lists may be truncated\n";
    std::cout << "CSR neighbor graph: " << n << " anchors, " << v.total_neighbor_pairs
              << " total pairs, max number of neighbors per anchor: " << v.max_num_of_neighbors << std::endl;
    std::cout << "Pairwise curve bundles formed: " << v.valid_pairs << " valid pairs" << std::endl;
    std::cout << "- Time of curvelet building (GPU, device): " << v.device_ms << " (ms)" << std::endl;
    std::cout << "- Number of curvelets formed: " << v.num_curvelets << std::endl;
    const unsigned out_h = v.num_curvelets, out_w = v.chain_width;
    std::cout << "(out_h, out_w) = (" << out_h << ", " << out_w << ")" << std::endl;

    {
        std::ofstream f;
        if (open_out(out_file, f)) {
            for (unsigned i = 0; i < out_h; i++) {
                for (unsigned j = 0; j < out_w; j++) f << (int)v.chains[(size_t)i * out_w + j] << "\t";
                f << "\n";
            }
        }
    }
    {
        std::ofstream f;
        if (open_out(info_name(out_file), f)) {
            for (unsigned i = 0; i < out_h; i++) {
                for (unsigned j = 0; j < 10; j++) f << v.info[(size_t)i * 10 + j] << "\t";
                f << "\n";
            }
        }
    }
    if (frags) {
        // curve_fragment_graph::get_output_array (output type 1 of original_code/main.cpp): one
        // fragment per row, 1-based ids, as wide as the longest fragment, zero-padded
        cvl_contours_view cv;
        cvl_contours_get(frags, &cv);
        std::cout << "Link graph: " << cv.num_links << " links; contour fragments: " << cv.num_fragments
                  << " (longest " << cv.max_fragment_length << ")" << std::endl;
        std::ofstream f;
        if (!frag_file.empty() && open_out(frag_file, f)) {
            for (int64_t i = 0; i < cv.num_fragments; i++) {
                const int64_t b = cv.fragment_offsets[i], e = cv.fragment_offsets[i + 1];
                for (int64_t j = 0; j < cv.max_fragment_length; j++)
                    f << (b + j < e ? cv.fragment_ids[b + j] + 1 : 0) << "\t";
                f << "\n";
            }
        }
        if (!poly_file.empty()) {
            // output type 2 of original_code/main.cpp: polyarc chains (1-based, as wide as the
            // longest, zero-padded) and their 12 info columns (curvelet::set_output)
            std::cout << "Polyarcs: " << cv.num_polyarcs << std::endl;
            int64_t w = 0;
            for (int64_t i = 0; i < cv.num_polyarcs; i++)
                w = std::max<int64_t>(w, cv.polyarc_offsets[i + 1] - cv.polyarc_offsets[i]);
            std::ofstream pf, pi;
            if (open_out(poly_file, pf)) {
                for (int64_t i = 0; i < cv.num_polyarcs; i++) {
                    const int64_t b = cv.polyarc_offsets[i], e = cv.polyarc_offsets[i + 1];
                    for (int64_t j = 0; j < w; j++) pf << (b + j < e ? cv.polyarc_ids[b + j] + 1 : 0) << "\t";
                    pf << "\n";
                }
            }
            if (open_out(info_name(poly_file), pi)) {
                for (int64_t i = 0; i < cv.num_polyarcs; i++) {
                    for (int j = 0; j < 12; j++) pi << cv.polyarc_info[i * 12 + j] << "\t";
                    pi << "\n";
                }
            }
        }
        cvl_contours_free(frags);
    }
    cvl_result_free(res);
    cvl_engine_destroy(eng);
    return 0;
}
