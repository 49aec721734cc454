// cvl_io.cpp -- edge files: the reference's text format, read in parallel, and a
// binary format for serving (cvl_read_edges / cvl_write_edges_binary, include/cvl.h).
//
// Text (read_TO_edges_from_file, data_io.hpp:22-79): one edge per line, exactly
// values_per_edge numbers, read with `std::istream >> double`. A blank line, a
// missing number or extra data is an error with the reference's message.
//
// The fast path reads the file at once, splits it at line boundaries over
// threads, and converts each number with std::from_chars. from_chars and the
// stream extraction (glibc strtod underneath) both round correctly, so the
// values are the same. The fast path accepts only the plain token grammar: an
// optional '-', digits with at most one '.', and an optional exponent, separated
// by spaces or tabs. Everything else goes to the exact stream loop of the
// reference, for the whole file: a '+' sign, inf or nan, hex, other
// whitespace, an out-of-range value, a blank line, and every error. Results and
// messages therefore match the reference on every input.
//
// Binary (.cvle): "CVLEDGE1", uint32 values_per_edge, uint32 0, uint64
// num_edges, then num_edges * values_per_edge little-endian doubles.
#include <algorithm>
#include <charconv>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <thread>
#include <type_traits>
#include <vector>

#include "../../include/cvl.h"
#include "cvl_internal.h"

namespace {

bool blank(const std::string &s) { return s.find_first_not_of(" \t\r\n") == std::string::npos; }

// The reference's reader, line by line (data_io.hpp:38-69), for T = double or
// float (read_TO_edges_from_file<T>: `iss >> value` into a T).
template <typename T>
int read_stream(const std::string &path, int per_edge, std::vector<T> &out) {
    std::ifstream in(path);
    if (!in) return cvl_fail(CVL_EINVAL, "Error: input file does not exist: " + path);
    out.clear();
    std::string line;
    int ln = 0, count = 0;
    while (std::getline(in, line)) {
        ++ln;
        if (blank(line)) {
            out.clear();
            return cvl_fail(CVL_EINVAL, "Error: blank line at line " + std::to_string(ln) + " in " + path +
                                            " (each line must contain exactly " + std::to_string(per_edge) +
                                            " numeric values)");
        }
        std::istringstream iss(line);
        for (int j = 0; j < per_edge; j++) {
            T v;
            if (!(iss >> v)) {
                out.clear();
                return cvl_fail(CVL_EINVAL, "Error: invalid edge file format in " + path + " at line " +
                                                std::to_string(ln) + ": expected " + std::to_string(per_edge) +
                                                " numeric values per line, found " + std::to_string(j) + ".");
            }
            out.push_back(v);
        }
        std::string rest;
        std::getline(iss, rest);
        if (!blank(rest)) {
            out.clear();
            return cvl_fail(CVL_EINVAL, "Error: invalid edge file format in " + path + " at line " +
                                            std::to_string(ln) + ": expected exactly " + std::to_string(per_edge) +
                                            " numeric values per line, found extra data.");
        }
        ++count;
    }
    if (count == 0) {
        out.clear();
        return cvl_fail(CVL_EINVAL, "Error: input file contains no valid edges: " + path);
    }
    return CVL_OK;
}

inline bool digit(char c) { return c >= '0' && c <= '9'; }

// One plain token at p (no leading whitespace): '-'? digits ('.' digits?)? or
// '.' digits, then ([eE] [+-]? digits)?. Returns its end, or nullptr.
const char *plain_token(const char *p, const char *end) {
    const char *q = p;
    if (q < end && *q == '-') ++q;
    const char *d0 = q;
    while (q < end && digit(*q)) ++q;
    bool any = q > d0;
    if (q < end && *q == '.') {
        ++q;
        const char *f0 = q;
        while (q < end && digit(*q)) ++q;
        any = any || q > f0;
    }
    if (!any) return nullptr;
    if (q < end && (*q == 'e' || *q == 'E')) {
        const char *e = q + 1;
        if (e < end && (*e == '+' || *e == '-')) ++e;
        const char *e0 = e;
        while (e < end && digit(*e)) ++e;
        if (e == e0) return nullptr;
        q = e;
    }
    return q;
}

// Lines [b, e) of the buffer, all plain: values appended to out. false sends the
// whole file to the exact reader.
template <typename T>
bool parse_plain(const char *b, const char *e, int per_edge, std::vector<T> &out, long long &lines) {
    const char *p = b;
    while (p < e) {
        const char *nl = (const char *)std::memchr(p, '\n', (size_t)(e - p));
        const char *le = nl ? nl : e;
        const char *q = p;
        for (int j = 0; j < per_edge; ++j) {
            while (q < le && (*q == ' ' || *q == '\t')) ++q;
            const char *t = plain_token(q, le);
            if (!t) return false;
            T v;
            const auto r = std::from_chars(q, t, v, std::chars_format::general);
            if (r.ec != std::errc() || r.ptr != t) return false;
            // the token must end at a separator (a stream would read "1.5x" as 1.5
            // and then fail; such input goes to the exact reader)
            if (t < le && *t != ' ' && *t != '\t') return false;
            out.push_back(v);
            q = t;
        }
        while (q < le && (*q == ' ' || *q == '\t')) ++q;
        if (q != le) return false;
        ++lines;
        p = nl ? nl + 1 : e;
    }
    return true;
}

template <typename T>
int read_text(const std::string &path, int per_edge, int nthreads, std::vector<T> &out) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return cvl_fail(CVL_EINVAL, "Error: input file does not exist: " + path);
    std::string buf;
    if (std::fseek(f, 0, SEEK_END) == 0) {
        const long sz = std::ftell(f);
        if (sz > 0) {
            buf.resize((size_t)sz);
            std::fseek(f, 0, SEEK_SET);
            if (std::fread(&buf[0], 1, buf.size(), f) != buf.size()) buf.clear();
        }
    }
    std::fclose(f);
    if (buf.empty()) return read_stream(path, per_edge, out);
    // a file that ends in '\n' has no empty last line for getline
    const char *b = buf.data(), *e = buf.data() + buf.size();
    const char *body_end = (e[-1] == '\n') ? e - 1 : e;
    // an empty body, or one that still ends in '\n' (an empty last line), goes to the
    // exact reader
    if (body_end == b || body_end[-1] == '\n') return read_stream(path, per_edge, out);
    const int NT = std::max(1, std::min(nthreads, (int)((body_end - b) >> 16) + 1));
    std::vector<const char *> cut(NT + 1);
    cut[0] = b;
    cut[NT] = body_end;
    for (int t = 1; t < NT; ++t) {
        const char *s = b + (size_t)(body_end - b) * t / NT;
        if (s < cut[t - 1]) s = cut[t - 1];
        const char *nl = (const char *)std::memchr(s, '\n', (size_t)(body_end - s));
        cut[t] = nl ? nl + 1 : body_end;
    }
    std::vector<std::vector<T>> parts(NT);
    std::vector<long long> lines(NT, 0);
    std::vector<char> ok(NT, 0);
    // a chunk ends just after a '\n' (the last one at the body's end): each of its
    // lines ends in '\n' or at the chunk's end, and an empty line fails the grammar
    auto work = [&](int t) { ok[t] = parse_plain(cut[t], cut[t + 1], per_edge, parts[t], lines[t]) ? 1 : 0; };
    std::vector<std::thread> th;
    for (int t = 1; t < NT; ++t) th.emplace_back(work, t);
    work(0);
    for (std::thread &x : th) x.join();
    long long n = 0;
    for (int t = 0; t < NT; ++t) {
        if (!ok[t]) return read_stream(path, per_edge, out);
        n += lines[t];
    }
    if (n == 0) return read_stream(path, per_edge, out);
    out.clear();
    out.reserve((size_t)n * per_edge);
    for (auto &p : parts) out.insert(out.end(), p.begin(), p.end());
    return CVL_OK;
}

constexpr char MAGIC[8] = {'C', 'V', 'L', 'E', 'D', 'G', 'E', '1'};

bool ends_with(const std::string &s, const char *suf) {
    const size_t k = std::strlen(suf);
    return s.size() >= k && s.compare(s.size() - k, k, suf) == 0;
}

int read_binary(const std::string &path, int per_edge, std::vector<double> &out) {
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) return cvl_fail(CVL_EINVAL, "Error: input file does not exist: " + path);
    char magic[8];
    uint32_t vpe = 0, zero = 0;
    uint64_t n = 0;
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, MAGIC, 8) == 0 && std::fread(&vpe, 4, 1, f) == 1 &&
              std::fread(&zero, 4, 1, f) == 1 && std::fread(&n, 8, 1, f) == 1;
    if (!ok) {
        std::fclose(f);
        return cvl_fail(CVL_EINVAL, "Error: not a binary edge file: " + path);
    }
    if ((int)vpe != per_edge) {
        std::fclose(f);
        return cvl_fail(CVL_EINVAL, "Error: binary edge file " + path + " has " + std::to_string(vpe) +
                                        " values per edge, expected " + std::to_string(per_edge));
    }
    if (n == 0 || n > (uint64_t)0x7fffffff) {
        std::fclose(f);
        return cvl_fail(CVL_EINVAL, "Error: input file contains no valid edges: " + path);
    }
    out.resize((size_t)n * vpe);
    const bool full = std::fread(out.data(), sizeof(double), out.size(), f) == out.size();
    std::fclose(f);
    if (!full) {
        out.clear();
        return cvl_fail(CVL_EINVAL, "Error: binary edge file is truncated: " + path);
    }
    return CVL_OK;
}

}  // namespace

template <typename T>
static int read_edges_t(const char *path, int32_t values_per_edge, int32_t nthreads, T **edges, int64_t *num_edges) {
    if (!path || !edges || !num_edges || values_per_edge < 4) return cvl_fail(CVL_EINVAL, "invalid arguments");
    *edges = nullptr;
    *num_edges = 0;
    const std::string p(path);
    std::vector<T> v;
    int rc;
    if (ends_with(p, ".cvle")) {
        if constexpr (std::is_same<T, double>::value)
            rc = read_binary(p, values_per_edge, v);
        else
            return cvl_fail(CVL_EINVAL, "the binary edge format holds doubles; read it with cvl_read_edges");
    } else if (nthreads < 0) {
        rc = read_stream(p, values_per_edge, v);
    } else {
        const int nt = nthreads > 0 ? nthreads : (int)std::max(1u, std::thread::hardware_concurrency());
        rc = read_text(p, values_per_edge, nt, v);
    }
    if (rc != CVL_OK) return rc;
    T *buf = (T *)std::malloc(sizeof(T) * v.size());
    if (!buf) return cvl_fail(CVL_ENOMEM, "host allocation failed");
    std::memcpy(buf, v.data(), sizeof(T) * v.size());
    *edges = buf;
    *num_edges = (int64_t)(v.size() / (size_t)values_per_edge);
    return CVL_OK;
}

extern "C" {

int cvl_read_edges(const char *path, int32_t values_per_edge, int32_t nthreads, double **edges, int64_t *num_edges) {
    return read_edges_t<double>(path, values_per_edge, nthreads, edges, num_edges);
}

int cvl_read_edges_f32(const char *path, int32_t values_per_edge, int32_t nthreads, float **edges,
                       int64_t *num_edges) {
    return read_edges_t<float>(path, values_per_edge, nthreads, edges, num_edges);
}

void cvl_free_edges(void *edges) { std::free(edges); }

int cvl_write_edges_binary(const char *path, const double *edges, int64_t num_edges, int32_t values_per_edge) {
    if (!path || !edges || num_edges <= 0 || num_edges > 0x7fffffff || values_per_edge < 4)
        return cvl_fail(CVL_EINVAL, "invalid arguments");
    std::FILE *f = std::fopen(path, "wb");
    if (!f) return cvl_fail(CVL_EINVAL, std::string("cannot open for writing: ") + path);
    const uint32_t vpe = (uint32_t)values_per_edge, zero = 0;
    const uint64_t n = (uint64_t)num_edges;
    bool ok = std::fwrite(MAGIC, 1, 8, f) == 8 && std::fwrite(&vpe, 4, 1, f) == 1 && std::fwrite(&zero, 4, 1, f) == 1 &&
              std::fwrite(&n, 8, 1, f) == 1 &&
              std::fwrite(edges, sizeof(double), (size_t)n * vpe, f) == (size_t)n * vpe;
    ok = (std::fclose(f) == 0) && ok;
    return ok ? CVL_OK : cvl_fail(CVL_EINVAL, std::string("write failed: ") + path);
}

}  // extern "C"
