// cvl_contours.cuh -- downstream of the curvelet path: the edgel link graph and
// its contour fragments ("one-chains"), as the reference's original_code builds
// them from a curvelet map:
//   construct_the_link_graph / form_links_from_a_curvelet
//       (original_code/form_curvelet_process.cpp:453-520)
//   link_edgels / are_linked / edgel_is_legal_first_edgel / edgel_is_legal
//       (original_code/edgel_link_graph.hpp:207-265)
//   extract_one_chains_from_the_link_graph (form_curvelet_process.cpp:563-654)
//   curve_fragment_graph::insert_fragment / get_output_array (curve_fragment_graph.hpp)
//
// What decides the result:
//  * A link joins two edgels in either direction (are_linked looks both ways).
//    Its direction is the one of its first occurrence, in the order curvelets
//    are visited: anchors ascending, each anchor's curvelets in record order,
//    each chain's consecutive pairs in order. So every occurrence gets the index
//    occ = row * (W - 1) + k, and each edge's bucket of occurrences decides its
//    links locally: the entry with the smallest occ per neighbour gives the
//    direction; votes count every entry.
//  * Tracing only ever takes front() of a list of exactly one link, so the
//    in/out degree, the single parent and the single child of each edge are all
//    the tracer needs.
//  * "Legal" (in <= 1, out <= 1, not linked) has a static part. Edges that pass
//    it, joined by links between two of them, form disjoint simple paths and
//    cycles. A trace marks edges of its own component only, so components are
//    independent: one thread per component replays the reference's loop over
//    start edges in ascending id order, restricted to its component. Fragments
//    are then written in start-id order, which is the reference's order.
#pragma once

#include <cstdint>

namespace cvlc {

constexpr unsigned DIR_OUT = 0x80000000u;    // bucket entry: the link leaves this edge
constexpr unsigned FIRST_OCC = 0x40000000u;  // bucket entry: the first occurrence of its link
constexpr unsigned ID_MASK = 0x3fffffffu;    // edge ids below 2^30

enum : unsigned char { F_LEGAL = 1, F_FIRST = 2, F_SEEN = 4 };

constexpr unsigned ERR_ID = 1u;       // a chain id outside the map
constexpr unsigned ERR_SCRATCH = 2u;  // scratch sizing violated (never expected)

struct Graph {
    int n;
    const unsigned long long *occ_off;  // [n + 1]
    uint2 *bucket;                      // (other | DIR_OUT | FIRST_OCC, occ)
    int *outdeg, *indeg, *child, *parent;
    int *succ, *pred;
    unsigned char *flags, *linked;
};

// row length of a chain row (column 0 is the anchor)
__device__ __forceinline__ int chain_len(const unsigned *row, int W) {
    int len = 0;
    while (len < W - 1 && row[1 + len] != 0u) ++len;
    return len;
}

// ---- 1. occurrences per edge -----------------------------------------------------
__global__ void k_link_count(const unsigned *chains, long long C, int W, unsigned min_group, int n,
                             unsigned *occ_cnt, unsigned *err) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= C) return;
    const unsigned *row = chains + r * W;
    const int len = chain_len(row, W);
    for (int k = 0; k < len; ++k)  // every row's ids, linked or not
        if (row[1 + k] - 1u >= (unsigned)n) {
            atomicOr(err, ERR_ID);
            return;
        }
    if ((unsigned)len < min_group) return;
    for (int k = 0; k + 1 < len; ++k) {
        const unsigned u = row[1 + k] - 1u, v = row[2 + k] - 1u;
        atomicAdd(&occ_cnt[u], 1u);
        atomicAdd(&occ_cnt[v], 1u);
    }
}

__global__ void k_link_fill(const unsigned *chains, long long C, int W, unsigned min_group, int n,
                            const unsigned long long *occ_off, unsigned *cursor, uint2 *bucket) {
    const long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= C) return;
    const unsigned *row = chains + r * W;
    const int len = chain_len(row, W);
    if ((unsigned)len < min_group) return;
    for (int k = 0; k < len; ++k)  // a row k_link_count rejected adds nothing, as there
        if (row[1 + k] - 1u >= (unsigned)n) return;
    for (int k = 0; k + 1 < len; ++k) {
        const unsigned u = row[1 + k] - 1u, v = row[2 + k] - 1u;
        const unsigned occ = (unsigned)(r * (W - 1) + k);
        const unsigned pu = atomicAdd(&cursor[u], 1u);
        bucket[occ_off[u] + pu] = make_uint2(v | DIR_OUT, occ);
        const unsigned pv = atomicAdd(&cursor[v], 1u);
        bucket[occ_off[v] + pv] = make_uint2(u, occ);
    }
}

// is entry i the first occurrence of its link within the bucket?
__device__ __forceinline__ bool first_of_link(const uint2 *b, unsigned m, unsigned i) {
    const unsigned w = b[i].x & ID_MASK, occ = b[i].y;
    for (unsigned j = 0; j < m; ++j)
        if ((b[j].x & ID_MASK) == w && b[j].y < occ) return false;
    return true;
}

// ---- 2. degrees, the single child / parent ----------------------------------------
__global__ void k_link_degrees(Graph g) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= g.n) return;
    uint2 *b = g.bucket + g.occ_off[u];
    const unsigned m = (unsigned)(g.occ_off[u + 1] - g.occ_off[u]);
    int od = 0, id = 0, ch = -1, pa = -1;
    for (unsigned i = 0; i < m; ++i) {
        if (!first_of_link(b, m, i)) continue;
        b[i].x |= FIRST_OCC;  // only this thread touches edge u's bucket
        if (b[i].x & DIR_OUT) {
            ++od;
            ch = (int)(b[i].x & ID_MASK);
        } else {
            ++id;
            pa = (int)(b[i].x & ID_MASK);
        }
    }
    g.outdeg[u] = od;
    g.indeg[u] = id;
    g.child[u] = ch;
    g.parent[u] = pa;
    unsigned char f = 0;
    if (od <= 1 && id <= 1) f |= F_LEGAL;                  // edgel_is_legal, static part
    if (od == 1 && id == 1 && pa != ch) f |= F_FIRST;      // edgel_is_legal_first_edgel, static part
    g.flags[u] = f;
    g.linked[u] = 0;
}

// the links leaving each edge in creation order (_cLinks), with their votes
__global__ void k_link_list(Graph g, const unsigned long long *link_off, int *pe, int *ce, int *votes) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= g.n) return;
    const uint2 *b = g.bucket + g.occ_off[u];
    const unsigned m = (unsigned)(g.occ_off[u + 1] - g.occ_off[u]);
    const unsigned long long base = link_off[u];
    constexpr unsigned OUT_FIRST = DIR_OUT | FIRST_OCC;
    for (unsigned i = 0; i < m; ++i) {
        if ((b[i].x & OUT_FIRST) != OUT_FIRST) continue;
        const unsigned w = b[i].x & ID_MASK;
        unsigned rank = 0, vote = 0;
        for (unsigned j = 0; j < m; ++j) {
            const unsigned wj = b[j].x & ID_MASK;
            if (wj == w) ++vote;
            else if ((b[j].x & OUT_FIRST) == OUT_FIRST && b[j].y < b[i].y) ++rank;
        }
        pe[base + rank] = u;
        ce[base + rank] = (int)w;
        votes[base + rank] = (int)vote;
    }
}

// ---- 3. component structure --------------------------------------------------------
__global__ void k_link_paths(Graph g) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= g.n) return;
    int s = -1, p = -1;
    if (g.flags[u] & F_LEGAL) {
        if (g.outdeg[u] == 1 && (g.flags[g.child[u]] & F_LEGAL)) s = g.child[u];
        if (g.indeg[u] == 1 && (g.flags[g.parent[u]] & F_LEGAL)) p = g.parent[u];
    }
    g.succ[u] = s;
    g.pred[u] = p;
}

struct FragOut {
    const double *edges;  // AoS [n][sz]: x, y in columns 0, 1
    int sz;
    double thres;         // gap * gap
    unsigned *first_ids;  // scratch for each component's start edges
    unsigned long long *first_ctr;
    int *region;          // fragment ids beyond the start edge: forward part, then backward part
    unsigned long long *region_ctr;
    unsigned long long region_cap, first_cap;
    unsigned long long *frag_src;  // per start edge: offset into region
    int *frag_nf, *frag_nb;        // per start edge: forward / backward counts (frag_nf = -1: no fragment)
    unsigned *err;
};

// sq_distance (original_code/curvelet_utils.hpp:17-20); the library builds with -fmad=false
__device__ __forceinline__ double pt_sqd(const FragOut &o, int a, int b) {
    const double *A = o.edges + (size_t)a * o.sz, *B = o.edges + (size_t)b * o.sz;
    return (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]);
}

__device__ void heap_sift(unsigned *a, long long i, long long n) {
    for (;;) {
        long long c = 2 * i + 1;
        if (c >= n) return;
        if (c + 1 < n && a[c + 1] > a[c]) ++c;
        if (a[i] >= a[c]) return;
        const unsigned t = a[i];
        a[i] = a[c];
        a[c] = t;
        i = c;
    }
}

__device__ void heap_sort(unsigned *a, long long n) {
    for (long long i = n / 2 - 1; i >= 0; --i) heap_sift(a, i, n);
    for (long long e = n - 1; e > 0; --e) {
        const unsigned t = a[0];
        a[0] = a[e];
        a[e] = t;
        heap_sift(a, 0, e);
    }
}

// Replays extract_one_chains_from_the_link_graph over one component (entered at
// `start`: a path's head, or a cycle's smallest id), start edges ascending.
// Region bound: a trace pushes, on each side, at most one edge it does not mark
// (the step that ends it) besides the edges it marks; every edge of the component
// is marked at most once and the start edge is not stored. So a component of m
// edges and f start edges stores at most m + f ids; m + 2f are reserved.
__device__ void trace_component(const Graph &g, const FragOut &o, int start) {
    long long m = 0, f = 0;
    int v = start;
    do {
        ++m;
        if (g.flags[v] & F_FIRST) ++f;
        v = g.succ[v];
    } while (v >= 0 && v != start);
    if (f == 0) return;
    const unsigned long long fb = atomicAdd(o.first_ctr, (unsigned long long)f);
    const unsigned long long rb = atomicAdd(o.region_ctr, (unsigned long long)(m + 2 * f));
    if (fb + f > o.first_cap || rb + m + 2 * f > o.region_cap) {
        atomicOr(o.err, ERR_SCRATCH);
        return;
    }
    unsigned *firsts = o.first_ids + fb;
    long long k = 0;
    v = start;
    do {
        if (g.flags[v] & F_FIRST) firsts[k++] = (unsigned)v;
        v = g.succ[v];
    } while (v >= 0 && v != start);
    heap_sort(firsts, f);
    int *out = o.region + rb;
    long long cur = 0;
    const long long cap = m + 2 * f;
#define CVLC_LEGAL(e) ((g.flags[e] & F_LEGAL) && !g.linked[e])
#define CVLC_PUT(e)                                  \
    do {                                             \
        if (cur >= cap) {                            \
            atomicOr(o.err, ERR_SCRATCH);            \
            return;                                  \
        }                                            \
        out[cur++] = (e);                            \
    } while (0)
    for (long long q = 0; q < f; ++q) {
        const int s = (int)firsts[q];
        if (g.linked[s]) continue;
        const long long src = cur;
        int nf = 0, nb = 0;
        g.linked[s] = 1;
        int eA = g.child[s], eB;
        if (pt_sqd(o, s, eA) < o.thres) {
            CVLC_PUT(eA);
            ++nf;
        }
        while (CVLC_LEGAL(eA)) {
            g.linked[eA] = 1;
            if (g.outdeg[eA] == 0) break;
            eB = eA;
            eA = g.child[eA];
            if (pt_sqd(o, eB, eA) < o.thres) {
                CVLC_PUT(eA);
                ++nf;
            } else {
                break;
            }
        }
        if (eA != s) {
            eA = g.parent[s];
            if (pt_sqd(o, s, eA) < o.thres) {
                CVLC_PUT(eA);
                ++nb;
            }
        }
        while (CVLC_LEGAL(eA)) {
            g.linked[eA] = 1;
            if (g.indeg[eA] == 0) break;
            eB = eA;
            eA = g.parent[eA];
            if (pt_sqd(o, eB, eA) < o.thres) {
                CVLC_PUT(eA);
                ++nb;
            } else {
                break;
            }
        }
        o.frag_src[s] = rb + src;
        o.frag_nf[s] = nf;
        o.frag_nb[s] = nb;
    }
#undef CVLC_PUT
#undef CVLC_LEGAL
}

// components that are paths: entered at their head (no legal predecessor)
__global__ void k_trace_paths(Graph g, FragOut o) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= g.n) return;
    if (!(g.flags[u] & F_LEGAL) || g.pred[u] >= 0) return;
    for (int v = u; v >= 0; v = g.succ[v]) g.flags[v] |= F_SEEN;
    trace_component(g, o, u);
}

// components that are cycles (legal edges no head reached): entered at their
// smallest id, found by walking both ways until a smaller id shows up
__global__ void k_trace_cycles(Graph g, FragOut o) {
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u >= g.n) return;
    if (!(g.flags[u] & F_LEGAL) || (g.flags[u] & F_SEEN)) return;
    int a = g.succ[u], b = g.pred[u];
    for (;;) {
        if (a < 0 || b < 0) return;  // not a cycle (cannot happen for an unseen legal edge)
        if (a == u) break;           // walked all the way round: u is the smallest
        if (a < u || b < u) return;
        if (a == b) break;           // the two walks met
        a = g.succ[a];
        if (a == u) break;
        if (a < u) return;
        if (a == b) break;
        b = g.pred[b];
    }
    trace_component(g, o, u);
}

// ---- 4. fragments in start order ------------------------------------------------------
__global__ void k_frag_sizes(int n, const int *frag_nf, const int *frag_nb, unsigned *is_frag,
                             unsigned long long *frag_len) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const int nf = frag_nf[s];
    const long long len = nf < 0 ? 0 : 1LL + nf + frag_nb[s];
    const bool keep = len > 2;  // "prune out the short ones"
    is_frag[s] = keep ? 1u : 0u;
    frag_len[s] = keep ? (unsigned long long)len : 0ull;
}

__global__ void k_frag_write(int n, const int *frag_nf, const int *frag_nb, const unsigned long long *frag_src,
                             const int *region, const unsigned *frag_idx, const unsigned long long *id_off,
                             long long *frag_offsets, int *frag_ids) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const long long len = frag_nf[s] < 0 ? 0 : 1LL + frag_nf[s] + frag_nb[s];
    if (s == n - 1) frag_offsets[frag_idx[n]] = (long long)id_off[n];
    if (len <= 2) return;
    const int nf = frag_nf[s], nb = frag_nb[s];
    const int *src = region + frag_src[s];
    int *dst = frag_ids + id_off[s];
    frag_offsets[frag_idx[s]] = (long long)id_off[s];
    for (int q = 0; q < nb; ++q) dst[q] = src[nf + nb - 1 - q];  // the backward part, pushed to the front
    dst[nb] = s;
    for (int q = 0; q < nf; ++q) dst[nb + 1 + q] = src[q];
}

}  // namespace cvlc
