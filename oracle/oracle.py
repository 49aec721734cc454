"""ctypes front end of the CPU checker -- TEST INFRASTRUCTURE ONLY.

Loads ``oracle/libcvl_oracle.so`` (the C restatement of the reference path,
``oracle/cvl_oracle.c``) and, when it was built, ``oracle/_ref/libcvlref.so``
(the reference's own cpu_curvelet templates behind ``oracle/ref_harness.cpp``).
Only tests/, ``__graft_entry__.smoke()`` and bench.py's cpu_baseline /
reference legs import this module; the engine never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "libcvl_oracle.so")
REF_SO = os.path.join(HERE, "_ref", "libcvlref.so")
REF_CLI = os.path.join(HERE, "_ref", "CURVELET")
ORIG_SO = os.path.join(HERE, "_ref", "liborigref.so")

# reference defaults, cpu_curvelet/param_settings.hpp:9-24
DEFAULTS = dict(nrad=3.5, dx=0.4, dt_deg=15.0, max_k=0.3, sx=0.1, st=0.08,
                group_max_sz=4, max_candidates=128)


def build(quiet: bool = True) -> None:
    """Builds the restatement (and the reference leg when its sources exist)."""
    out = subprocess.run(["make", "-C", HERE], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


class _OrcCsr(C.Structure):
    _fields_ = [("num_edges", C.c_int), ("total_neighbor_pairs", C.c_int),
                ("max_num_of_neighbors", C.c_uint), ("truncated_anchors", C.c_uint),
                ("tie_anchors", C.c_uint),
                ("neighbor_offsets", C.POINTER(C.c_int)), ("neighbor_ids", C.POINTER(C.c_int)),
                ("neighbor_dist2", C.POINTER(C.c_double))]


class _OrcResult(C.Structure):
    _fields_ = [("num_edges", C.c_int), ("total_neighbor_pairs", C.c_int),
                ("max_num_of_neighbors", C.c_uint), ("truncated_anchors", C.c_uint),
                ("tie_anchors", C.c_uint), ("valid_pairs", C.c_uint),
                ("num_curvelets", C.c_uint), ("chain_width", C.c_uint),
                ("chains", C.POINTER(C.c_uint)), ("info", C.POINTER(C.c_double)),
                ("anchor_count", C.POINTER(C.c_uint))]


class _RefOut(C.Structure):
    _fields_ = [("num_edges", C.c_int), ("total_neighbor_pairs", C.c_int),
                ("max_num_of_neighbors", C.c_uint), ("valid_pairs", C.c_uint),
                ("num_curvelets", C.c_uint), ("chain_width", C.c_uint),
                ("neighbor_offsets", C.POINTER(C.c_int)), ("neighbor_ids", C.POINTER(C.c_int)),
                ("neighbor_dist2", C.POINTER(C.c_double)),
                ("chains", C.POINTER(C.c_uint)), ("info", C.POINTER(C.c_double)),
                ("ms_csr", C.c_double), ("ms_pairwise", C.c_double), ("ms_greedy", C.c_double)]


@dataclass
class Csr:
    offsets: np.ndarray
    ids: np.ndarray
    dist2: np.ndarray
    max_deg: int
    truncated_anchors: int = 0
    tie_anchors: int = 0


@dataclass
class Result:
    """The observable outputs of one run: chains (uint32, 1-based ids, rows of
    group_max_sz + 1) and info (float64, rows of 10), plus the path's counters."""
    chains: np.ndarray
    info: np.ndarray
    valid_pairs: int
    total_neighbor_pairs: int
    max_num_of_neighbors: int
    truncated_anchors: int = 0
    tie_anchors: int = 0
    anchor_count: np.ndarray | None = None
    csr: Csr | None = None
    ms: dict = field(default_factory=dict)

    @property
    def num_curvelets(self) -> int:
        return int(self.chains.shape[0])


def _arr(ptr, n, dtype):
    if n == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(n,)).astype(dtype, copy=True)


_lib = None
_ref = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = C.CDLL(ORACLE_SO)
        dp = C.POINTER(C.c_double)
        L.orc_build_csr.argtypes = [dp, C.c_int, C.c_int, C.c_double, C.c_uint, C.c_uint, C.c_int,
                                    C.POINTER(_OrcCsr)]
        L.orc_csr_free.argtypes = [C.POINTER(_OrcCsr)]
        L.orc_run.argtypes = [dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                              C.c_double, C.c_double, C.c_uint, C.c_uint, C.c_int, C.POINTER(_OrcResult)]
        L.orc_result_free.argtypes = [C.POINTER(_OrcResult)]
        L.orc_pair_bundle.argtypes = [C.c_double] * 12 + [dp, dp, C.POINTER(C.c_int)]
        _lib = L
    return _lib


def ref_available() -> bool:
    return os.path.exists(REF_SO)


def ref_lib():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError("reference harness not built: " + REF_SO)
        L = C.CDLL(REF_SO)
        dp = C.POINTER(C.c_double)
        L.cvlref_run.argtypes = [dp, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                 C.c_double, C.c_double, C.c_uint, C.c_uint, C.c_int, C.c_int, C.c_int,
                                 C.POINTER(_RefOut)]
        L.cvlref_run_f32.argtypes = [C.POINTER(C.c_float)] + L.cvlref_run.argtypes[1:]
        L.cvlref_free.argtypes = [C.POINTER(_RefOut)]
        L.cvlref_pair_bundle.argtypes = [C.c_double] * 12 + [dp, dp, C.POINTER(C.c_int)]
        ip = C.POINTER(C.c_int)
        L.cvlref_run_csr.argtypes = [dp, C.c_int, C.c_int] + [C.c_double] * 6 + [C.c_uint, C.c_uint, ip, ip,
                                                                               C.POINTER(_RefOut)]
        L.cvlref_run_csr_f32.argtypes = [C.POINTER(C.c_float)] + L.cvlref_run_csr.argtypes[1:]
        _ref = L
    return _ref


def _edges_arg(edges):
    e = np.ascontiguousarray(edges, dtype=np.float64)
    assert e.ndim == 2 and e.shape[1] >= 4
    return e, e.ctypes.data_as(C.POINTER(C.c_double)), e.shape[0], e.shape[1]


def build_csr(edges, nrad=3.5, neighbor_radius=3, max_candidates=128, nthreads=1) -> Csr:
    e, p, n, sz = _edges_arg(edges)
    g = _OrcCsr()
    rc = lib().orc_build_csr(p, n, sz, nrad, neighbor_radius, max_candidates, nthreads, C.byref(g))
    if rc != 0:
        raise ValueError("orc_build_csr rejected the input")
    try:
        np_ = g.total_neighbor_pairs
        return Csr(_arr(g.neighbor_offsets, n + 1, np.int32), _arr(g.neighbor_ids, np_, np.int32),
                   _arr(g.neighbor_dist2, np_, np.float64), int(g.max_num_of_neighbors),
                   int(g.truncated_anchors), int(g.tie_anchors))
    finally:
        lib().orc_csr_free(C.byref(g))


def run(edges, nthreads=1, **params) -> Result:
    """The restatement over one edge map (AoS rows of >= 4 values)."""
    p = dict(DEFAULTS, **params)
    e, ptr, n, sz = _edges_arg(edges)
    r = _OrcResult()
    rc = lib().orc_run(ptr, n, sz, p["nrad"], p["dx"], p["dt_deg"], p["max_k"], p["sx"], p["st"],
                       p["group_max_sz"], p["max_candidates"], nthreads, C.byref(r))
    if rc != 0:
        raise ValueError(f"orc_run failed ({rc})")
    try:
        w = r.chain_width
        nc = r.num_curvelets
        return Result(_arr(r.chains, nc * w, np.uint32).reshape(nc, w),
                      _arr(r.info, nc * 10, np.float64).reshape(nc, 10),
                      int(r.valid_pairs), int(r.total_neighbor_pairs), int(r.max_num_of_neighbors),
                      int(r.truncated_anchors), int(r.tie_anchors),
                      _arr(r.anchor_count, n, np.uint32))
    finally:
        lib().orc_result_free(C.byref(r))


def ref_run(edges, nthreads=1, want_outputs=True, scalar="double", **params) -> Result:
    """The reference's own cpu_curvelet code over one edge map: run_curvelet<double>,
    or run_curvelet<float> (its --float mode) for scalar="float", which takes the
    edges as float32 (convert them the way the reference reads them: float32
    values, as from parse_edges_f32)."""
    p = dict(DEFAULTS, **params)
    r = _RefOut()
    if scalar == "float":
        e = np.ascontiguousarray(edges, dtype=np.float32)
        assert e.ndim == 2 and e.shape[1] >= 4
        n, sz = e.shape
        rc = ref_lib().cvlref_run_f32(e.ctypes.data_as(C.POINTER(C.c_float)), n, sz, p["nrad"], p["dx"],
                                      p["dt_deg"], p["max_k"], p["sx"], p["st"], p["group_max_sz"],
                                      p["max_candidates"], nthreads, 1, int(want_outputs), C.byref(r))
    else:
        e, ptr, n, sz = _edges_arg(edges)
        rc = ref_lib().cvlref_run(ptr, n, sz, p["nrad"], p["dx"], p["dt_deg"], p["max_k"], p["sx"], p["st"],
                                  p["group_max_sz"], p["max_candidates"], nthreads, 1, int(want_outputs),
                                  C.byref(r))
    if rc != 0:
        raise ValueError(f"cvlref_run failed ({rc})")
    try:
        w, nc, np_ = r.chain_width, r.num_curvelets, r.total_neighbor_pairs
        ms = dict(csr=r.ms_csr, pairwise=r.ms_pairwise, greedy=r.ms_greedy)
        if not want_outputs:
            return Result(np.zeros((0, w), np.uint32), np.zeros((0, 10)), int(r.valid_pairs), np_,
                          int(r.max_num_of_neighbors), ms=ms)
        csr = Csr(_arr(r.neighbor_offsets, n + 1, np.int32), _arr(r.neighbor_ids, np_, np.int32),
                  _arr(r.neighbor_dist2, np_, np.float64), int(r.max_num_of_neighbors))
        return Result(_arr(r.chains, nc * w, np.uint32).reshape(nc, w),
                      _arr(r.info, nc * 10, np.float64).reshape(nc, 10),
                      int(r.valid_pairs), np_, int(r.max_num_of_neighbors), csr=csr, ms=ms)
    finally:
        ref_lib().cvlref_free(C.byref(r))


def ref_run_csr(edges, offsets, ids, scalar="double", **params) -> Result:
    """The reference's CurveletCPU stage (form_pairwise_bundles, build_curvelets_greedy,
    cpu_curvelet.hpp:305-634) run on the given neighbour lists instead of the ones
    build_neighbor_csr_graph makes: the reference's own answer for a chosen CSR,
    e.g. one whose truncated anchors keep the lowest edge indices of a pixel cell."""
    p = dict(DEFAULTS, **params)
    off = np.ascontiguousarray(offsets, dtype=np.int32)
    nid = np.ascontiguousarray(ids, dtype=np.int32)
    ip = C.POINTER(C.c_int)
    r = _RefOut()
    if scalar == "float":
        e = np.ascontiguousarray(edges, dtype=np.float32)
        f, ptr = ref_lib().cvlref_run_csr_f32, e.ctypes.data_as(C.POINTER(C.c_float))
    else:
        e = np.ascontiguousarray(edges, dtype=np.float64)
        f, ptr = ref_lib().cvlref_run_csr, e.ctypes.data_as(C.POINTER(C.c_double))
    n, sz = e.shape
    assert off.shape == (n + 1,) and nid.shape == (int(off[-1]),)
    rc = f(ptr, n, sz, p["nrad"], p["dx"], p["dt_deg"], p["max_k"], p["sx"], p["st"], p["group_max_sz"],
           p["max_candidates"], off.ctypes.data_as(ip), nid.ctypes.data_as(ip), C.byref(r))
    if rc != 0:
        raise ValueError(f"cvlref_run_csr failed ({rc})")
    try:
        w, nc, np_ = r.chain_width, r.num_curvelets, r.total_neighbor_pairs
        csr = Csr(_arr(r.neighbor_offsets, n + 1, np.int32), _arr(r.neighbor_ids, np_, np.int32),
                  _arr(r.neighbor_dist2, np_, np.float64), int(r.max_num_of_neighbors))
        return Result(_arr(r.chains, nc * w, np.uint32).reshape(nc, w),
                      _arr(r.info, nc * 10, np.float64).reshape(nc, 10),
                      int(r.valid_pairs), np_, int(r.max_num_of_neighbors), csr=csr)
    finally:
        ref_lib().cvlref_free(C.byref(r))


def build_csr_f32(edges, nrad=3.5, neighbor_radius=3, max_candidates=128) -> Csr:
    """The neighbour CSR of run_curvelet<float> (preprocess.hpp:62-274 with T = float),
    restated in numpy float32 arithmetic, for small maps. Pixel cells are
    (lrint(x), lrint(y)) of the float coordinates (:84-86); a candidate is an edge of
    a cell of the (2w+1)^2 window, scanned py outer and px inner (:137-138), whose
    float squared distance, ((x1-x2)*(x1-x2)) + ((y1-y2)*(y1-y2)) (curvelet_utils.hpp:14-17),
    is <= rad*rad, a float product (:223, :157-160); the first max_candidates in scan
    order are kept (:162-164) and sorted by distance (:168-173). Inside a cell, edges
    come in ascending index, and equal distances keep scan order: the orders the
    reference's unstable std::sort leaves to libstdc++ (:90-92, :168) are fixed the
    same way as in the C restatement of the FP64 path (orc_build_csr)."""
    e = np.ascontiguousarray(edges, dtype=np.float32)
    n = e.shape[0]
    if n <= 0 or e.shape[1] < 4:
        raise ValueError("build_csr_f32 takes a non-empty map of >= 4 values per edge")
    x, y = e[:, 0], e[:, 1]
    cx = np.rint(x).astype(np.int64)
    cy = np.rint(y).astype(np.int64)
    cells: dict = {}
    for i in range(n):
        cells.setdefault((int(cx[i]), int(cy[i])), []).append(i)
    cells = {k: np.array(v, np.int64) for k, v in cells.items()}
    rad = np.float32(nrad)
    rad_sqr = np.float32(rad * rad)
    w = int(neighbor_radius)
    offs = [0]
    ids_out, d2_out = [], []
    maxdeg = truncated = ties = 0
    for te in range(n):
        scan = [cells[(px, py)] for py in range(int(cy[te]) - w, int(cy[te]) + w + 1)
                for px in range(int(cx[te]) - w, int(cx[te]) + w + 1) if (px, py) in cells]
        cand = np.concatenate(scan) if scan else np.zeros(0, np.int64)
        cand = cand[cand != te]
        dxs = x[te] - x[cand]
        dys = y[te] - y[cand]
        d = dxs * dxs + dys * dys  # float32 throughout
        keep = ~(d > rad_sqr)
        cand, d = cand[keep][:max_candidates], d[keep][:max_candidates]
        order = np.argsort(d, kind="stable")
        cand, d = cand[order], d[order]
        if len(d) >= max_candidates:
            truncated += 1
        if len(d) > 1 and np.any(d[1:] == d[:-1]):
            ties += 1
        maxdeg = max(maxdeg, len(d))
        ids_out.append(cand.astype(np.int32))
        d2_out.append(d.astype(np.float64))
        offs.append(offs[-1] + len(d))
    return Csr(np.array(offs, np.int32), np.concatenate(ids_out) if ids_out else np.zeros(0, np.int32),
               np.concatenate(d2_out) if d2_out else np.zeros(0), int(maxdeg), int(truncated), int(ties))


def pair_bundle(te, le, use_ref=False, **params):
    """One pair's bundle grid: (valid, bmin[cells], bmax[cells]). te/le = (x, y, theta)."""
    p = dict(DEFAULTS, **params)
    bmin = np.zeros(1024)
    bmax = np.zeros(1024)
    nc = C.c_int(0)
    f = ref_lib().cvlref_pair_bundle if use_ref else lib().orc_pair_bundle
    dp = C.POINTER(C.c_double)
    v = f(te[0], te[1], te[2], le[0], le[1], le[2], p["nrad"], p["dx"], p["dt_deg"], p["max_k"],
          p["sx"], p["st"], bmin.ctypes.data_as(dp), bmax.ctypes.data_as(dp), C.byref(nc))
    return bool(v), bmin[:nc.value].copy(), bmax[:nc.value].copy()


def read_edge_file(path: str, values_per_edge: int = 4) -> np.ndarray:
    """Parses the reference's edge-file format (data_io.hpp:22-79) into [N, values_per_edge]."""
    rows = []
    with open(path) as fh:
        for ln, line in enumerate(fh, 1):
            toks = line.split()
            if len(toks) != values_per_edge:
                raise ValueError(f"{path}:{ln}: expected {values_per_edge} values, found {len(toks)}")
            rows.append([float(t) for t in toks])
    if not rows:
        raise ValueError(f"{path}: no edges")
    return np.asarray(rows, dtype=np.float64)


def parse_edges_f32(path: str, values_per_edge: int = 4) -> np.ndarray:
    """An edge file read into float32 the way `std::istream >> float` reads it
    (read_TO_edges_from_file<float>, data_io.hpp:22-79): each token converted
    straight to float by the C library's strtof (correctly rounded), not through
    double. Plain files only (the rows of read_edge_file)."""
    libc = C.CDLL(None)
    libc.strtof.restype = C.c_float
    libc.strtof.argtypes = [C.c_char_p, C.c_void_p]
    rows = []
    with open(path) as fh:
        for line in fh:
            toks = line.split()
            if len(toks) != values_per_edge:
                raise ValueError(f"{path}: expected {values_per_edge} values, found {len(toks)}")
            rows.append([libc.strtof(t.encode(), None) for t in toks])
    return np.asarray(rows, dtype=np.float32)


# ---- downstream: curvelets -> edgel link graph -> contour fragments ----------------
class _OrcContours(C.Structure):
    _fields_ = [("num_links", C.c_int), ("link_pe", C.POINTER(C.c_int)), ("link_ce", C.POINTER(C.c_int)),
                ("link_votes", C.POINTER(C.c_int)), ("num_frags", C.c_int),
                ("frag_offsets", C.POINTER(C.c_int64)), ("frag_ids", C.POINTER(C.c_int))]


class _OrigContours(C.Structure):
    _fields_ = [("num_links", C.c_int32), ("link_pe", C.POINTER(C.c_int32)), ("link_ce", C.POINTER(C.c_int32)),
                ("link_votes", C.POINTER(C.c_int32)), ("num_frags", C.c_int32),
                ("frag_offsets", C.POINTER(C.c_int64)), ("frag_ids", C.POINTER(C.c_int32)),
                ("seconds", C.c_double)]


@dataclass
class Contours:
    """links: [L, 3] (parent id, child id, votes), 0-based, in _cLinks order (parent
    ascending, creation order); fragments: CSR (offsets [F+1], ids 0-based)."""
    links: np.ndarray
    frag_offsets: np.ndarray
    frag_ids: np.ndarray
    seconds: float = 0.0

    @property
    def num_frags(self) -> int:
        return int(self.frag_offsets.shape[0] - 1)

    def fragments(self):
        return [self.frag_ids[self.frag_offsets[i]:self.frag_offsets[i + 1]] for i in range(self.num_frags)]


def _contours_from(o, seconds=0.0) -> Contours:
    L = o.num_links
    links = np.column_stack([_arr(o.link_pe, L, np.int32), _arr(o.link_ce, L, np.int32),
                             _arr(o.link_votes, L, np.int32)]) if L else np.zeros((0, 3), np.int32)
    offs = _arr(o.frag_offsets, o.num_frags + 1, np.int64)
    ids = _arr(o.frag_ids, int(offs[-1]), np.int32) if offs[-1] else np.zeros(0, np.int32)
    return Contours(links.astype(np.int32), offs, ids, seconds)


def _contour_args(edges, chains, forward=None):
    e, ep, n, sz = _edges_arg(edges)
    ch = np.ascontiguousarray(chains, dtype=np.uint32)
    assert ch.ndim == 2
    return e, ep, n, sz, ch


def link_contours(edges, chains, min_group_size=4, gap=1.5) -> Contours:
    """The C restatement (oracle/cvl_oracle.c: orc_link_contours)."""
    L = lib()
    if not hasattr(L, "_contours_set"):
        L.orc_link_contours.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(C.c_uint), C.c_int,
                                        C.c_int, C.c_uint, C.c_double, C.POINTER(_OrcContours)]
        L.orc_contours_free.argtypes = [C.POINTER(_OrcContours)]
        L._contours_set = True
    e, ep, n, sz, ch = _contour_args(edges, chains)
    o = _OrcContours()
    rc = L.orc_link_contours(ep, n, sz, ch.ctypes.data_as(C.POINTER(C.c_uint)), ch.shape[0], ch.shape[1],
                             min_group_size, gap, C.byref(o))
    if rc != 0:
        raise ValueError(f"orc_link_contours: {rc}")
    try:
        return _contours_from(o)
    finally:
        L.orc_contours_free(C.byref(o))


_orig = None


def orig_available() -> bool:
    return os.path.exists(ORIG_SO)


def ref_link_contours(edges, chains, forward=None, min_group_size=4, gap=1.5) -> Contours:
    """The reference's own original_code link graph + one-chain extraction
    (oracle/orig_harness.cpp, built into oracle/_ref/liborigref.so)."""
    global _orig
    if _orig is None:
        if not os.path.exists(ORIG_SO):
            raise FileNotFoundError("original_code harness not built: " + ORIG_SO)
        L = C.CDLL(ORIG_SO)
        L.origref_link_contours.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(C.c_uint32),
                                            C.c_int, C.c_int, C.POINTER(C.c_uint8), C.c_uint, C.c_double,
                                            C.POINTER(_OrigContours)]
        L.origref_contours_free.argtypes = [C.POINTER(_OrigContours)]
        _orig = L
    e, ep, n, sz, ch = _contour_args(edges, chains)
    fw = None
    if forward is not None:
        fw = np.ascontiguousarray(forward, dtype=np.uint8)
    o = _OrigContours()
    rc = _orig.origref_link_contours(ep, n, sz, ch.ctypes.data_as(C.POINTER(C.c_uint32)), ch.shape[0],
                                     ch.shape[1], fw.ctypes.data_as(C.POINTER(C.c_uint8)) if fw is not None
                                     else None, min_group_size, gap, C.byref(o))
    if rc != 0:
        raise ValueError(f"origref_link_contours: {rc}")
    try:
        return _contours_from(o, o.seconds)
    finally:
        _orig.origref_contours_free(C.byref(o))


class _OrigPolyarcs(C.Structure):
    _fields_ = [("num_polyarcs", C.c_int32), ("offsets", C.POINTER(C.c_int64)), ("ids", C.POINTER(C.c_int32)),
                ("info", C.POINTER(C.c_double)), ("seconds", C.c_double)]


@dataclass
class Polyarcs:
    """Polyarcs in polyarcmap order: CSR chains (offsets [P+1], 0-based ids) and
    info [P, 12] (curvelet::set_output's columns; unset columns 0)."""
    offsets: np.ndarray
    ids: np.ndarray
    info: np.ndarray
    seconds: float = 0.0

    @property
    def num(self) -> int:
        return int(self.offsets.shape[0] - 1)


def ref_polyarcs(edges, chains, min_group_size=4, gap=1.5, dx=0.4, dt=(15.0 / 180.0) * np.pi, max_k=0.3,
                 rad=3.5, token_len=1.0) -> Polyarcs:
    """The reference's original_code fit_polyarcs_to_all_edgel_chains after the link
    graph and the one-chains (oracle/orig_harness.cpp: origref_polyarcs)."""
    ref_link_contours  # noqa: B018 (loads the library through the same path)
    global _orig
    if _orig is None:
        L = C.CDLL(ORIG_SO)
        L.origref_link_contours.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(C.c_uint32),
                                            C.c_int, C.c_int, C.POINTER(C.c_uint8), C.c_uint, C.c_double,
                                            C.POINTER(_OrigContours)]
        L.origref_contours_free.argtypes = [C.POINTER(_OrigContours)]
        _orig = L
    if not hasattr(_orig, "_poly_set"):
        _orig.origref_polyarcs.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(C.c_uint32), C.c_int,
                                           C.c_int, C.c_uint, C.c_double, C.c_double, C.c_double, C.c_double,
                                           C.c_double, C.c_double, C.POINTER(_OrigPolyarcs)]
        _orig.origref_polyarcs_free.argtypes = [C.POINTER(_OrigPolyarcs)]
        _orig._poly_set = True
    e, ep, n, sz, ch = _contour_args(edges, chains)
    o = _OrigPolyarcs()
    rc = _orig.origref_polyarcs(ep, n, sz, ch.ctypes.data_as(C.POINTER(C.c_uint32)), ch.shape[0], ch.shape[1],
                                min_group_size, gap, dx, dt, max_k, rad, token_len, C.byref(o))
    if rc != 0:
        raise ValueError(f"origref_polyarcs: {rc}")
    try:
        P = o.num_polyarcs
        offs = _arr(o.offsets, P + 1, np.int64)
        ids = _arr(o.ids, int(offs[-1]), np.int32) if offs[-1] else np.zeros(0, np.int32)
        info = _arr(o.info, 12 * P, np.float64).reshape(P, 12)
        return Polyarcs(offs, ids, info, o.seconds)
    finally:
        _orig.origref_polyarcs_free(C.byref(o))


class _OrcPolyarcs(C.Structure):
    _fields_ = [("num", C.c_int), ("offsets", C.POINTER(C.c_int64)), ("ids", C.POINTER(C.c_int)),
                ("info", C.POINTER(C.c_double))]


def polyarcs(edges, frag_offsets, frag_ids, dx=0.4, dt=(15.0 / 180.0) * np.pi, max_k=0.3, rad=3.5,
             token_len=1.0) -> Polyarcs:
    """The C restatement of the polyarc fit (oracle/cvl_oracle.c: orc_polyarcs_fit)
    on given contour fragments (CSR, 0-based ids)."""
    L = lib()
    if not hasattr(L, "_poly_set"):
        L.orc_polyarcs_fit.argtypes = [C.POINTER(C.c_double), C.c_int, C.c_int, C.POINTER(C.c_int64),
                                       C.POINTER(C.c_int), C.c_int, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, C.POINTER(_OrcPolyarcs)]
        L.orc_polyarcs_free.argtypes = [C.POINTER(_OrcPolyarcs)]
        L._poly_set = True
    e, ep, n, sz = _edges_arg(edges)
    fo = np.ascontiguousarray(frag_offsets, dtype=np.int64)
    fi = np.ascontiguousarray(frag_ids, dtype=np.int32)
    if fi.size == 0:
        fi = np.zeros(1, np.int32)
    o = _OrcPolyarcs()
    rc = L.orc_polyarcs_fit(ep, n, sz, fo.ctypes.data_as(C.POINTER(C.c_int64)), fi.ctypes.data_as(C.POINTER(C.c_int)),
                            fo.shape[0] - 1, dx, dt, max_k, rad, token_len, C.byref(o))
    if rc != 0:
        raise ValueError(f"orc_polyarcs_fit: {rc}")
    try:
        P = o.num
        offs = _arr(o.offsets, P + 1, np.int64)
        ids = _arr(o.ids, int(offs[-1]), np.int32) if offs[-1] else np.zeros(0, np.int32)
        info = _arr(o.info, 12 * P, np.float64).reshape(P, 12)
        return Polyarcs(offs, ids, info)
    finally:
        L.orc_polyarcs_free(C.byref(o))
