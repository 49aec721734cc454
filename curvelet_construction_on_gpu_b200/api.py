"""Host-side API over libcvl.so.

Two layers, mirroring the reference:

* the engine layer (``Engine``): one-shot ``run`` (run_curvelet<double> without
  file I/O, cpu_curvelet/main.cpp:20-96), device-resident ragged batches,
  per-kernel timings;
* the reference's template API, same names and argument meaning:
  ``build_neighbor_csr_graph`` (cpu_curvelet/preprocess.hpp:186-274) filling a
  ``GPUNeighborGraph`` (the CPUNeighborGraph fields, preprocess.hpp:18-31), and
  ``CurveletGPU`` (CurveletCPU, cpu_curvelet/cpu_curvelet.hpp:22-123) with
  ``form_pairwise_bundles`` / ``build_curvelets_greedy`` / ``num_curvelets`` /
  ``chain_width`` / ``_edge_chain_final`` / ``_curvelet_info``.

Everything computes on the GPU through the C ABI; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from ._abi import CvlEngineCfg, CvlGraphView, CvlParams, CvlResultView, check

M_PI = 3.14159265358979323846  # curvelet_utils.hpp:10


@dataclass
class CurveletParams:
    """CurveletParams (cpu_curvelet/param_settings.hpp:9-24): same fields and defaults."""
    nrad: float = 3.5
    gap: float = 1.5
    dx: float = 0.4
    dt_deg: float = 15.0
    max_k: float = 0.3
    curvelet_style: int = 2
    group_max_sz: int = 4
    out_type: int = 0
    sx: float = 0.1
    st: float = 0.08
    edge_file: str = "eth3d_cables2.txt"
    edge_data_sz: int = 4
    max_candidates: int = 128

    def to_c(self, dt_rad: float = 0.0) -> CvlParams:
        p = CvlParams()
        _abi.load().cvl_params_default(C.byref(p))
        p.nrad, p.gap, p.dx, p.dt_deg, p.dt_rad, p.max_k = (self.nrad, self.gap, self.dx, self.dt_deg, dt_rad,
                                                            self.max_k)
        p.curvelet_style, p.group_max_sz, p.out_type = self.curvelet_style, self.group_max_sz, self.out_type
        p.sx, p.st, p.edge_data_sz, p.max_candidates = self.sx, self.st, self.edge_data_sz, self.max_candidates
        return p


@dataclass
class Result:
    """Curvelets of one map: chains [C, group_max_sz + 1] uint32 (1-based ids,
    zero padded) and info [C, 10] float64 (the info file's rows)."""
    chains: np.ndarray
    info: np.ndarray
    valid_pairs: int
    total_neighbor_pairs: int
    max_num_of_neighbors: int
    truncated_anchors: int
    num_edges: int
    device_ms: float = 0.0

    @property
    def num_curvelets(self) -> int:
        return int(self.chains.shape[0])


class _Owner:
    """Frees a C result handle when the last numpy view onto it goes away."""

    def __init__(self, lib, handle, free_name: str):
        self._lib, self._h, self._free = lib, handle, free_name

    def __del__(self):
        try:
            if self._h:
                getattr(self._lib, self._free)(self._h)
                self._h = None
        except Exception:
            pass


def _view_to_result(v: CvlResultView, owner: "_Owner | None" = None) -> Result:
    """numpy views onto the result's page-locked buffers (no copy when an owner
    keeps the C result alive; a copy otherwise)."""
    nc, w = int(v.num_curvelets), int(v.chain_width)
    if nc:
        chains = np.ctypeslib.as_array(v.chains, shape=(nc * w,)).reshape(nc, w)
        info = np.ctypeslib.as_array(v.info, shape=(nc * 10,)).reshape(nc, 10)
        if owner is None:
            chains, info = chains.copy(), info.copy()
        else:
            chains = _OwnedArray.wrap(chains, owner)
            info = _OwnedArray.wrap(info, owner)
    else:
        chains = np.zeros((0, w), np.uint32)
        info = np.zeros((0, 10), np.float64)
    return Result(chains, info, int(v.valid_pairs), int(v.total_neighbor_pairs), int(v.max_num_of_neighbors),
                  int(v.truncated_anchors), int(v.num_edges), float(v.device_ms))


@dataclass
class ContourParams:
    """construct_the_link_graph's min_group_size (4 in form_curvelet_process::execute,
    original_code/form_curvelet_process.cpp:79) and the gap between consecutive
    edges of a fragment (1.5 in original_code/main.cpp:146)."""
    min_group_size: int = 4
    gap: float = 1.5
    # C^1 polyarcs along the fragments (fit_polyarcs_to_all_edgel_chains,
    # original_code/form_curvelet_process.cpp:661-796), with form_curvelet_mex's
    # dx, dt, max_k, rad and token_len (original_code/main.cpp:145-151)
    fit_polyarcs: bool = False
    dx: float = 0.4
    dt_rad: float = (15.0 / 180.0) * M_PI
    max_k: float = 0.3
    rad: float = 3.5
    token_len: float = 1.0

    def to_c(self) -> _abi.CvlContourParams:
        return _abi.CvlContourParams(int(self.min_group_size), float(self.gap), 1 if self.fit_polyarcs else 0,
                                     float(self.dx), float(self.dt_rad), float(self.max_k), float(self.rad),
                                     float(self.token_len))


@dataclass
class Contours:
    """The edgel link graph and its contour fragments (one-chains) of one map.
    links: [L, 3] int32 (parent id, child id, votes), 0-based, in _cLinks order
    (parent ascending, then creation order); fragments in start-edge order as
    CSR: frag_offsets [F + 1] int64, frag_ids int32 (0-based)."""
    links: np.ndarray
    frag_offsets: np.ndarray
    frag_ids: np.ndarray
    num_edges: int
    device_ms: float = 0.0
    # polyarcs (ContourParams.fit_polyarcs): CSR chains and info [P, 12]
    # (curvelet::set_output's columns; the centre columns 10-11 are 0 for a line)
    poly_offsets: np.ndarray | None = None
    poly_ids: np.ndarray | None = None
    poly_info: np.ndarray | None = None

    @property
    def num_polyarcs(self) -> int:
        return 0 if self.poly_offsets is None else int(self.poly_offsets.shape[0] - 1)

    def polyarcs(self) -> list:
        return [self.poly_ids[self.poly_offsets[i]:self.poly_offsets[i + 1]] for i in range(self.num_polyarcs)]

    @property
    def num_frags(self) -> int:
        return int(self.frag_offsets.shape[0] - 1)

    def fragments(self) -> list:
        return [self.frag_ids[self.frag_offsets[i]:self.frag_offsets[i + 1]] for i in range(self.num_frags)]

    def as_array(self) -> np.ndarray:
        """curve_fragment_graph::get_output_array: one row per fragment, 1-based
        edge ids, width = the longest fragment, zero-padded (the reference leaves
        the padding unset)."""
        lens = np.diff(self.frag_offsets)
        w = int(lens.max()) if lens.size else 0
        out = np.zeros((self.num_frags, w), np.int32)
        for i in range(self.num_frags):
            out[i, :lens[i]] = self.frag_ids[self.frag_offsets[i]:self.frag_offsets[i + 1]] + 1
        return out


def _contours_from_handle(lib, h) -> Contours:
    try:
        v = _abi.CvlContoursView()
        check(lib.cvl_contours_get(h, C.byref(v)), "cvl_contours_get")
        L, F = int(v.num_links), int(v.num_fragments)
        if L:
            links = np.column_stack([np.ctypeslib.as_array(v.link_parent, shape=(L,)),
                                     np.ctypeslib.as_array(v.link_child, shape=(L,)),
                                     np.ctypeslib.as_array(v.link_votes, shape=(L,))]).astype(np.int32)
        else:
            links = np.zeros((0, 3), np.int32)
        offs = np.ctypeslib.as_array(v.fragment_offsets, shape=(F + 1,)).copy()
        nid = int(offs[-1])
        ids = np.ctypeslib.as_array(v.fragment_ids, shape=(nid,)).copy() if nid else np.zeros(0, np.int32)
        out = Contours(links, offs, ids, int(v.num_edges), float(v.device_ms))
        if v.polyarc_offsets:
            P = int(v.num_polyarcs)
            out.poly_offsets = np.ctypeslib.as_array(v.polyarc_offsets, shape=(P + 1,)).copy()
            npid = int(out.poly_offsets[-1])
            out.poly_ids = (np.ctypeslib.as_array(v.polyarc_ids, shape=(npid,)).copy() if npid
                            else np.zeros(0, np.int32))
            out.poly_info = (np.ctypeslib.as_array(v.polyarc_info, shape=(P * 12,)).reshape(P, 12).copy() if P
                             else np.zeros((0, 12)))
        return out
    finally:
        lib.cvl_contours_free(h)


def _result_from_handle(lib, r) -> Result:
    owner = _Owner(lib, r, "cvl_result_free")
    v = CvlResultView()
    check(lib.cvl_result_get(r, C.byref(v)), "cvl_result_get")
    return _view_to_result(v, owner)


class _OwnedArray(np.ndarray):
    """An ndarray view that keeps the buffer's owner alive."""

    @classmethod
    def wrap(cls, arr: np.ndarray, owner: _Owner) -> "_OwnedArray":
        out = arr.view(cls)
        out._owner = owner
        return out

    def __array_finalize__(self, obj):
        self._owner = getattr(obj, "_owner", None)


def _edges(edges) -> np.ndarray:
    e = np.ascontiguousarray(edges, dtype=np.float64)
    if e.ndim != 2:
        raise ValueError("edges must be a 2-D array [num_edges, edge_data_sz]")
    return e


class Engine:
    """One CUDA device, one stream, a grow-only device workspace."""

    def __init__(self, device: int = 0, mem_budget_bytes: int = 0, cell_size: int = 0, seeds_per_group: int = 0,
                 bundle_slots: int = 0):
        lib = _abi.load()
        cfg = CvlEngineCfg()
        lib.cvl_engine_cfg_default(C.byref(cfg))
        cfg.device, cfg.mem_budget_bytes, cfg.cell_size = device, mem_budget_bytes, cell_size
        cfg.seeds_per_group, cfg.bundle_slots = seeds_per_group, bundle_slots
        h = C.c_void_p()
        check(lib.cvl_engine_create(C.byref(cfg), C.byref(h)), "cvl_engine_create")
        self._h = h
        self._lib = lib

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.cvl_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- the plain form
    def run(self, edges, params: CurveletParams | None = None, dt_rad: float = 0.0, scalar: str = "double") -> Result:
        """run_curvelet<double>, or run_curvelet<float> (the reference's --float
        mode) for scalar="float": then the edges are taken as float32, as the
        reference reads them in that mode (data_io.read_edges(..., scalar="float"))."""
        params = params or CurveletParams()
        p = params.to_c(dt_rad)
        r = C.c_void_p()
        if scalar == "float":
            if np.asarray(edges).dtype != np.float32:
                raise TypeError("scalar='float' takes float32 edges (as read_edges(..., scalar='float') gives); "
                                "a float64 array would be rounded here, not read as the reference reads it")
            e = np.ascontiguousarray(edges)
            if e.ndim != 2:
                raise ValueError("edges must be a 2-D array [num_edges, edge_data_sz]")
            check(self._lib.cvl_run_f32(self._h, e.ctypes.data_as(C.POINTER(C.c_float)), e.shape[0], e.shape[1],
                                        C.byref(p), C.byref(r)), "cvl_run_f32")
        elif scalar == "double":
            e = _edges(edges)
            check(self._lib.cvl_run(self._h, e.ctypes.data_as(_abi._dp), e.shape[0], e.shape[1], C.byref(p),
                                    C.byref(r)), "cvl_run")
        else:
            raise ValueError("scalar must be 'double' or 'float'")
        owner = _Owner(self._lib, r, "cvl_result_free")
        v = CvlResultView()
        check(self._lib.cvl_result_get(r, C.byref(v)), "cvl_result_get")
        return _view_to_result(v, owner)

    def run_device(self, d_edges: int, num_edges: int, edge_data_sz: int = 4, params: CurveletParams | None = None,
                   dt_rad: float = 0.0, ready_event: int | None = None, to_host: bool = True) -> Result | None:
        """cvl_run_device: edges already in this engine's device memory (d_edges: a
        device pointer, e.g. a torch CUDA tensor's data_ptr()), read in place after
        ready_event (a cudaEvent_t handle, e.g. torch.cuda.Event().cuda_event) if
        given. to_host=False leaves the results on the device (device_results())."""
        params = params or CurveletParams()
        p = params.to_c(dt_rad)
        r = C.c_void_p()
        check(self._lib.cvl_run_device(self._h, C.c_void_p(d_edges), num_edges, edge_data_sz, C.byref(p),
                                       C.c_void_p(ready_event) if ready_event else None,
                                       C.byref(r) if to_host else None), "cvl_run_device")
        return _result_from_handle(self._lib, r) if to_host else None

    def device_results(self) -> dict:
        """The device-resident outputs of the last run_device(to_host=False):
        chains/info device pointers (cvl_result_view layout) and the event to wait on."""
        v = _abi.CvlDeviceResults()
        check(self._lib.cvl_engine_device_results(self._h, C.byref(v)), "cvl_engine_device_results")
        return {"num_curvelets": int(v.num_curvelets), "chain_width": int(v.chain_width),
                "chains": int(v.chains or 0), "info": int(v.info or 0), "done_event": int(v.done_event or 0)}

    def run_maps(self, maps, params: CurveletParams | None = None, dt_rad: float = 0.0,
                 group_edges: int = 0, counts=None) -> list:
        """Many maps, host to host (cvl_run_maps): one Result per map, as run()
        would give it; the result copies of one group of maps overlap the compute
        of the next. maps: a list of [n_i, sz] arrays, or one array of all rows
        back to back with counts."""
        params = params or CurveletParams()
        if counts is None:
            cnt = np.array([np.asarray(m).shape[0] for m in maps], np.int32)
            e = maps[0] if len(maps) == 1 else np.concatenate([np.asarray(m, np.float64) for m in maps])
        else:
            cnt = np.ascontiguousarray(counts, dtype=np.int32)
            e = maps
        e = _edges(e)
        p = params.to_c(dt_rad)
        hs = (C.c_void_p * len(cnt))()
        check(self._lib.cvl_run_maps(self._h, e.ctypes.data_as(_abi._dp), cnt.ctypes.data_as(C.POINTER(C.c_int32)),
                                     len(cnt), e.shape[1], C.byref(p), int(group_edges), hs), "cvl_run_maps")
        return [_result_from_handle(self._lib, C.c_void_p(h)) for h in hs]

    # ---- downstream: link graph and contour fragments
    def link_contours(self, edges, chains, contour_params: ContourParams | None = None) -> Contours:
        """construct_the_link_graph + extract_regular_contours_from_the_link_graph
        (original_code/form_curvelet_process.cpp:453-654) on curvelets the caller
        holds (chains as Result.chains gives them)."""
        cp = (contour_params or ContourParams()).to_c()
        e = _edges(edges)
        ch = np.ascontiguousarray(chains, dtype=np.uint32)
        if ch.ndim != 2:
            raise ValueError("chains must be a 2-D array [num_curvelets, chain_width]")
        h = C.c_void_p()
        check(self._lib.cvl_link_contours(self._h, e.ctypes.data_as(_abi._dp), e.shape[0], e.shape[1],
                                          ch.ctypes.data_as(C.POINTER(C.c_uint32)), ch.shape[0], ch.shape[1],
                                          C.byref(cp), C.byref(h)), "cvl_link_contours")
        return _contours_from_handle(self._lib, h)

    def run_contours(self, edges, params: CurveletParams | None = None,
                     contour_params: ContourParams | None = None, dt_rad: float = 0.0,
                     want_curvelets: bool = True):
        """Edges -> curvelets -> link graph -> fragments in one device pass.
        Returns (Result or None, Contours)."""
        params = params or CurveletParams()
        cp = (contour_params or ContourParams(gap=params.gap, dx=params.dx, max_k=params.max_k, rad=params.nrad,
                                              dt_rad=dt_rad if dt_rad > 0 else (params.dt_deg / 180.0) * M_PI)).to_c()
        e = _edges(edges)
        p = params.to_c(dt_rad)
        r = C.c_void_p()
        h = C.c_void_p()
        check(self._lib.cvl_run_contours(self._h, e.ctypes.data_as(_abi._dp), e.shape[0], e.shape[1], C.byref(p),
                                         C.byref(cp), C.byref(r) if want_curvelets else None, C.byref(h)),
              "cvl_run_contours")
        res = _result_from_handle(self._lib, r) if want_curvelets else None
        return res, _contours_from_handle(self._lib, h)

    # ---- staged API
    def build_neighbor_graph(self, edges, rad: float = 3.5, neighbor_radius: int = 3,
                             max_candidates: int = 128) -> "GPUNeighborGraph":
        e = _edges(edges)
        g = C.c_void_p()
        check(self._lib.cvl_build_neighbor_graph(self._h, e.ctypes.data_as(_abi._dp), e.shape[0], e.shape[1], rad,
                                                 neighbor_radius, max_candidates, C.byref(g)),
              "cvl_build_neighbor_graph")
        return GPUNeighborGraph._from_handle(self, g, e)

    def form_pairwise_bundles(self, graph: "GPUNeighborGraph", params: CurveletParams, dt_rad: float = 0.0) -> int:
        p = params.to_c(dt_rad)
        vp = C.c_uint32(0)
        check(self._lib.cvl_form_pairwise_bundles(self._h, graph._h, C.byref(p), C.byref(vp)),
              "cvl_form_pairwise_bundles")
        return int(vp.value)

    def build_curvelets(self, graph: "GPUNeighborGraph", params: CurveletParams, dt_rad: float = 0.0) -> Result:
        p = params.to_c(dt_rad)
        r = C.c_void_p()
        check(self._lib.cvl_build_curvelets(self._h, graph._h, C.byref(p), C.byref(r)), "cvl_build_curvelets")
        try:
            v = CvlResultView()
            check(self._lib.cvl_result_get(r, C.byref(v)), "cvl_result_get")
            return _view_to_result(v)
        finally:
            self._lib.cvl_result_free(r)

    def pair_bundles(self, pairs, params: CurveletParams | None = None, dt_rad: float = 0.0,
                     literal: bool = False):
        """Bundles of independent (anchor, neighbour) pairs, rows (te_x, te_y, te_theta, le_x, le_y, le_theta).
        Returns (bmin [n, cells], bmax [n, cells], valid [n] bool). literal=True runs the
        checking entry point cvl_check_pair_bundles_literal (the reference's two branches
        as written, on the same device trig values)."""
        params = params or CurveletParams()
        fn = self._lib.cvl_check_pair_bundles_literal if literal else self._lib.cvl_pair_bundles
        name = "cvl_check_pair_bundles_literal" if literal else "cvl_pair_bundles"
        q = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1, 6)
        n = q.shape[0]
        p = params.to_c(dt_rad)
        cells = C.c_int32(0)
        cap = 128
        bmin = np.zeros((max(n, 1), cap))
        bmax = np.zeros((max(n, 1), cap))
        valid = np.zeros(max(n, 1), np.uint8)
        # first call sizes the grid
        check(fn(self._h, q.ctypes.data_as(_abi._dp), 0, C.byref(p), bmin.ctypes.data_as(_abi._dp),
                 bmax.ctypes.data_as(_abi._dp), valid.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(cells)), name)
        nc = cells.value
        bmin = np.zeros((max(n, 1), nc))
        bmax = np.zeros((max(n, 1), nc))
        check(fn(self._h, q.ctypes.data_as(_abi._dp), n, C.byref(p), bmin.ctypes.data_as(_abi._dp),
                 bmax.ctypes.data_as(_abi._dp), valid.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(cells)), name)
        return bmin[:n], bmax[:n], valid[:n].astype(bool)

    def workspace_bytes(self, num_edges: int, num_pairs: int, num_curvelets: int, num_maps: int = 1,
                        params: CurveletParams | None = None, edge_data_sz: int = 4) -> tuple[int, int]:
        """cvl_engine_workspace_bytes: (total, per-launch bundle chunk) device bytes of a launch of that shape."""
        shp = _abi.CvlWorkspaceShape(num_edges, num_pairs, num_curvelets, num_maps, edge_data_sz)
        p = (params or CurveletParams()).to_c()
        tot, chunk = C.c_size_t(0), C.c_size_t(0)
        check(self._lib.cvl_engine_workspace_bytes(self._h, C.byref(shp), C.byref(p), C.byref(tot), C.byref(chunk)),
              "cvl_engine_workspace_bytes")
        return int(tot.value), int(chunk.value)

    def reserve_workspace(self, num_edges: int, num_pairs: int, num_curvelets: int, num_maps: int = 1,
                          params: CurveletParams | None = None, edge_data_sz: int = 4) -> None:
        """cvl_engine_reserve_workspace: allocate the workspace of that launch shape now."""
        shp = _abi.CvlWorkspaceShape(num_edges, num_pairs, num_curvelets, num_maps, edge_data_sz)
        p = (params or CurveletParams()).to_c()
        check(self._lib.cvl_engine_reserve_workspace(self._h, C.byref(shp), C.byref(p)),
              "cvl_engine_reserve_workspace")

    def warmup(self) -> None:
        """cvl_engine_warmup: run two built-in maps through the engine's forms of the path,
        so that the first real run pays no module loading or pool growth."""
        check(self._lib.cvl_engine_warmup(self._h), "cvl_engine_warmup")

    def set_graphs(self, enable: bool) -> None:
        """cvl_engine_set_graphs: replay a CUDA graph per size bucket (default) or launch kernel by kernel."""
        check(self._lib.cvl_engine_set_graphs(self._h, 1 if enable else 0), "cvl_engine_set_graphs")

    def graph_stats(self) -> dict:
        """cvl_engine_graph_stats: enabled, graphs, captures, replays, fallbacks."""
        g = _abi.CvlEngineGraphs()
        check(self._lib.cvl_engine_graph_stats(self._h, C.byref(g)), "cvl_engine_graph_stats")
        return {name: getattr(g, name) for name, _ in g._fields_}

    def memory(self) -> dict:
        """cvl_engine_memory_get: held_bytes, device_grows, device_grow_ms."""
        m = _abi.CvlEngineMemory()
        check(self._lib.cvl_engine_memory_get(self._h, C.byref(m)), "cvl_engine_memory_get")
        return {name: getattr(m, name) for name, _ in m._fields_}

    def transport_cells(self, ops, params: CurveletParams | None = None, dt_rad: float = 0.0,
                        shared_quotients: bool = False):
        """cvl_check_transport_cells: one orientation column of the transport per row of
        ops [n, 10] = (DX, DY, tt, s_m, s_p, cos_m, sin_m, cos_p, sin_p, branch1).
        shared_quotients: the rewrite's two k_dx quotients from one reciprocal
        (Markstein's corrections, operands checked per cell) instead of two divisions.
        Returns (rewrite_min, rewrite_max, literal_min, literal_max), each [n, P]."""
        params = params or CurveletParams()
        q = np.ascontiguousarray(ops, dtype=np.float64).reshape(-1, 10)
        n = q.shape[0]
        p = params.to_c(dt_rad)
        rows = C.c_int32(0)
        one = np.zeros(1)
        quot = 1 if shared_quotients else 0
        check(self._lib.cvl_check_transport_cells(self._h, q.ctypes.data_as(_abi._dp), 0, C.byref(p), quot,
                                                  one.ctypes.data_as(_abi._dp), C.byref(rows)),
              "cvl_check_transport_cells")
        P = rows.value
        out = np.zeros((max(n, 1), 4, P))
        check(self._lib.cvl_check_transport_cells(self._h, q.ctypes.data_as(_abi._dp), n, C.byref(p), quot,
                                                  out.ctypes.data_as(_abi._dp), C.byref(rows)),
              "cvl_check_transport_cells")
        out = out[:n]
        return out[:, 0], out[:, 1], out[:, 2], out[:, 3]

    # ---- batches
    def upload_batch(self, maps: list) -> "Batch":
        arrs = [_edges(m) for m in maps]
        sz = arrs[0].shape[1]
        if any(a.shape[1] != sz for a in arrs):
            raise ValueError("all maps of a batch need the same edge_data_sz")
        cat = np.ascontiguousarray(np.concatenate(arrs, axis=0))
        counts = np.asarray([a.shape[0] for a in arrs], dtype=np.int32)
        b = C.c_void_p()
        check(self._lib.cvl_batch_upload(self._h, cat.ctypes.data_as(_abi._dp),
                                         counts.ctypes.data_as(C.POINTER(C.c_int32)), len(arrs), sz, C.byref(b)),
              "cvl_batch_upload")
        return Batch(self, b, counts)

    def upload_ragged(self, edges, counts) -> "Batch":
        """A batch from maps already concatenated: edges [sum(counts), sz] (page-locked
        memory, when it is, is copied to the device without staging)."""
        e = _edges(edges)
        c = np.ascontiguousarray(counts, dtype=np.int32)
        if int(c.sum()) != e.shape[0]:
            raise ValueError("counts must sum to the number of edge rows")
        b = C.c_void_p()
        check(self._lib.cvl_batch_upload(self._h, e.ctypes.data_as(_abi._dp), c.ctypes.data_as(C.POINTER(C.c_int32)),
                                         len(c), e.shape[1], C.byref(b)), "cvl_batch_upload")
        return Batch(self, b, c)

    def run_batch(self, batch: "Batch", params: CurveletParams | None = None) -> "BatchResult":
        params = params or CurveletParams()
        p = params.to_c()
        r = C.c_void_p()
        check(self._lib.cvl_batch_run(self._h, batch._h, C.byref(p), C.byref(r)), "cvl_batch_run")
        return BatchResult(self, r, len(batch.counts))

    # ---- tuning (every tuning gives the same results; only the time changes)
    def get_tuning(self, bucket: int) -> dict:
        t = _abi.CvlTuning()
        check(self._lib.cvl_engine_get_tuning(self._h, bucket, C.byref(t)), "cvl_engine_get_tuning")
        return {name: getattr(t, name) for name, _ in t._fields_}

    def set_tuning(self, bucket: int, **knobs) -> None:
        """Sets knobs of one bucket (-1: every bucket); unnamed knobs keep their values."""
        cur = self.get_tuning(max(bucket, 0))
        cur.update(knobs)
        t = _abi.CvlTuning(**cur)
        check(self._lib.cvl_engine_set_tuning(self._h, bucket, C.byref(t)), "cvl_engine_set_tuning")

    def autotune(self, batch: "Batch", params: CurveletParams | None = None, passes: int = 1) -> tuple[dict, float]:
        """Coordinate descent over the batch's bucket; installs and returns (tuning, device ms)."""
        p = (params or CurveletParams()).to_c()
        t = _abi.CvlTuning()
        ms = C.c_double(0.0)
        check(self._lib.cvl_engine_autotune(self._h, batch._h, C.byref(p), passes, C.byref(t), C.byref(ms)),
              "cvl_engine_autotune")
        return {name: getattr(t, name) for name, _ in t._fields_}, float(ms.value)

    # ---- measurement helpers
    def flush_l2(self) -> None:
        check(self._lib.cvl_engine_flush_l2(self._h), "cvl_engine_flush_l2")

    def kernel_times(self) -> list[tuple[str, float]]:
        n = self._lib.cvl_engine_last_kernel_times(self._h, None, None, 0)
        if n < 0:
            check(n, "cvl_engine_last_kernel_times")
        cap = max(n, 1)
        names = (C.c_char_p * cap)()
        ms = (C.c_double * cap)()
        n = self._lib.cvl_engine_last_kernel_times(self._h, names, ms, cap)
        if n < 0:
            check(n, "cvl_engine_last_kernel_times")
        return [(names[k].decode(), float(ms[k])) for k in range(min(n, cap))]

    def launch_count(self) -> int:
        n = self._lib.cvl_engine_last_launch_count(self._h)
        if n < 0:
            check(n, "cvl_engine_last_launch_count")
        return int(n)

    def fp64_peak_tflops(self) -> float:
        t = C.c_double(0)
        check(self._lib.cvl_measure_fp64_peak(self._h, C.byref(t)), "cvl_measure_fp64_peak")
        return float(t.value)


class Batch:
    def __init__(self, eng: Engine, h, counts):
        self._eng, self._h, self.counts = eng, h, counts

    def close(self):
        # a batch's device memory goes with its engine; after Engine.close there is nothing to free
        if self._h and getattr(self._eng, "_h", None):
            self._eng._lib.cvl_batch_free(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BatchResult:
    def __init__(self, eng: Engine, h, num_maps: int):
        self._eng, self._h, self.num_maps = eng, h, num_maps

    def stats(self) -> dict:
        st = _abi.CvlBatchStats()
        check(self._eng._lib.cvl_batch_result_stats(self._h, C.byref(st)), "cvl_batch_result_stats")
        return {name: getattr(st, name) for name, _ in st._fields_}

    def map(self, m: int) -> Result:
        """Map m, copied out of the batch's downloaded outputs."""
        v = CvlResultView()
        check(self._eng._lib.cvl_batch_result_map(self._h, m, C.byref(v)), "cvl_batch_result_map")
        return _view_to_result(v)

    def take_map(self, m: int) -> Result:
        """Map m as an independent result: only its rows are copied to page-locked
        memory, and the arrays are views onto it."""
        lib = self._eng._lib
        r = C.c_void_p()
        check(lib.cvl_batch_result_take_map(self._h, m, C.byref(r)), "cvl_batch_result_take_map")
        return _result_from_handle(lib, r)

    def close(self):
        if self._h:
            self._eng._lib.cvl_batch_result_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# Serving: continuous batching with memory-budget admission (cvl_server_*)
# ---------------------------------------------------------------------------
class Server:
    """Requests in, results out; workers fold waiting maps into shared launches.
    submit() copies the map and returns at once; wait()/poll() hand the result
    out once."""

    def __init__(self, params: CurveletParams | None = None, device: int = 0, workers: int = 4,
                 mem_budget_bytes: int = 40 << 30, admit_bytes_per_edge: int = 0,
                 max_batch_edges: int = 2 << 20, large_map_edges: int = 1_000_000,
                 host_reserve_bytes: int = 2 << 30, small_takes_large: bool = False, large_workers: int = 0,
                 large_yield_ms: int = 10, max_map_edges: int = 4 << 20, pairs_per_edge: float = 40.0,
                 curvelets_per_edge: float = 8.0, device_reserve_bytes: int = 0):
        lib = _abi.load()
        self._lib = lib
        cfg = _abi.CvlServerCfg()
        lib.cvl_server_cfg_default(C.byref(cfg))
        cfg.device, cfg.workers, cfg.mem_budget_bytes = device, workers, mem_budget_bytes
        cfg.admit_bytes_per_edge, cfg.max_batch_edges, cfg.large_map_edges = (admit_bytes_per_edge, max_batch_edges,
                                                                              large_map_edges)
        cfg.host_reserve_bytes = host_reserve_bytes
        cfg.small_takes_large = 1 if small_takes_large else 0
        cfg.large_workers = large_workers
        cfg.large_yield_ms = large_yield_ms
        cfg.max_map_edges, cfg.pairs_per_edge, cfg.curvelets_per_edge = max_map_edges, pairs_per_edge, curvelets_per_edge
        cfg.device_reserve_bytes = device_reserve_bytes
        self._p = (params or CurveletParams()).to_c()
        h = C.c_void_p()
        check(lib.cvl_server_create(C.byref(cfg), C.byref(self._p), C.byref(h)), "cvl_server_create")
        self._h = h

    def submit(self, edges) -> int:
        e = _edges(edges)
        rid = C.c_uint64(0)
        check(self._lib.cvl_server_submit(self._h, e.ctypes.data_as(_abi._dp), e.shape[0], e.shape[1],
                                          C.byref(rid)), "cvl_server_submit")
        return int(rid.value)

    def poll(self, rid: int) -> Result | None:
        r = C.c_void_p()
        rc = self._lib.cvl_server_poll(self._h, rid, C.byref(r))
        if rc == _abi.CVL_EAGAIN:
            return None
        check(rc, "cvl_server_poll")
        return _result_from_handle(self._lib, r)

    def wait(self, rid: int, timeout_s: float | None = None) -> Result:
        """The result; raises CvlError(CVL_ETIMEDOUT) if it is not ready in time."""
        r = C.c_void_p()
        us = -1 if timeout_s is None else int(timeout_s * 1e6)
        check(self._lib.cvl_server_wait(self._h, rid, us, C.byref(r)), "cvl_server_wait")
        return _result_from_handle(self._lib, r)

    def next(self, timeout_s: float | None = None) -> tuple[int, Result] | None:
        """(id, result) of the earliest finished request not handed out yet, in
        completion order; None when nothing is queued or running."""
        r = C.c_void_p()
        rid = C.c_uint64(0)
        us = -1 if timeout_s is None else int(timeout_s * 1e6)
        rc = self._lib.cvl_server_next(self._h, us, C.byref(rid), C.byref(r))
        if rc == _abi.CVL_EAGAIN:
            return None
        check(rc, "cvl_server_next")
        return int(rid.value), _result_from_handle(self._lib, r)

    def stats(self) -> dict:
        st = _abi.CvlServerStats()
        check(self._lib.cvl_server_stats_get(self._h, C.byref(st)), "cvl_server_stats_get")
        return {name: getattr(st, name) for name, _ in st._fields_}

    def latencies(self, with_ids: bool = False):
        """(ms, edges[, ids]) of every completed request, in completion order."""
        n = int(self.stats()["completed"])
        ms = np.zeros(max(n, 1))
        ed = np.zeros(max(n, 1), np.int64)
        ids = np.zeros(max(n, 1), np.uint64)
        k = self._lib.cvl_server_latencies(self._h, ms.ctypes.data_as(_abi._dp),
                                           ed.ctypes.data_as(C.POINTER(C.c_int64)),
                                           ids.ctypes.data_as(C.POINTER(C.c_uint64)), n)
        if k < 0:
            check(int(k), "cvl_server_latencies")
        return (ms[:k], ed[:k], ids[:k]) if with_ids else (ms[:k], ed[:k])

    def request_times(self) -> np.ndarray:
        """cvl_server_request_times: a structured array (id, edges, queue_ms, upload_ms,
        run_ms, result_ms, total_ms, launch_maps, worker) per completed request."""
        n = int(self.stats()["completed"])
        buf = (_abi.CvlRequestTimes * max(n, 1))()
        k = self._lib.cvl_server_request_times(self._h, buf, n)
        if k < 0:
            check(int(k), "cvl_server_request_times")
        dt = np.dtype([(name, np.int64 if name == "edges" else np.uint64 if name == "id" else
                        np.int32 if name in ("launch_maps", "worker") else np.float64)
                       for name, _ in _abi.CvlRequestTimes._fields_], align=True)
        return np.frombuffer(bytes(buf), dtype=dt, count=k).copy() if k else np.zeros(0, dt)

    def close(self):
        if self._h:
            self._lib.cvl_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# The reference's template API, same names and argument meaning
# ---------------------------------------------------------------------------
_default_engine: Engine | None = None


def default_engine() -> Engine:
    global _default_engine
    if _default_engine is None:
        _default_engine = Engine()
    return _default_engine


def pair_bundles_noalloc(pairs, params: CurveletParams | None = None, dt_rad: float = 0.0):
    """Engine.pair_bundles through cvl_pair_bundles_noalloc: no engine, no device
    allocation, a fixed per-device scratch (at most 15,872 pairs of the default
    63-cell grid per call). Returns (bmin [n, cells], bmax [n, cells], valid [n]
    bool, valid_pairs)."""
    lib = _abi.load()
    params = params or CurveletParams()
    q = np.ascontiguousarray(pairs, dtype=np.float64).reshape(-1, 6)
    n = q.shape[0]
    p = params.to_c(dt_rad)
    cells = C.c_int32(0)
    count = C.c_uint32(0)
    u8p = C.POINTER(C.c_uint8)
    one = np.zeros(1)
    # n = 0 sizes the grid without touching the device
    check(lib.cvl_pair_bundles_noalloc(q.ctypes.data_as(_abi._dp), 0, C.byref(p), one.ctypes.data_as(_abi._dp),
                                       one.ctypes.data_as(_abi._dp), np.zeros(1, np.uint8).ctypes.data_as(u8p),
                                       C.byref(count), C.byref(cells)), "cvl_pair_bundles_noalloc")
    nc = cells.value
    bmin = np.zeros((max(n, 1), nc))
    bmax = np.zeros((max(n, 1), nc))
    valid = np.zeros(max(n, 1), np.uint8)
    check(lib.cvl_pair_bundles_noalloc(q.ctypes.data_as(_abi._dp), n, C.byref(p), bmin.ctypes.data_as(_abi._dp),
                                       bmax.ctypes.data_as(_abi._dp), valid.ctypes.data_as(u8p), C.byref(count),
                                       C.byref(cells)), "cvl_pair_bundles_noalloc")
    return bmin[:n], bmax[:n], valid[:n].astype(bool), int(count.value)


@dataclass
class GPUNeighborGraph:
    """CPUNeighborGraph<T> (preprocess.hpp:18-31): CSR over anchors in input order,
    neighbour lists sorted by ascending squared distance."""
    num_edges: int = 0
    total_neighbor_pairs: int = 0
    max_num_of_neighbors: int = 0
    edges: np.ndarray = field(default_factory=lambda: np.zeros((0, 4)))
    neighbor_offsets: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int32))
    neighbor_ids: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    neighbor_dist2: np.ndarray = field(default_factory=lambda: np.zeros(0))
    truncated_anchors: int = 0
    _h: object = None
    _eng: object = None

    @classmethod
    def _from_handle(cls, eng: Engine, h, edges: np.ndarray) -> "GPUNeighborGraph":
        v = CvlGraphView()
        check(eng._lib.cvl_graph_get(h, C.byref(v)), "cvl_graph_get")
        n, p = int(v.num_edges), int(v.total_neighbor_pairs)
        g = cls()
        g._fill(eng, h, edges, v, n, p)
        return g

    def _fill(self, eng, h, edges, v, n, p):
        self.num_edges, self.total_neighbor_pairs = n, p
        self.max_num_of_neighbors = int(v.max_num_of_neighbors)
        self.truncated_anchors = int(v.truncated_anchors)
        self.edges = edges
        self.neighbor_offsets = np.ctypeslib.as_array(v.neighbor_offsets, shape=(n + 1,)).copy()
        self.neighbor_ids = (np.ctypeslib.as_array(v.neighbor_ids, shape=(p,)).copy() if p
                             else np.zeros(0, np.int32))
        self.neighbor_dist2 = (np.ctypeslib.as_array(v.neighbor_dist2, shape=(p,)).copy() if p
                               else np.zeros(0))
        if self._h is not None and self._eng is not None:
            self._eng._lib.cvl_graph_free(self._h)
        self._h, self._eng = h, eng

    def __del__(self):
        try:
            if self._h is not None and self._eng is not None and self._eng._h:
                self._eng._lib.cvl_graph_free(self._h)
                self._h = None
        except Exception:
            pass


def build_neighbor_csr_graph(num_edges: int, sz_edge_data: int, edges, rad: float, neighbor_radius: int,
                             max_candidates: int, nthreads: int, graph: GPUNeighborGraph,
                             engine: Engine | None = None) -> bool:
    """build_neighbor_csr_graph<T> (preprocess.hpp:186-274): returns False on
    num_edges <= 0, sz_edge_data < 4 or no edges, as the reference does."""
    del nthreads  # the GPU path has no host thread count
    if num_edges <= 0 or sz_edge_data < 4 or edges is None:
        return False
    e = np.ascontiguousarray(edges, dtype=np.float64).reshape(-1)[: num_edges * sz_edge_data]
    e = e.reshape(num_edges, sz_edge_data)
    eng = engine or default_engine()
    g = eng.build_neighbor_graph(e, rad, neighbor_radius, max_candidates)
    # move the arrays and the handle over to the caller's graph object
    if graph._h is not None and graph._eng is not None:
        graph._eng._lib.cvl_graph_free(graph._h)
    for k in ("num_edges", "total_neighbor_pairs", "max_num_of_neighbors", "edges", "neighbor_offsets",
              "neighbor_ids", "neighbor_dist2", "truncated_anchors"):
        setattr(graph, k, getattr(g, k))
    graph._h, graph._eng = g._h, g._eng
    g._h = None
    return True


@dataclass
class CurveletFormationResult:
    """CPUCurveletFormationResult (cpu_curvelet.hpp:18-20)."""
    valid_pairs: int = 0


class CurveletGPU:
    """CurveletCPU<T> (cpu_curvelet.hpp:22-123) on the GPU. The constructor takes
    the reference's arguments (dt in radians); the outputs are exposed under the
    reference's member names:

    * ``_edge_chain_final``: [num_curvelets, chain_width] uint32, 1-based ids;
    * ``_curvelet_info``: column-major like the reference ([10, num_curvelets],
      _curvelet_info[col, row]); ``curvelet_info_rows`` is the row-major file layout.
    """

    def __init__(self, num_edges: int, sz_edge_data: int, csr: GPUNeighborGraph, dx: float, dt: float, sx: float,
                 st: float, max_k: float, group_max_sz: int, nthreads: int, to_edges, nrad: float,
                 engine: Engine | None = None):
        del nthreads, to_edges  # edges come from the graph, as the reference reads csr.edges
        self._n, self._sz, self._csr = num_edges, sz_edge_data, csr
        self._dt = dt
        self._params = CurveletParams(nrad=nrad, dx=dx, dt_deg=dt * 180.0 / M_PI, max_k=max_k, sx=sx, st=st,
                                      group_max_sz=group_max_sz, edge_data_sz=sz_edge_data)
        self._eng = engine or csr._eng or default_engine()
        self._group_max_sz = group_max_sz
        self._num_curvelets = 0
        self._edge_chain_final = np.zeros((0, group_max_sz + 1), np.uint32)
        self._curvelet_info = np.zeros((10, 0))
        self.curvelet_info_rows = np.zeros((0, 10))
        self._max_curvelets = num_edges * (csr.max_num_of_neighbors + 1) * 2  # cpu_curvelet.hpp:64

    def form_pairwise_bundles(self, result: CurveletFormationResult) -> bool:
        result.valid_pairs = self._eng.form_pairwise_bundles(self._csr, self._params, dt_rad=self._dt)
        return True

    def build_curvelets_greedy(self) -> None:
        r = self._eng.build_curvelets(self._csr, self._params, dt_rad=self._dt)
        self._num_curvelets = r.num_curvelets
        self._edge_chain_final = r.chains
        self.curvelet_info_rows = r.info
        self._curvelet_info = r.info.T
        self.last_result = r

    def num_curvelets(self) -> int:
        return self._num_curvelets

    def chain_width(self) -> int:
        return self._group_max_sz + 1


def run_curvelet(edges, params: CurveletParams | None = None, engine: Engine | None = None) -> Result:
    """run_curvelet<double> (main.cpp:20-96) without the file I/O."""
    return (engine or default_engine()).run(edges, params or CurveletParams())
