"""ctypes binding of libcvl.so (include/cvl.h). No fallback: importing the
package on a machine without the built library raises, and every call that
needs a GPU fails with the engine's own error when none is present."""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libcvl.so")

CVL_OK = 0
CVL_EINVAL = -1
CVL_ENOMEM = -2
CVL_ECUDA = -3
CVL_EUNSUPPORTED = -4
CVL_ETIMEDOUT = -5
CVL_EOVERFLOW = -6
CVL_EAGAIN = -7
CVL_ENODEV = -8

ERRNAMES = {0: "CVL_OK", -1: "CVL_EINVAL", -2: "CVL_ENOMEM", -3: "CVL_ECUDA", -4: "CVL_EUNSUPPORTED",
            -5: "CVL_ETIMEDOUT", -6: "CVL_EOVERFLOW", -7: "CVL_EAGAIN", -8: "CVL_ENODEV"}


class CvlParams(C.Structure):
    _fields_ = [("nrad", C.c_double), ("gap", C.c_double), ("dx", C.c_double), ("dt_deg", C.c_double),
                ("dt_rad", C.c_double), ("max_k", C.c_double), ("curvelet_style", C.c_uint),
                ("group_max_sz", C.c_uint), ("out_type", C.c_uint), ("sx", C.c_double), ("st", C.c_double),
                ("edge_data_sz", C.c_int), ("max_candidates", C.c_uint)]


class CvlEngineCfg(C.Structure):
    _fields_ = [("device", C.c_int), ("mem_budget_bytes", C.c_size_t), ("cell_size", C.c_int),
                ("seeds_per_group", C.c_int), ("bundle_slots", C.c_int), ("warps_per_block", C.c_int),
                ("stream_priority", C.c_int)]


class CvlResultView(C.Structure):
    _fields_ = [("num_curvelets", C.c_uint32), ("chain_width", C.c_uint32),
                ("chains", C.POINTER(C.c_uint32)), ("info", C.POINTER(C.c_double)),
                ("valid_pairs", C.c_uint32), ("total_neighbor_pairs", C.c_int64),
                ("max_num_of_neighbors", C.c_uint32), ("truncated_anchors", C.c_uint32),
                ("num_edges", C.c_uint32), ("flags", C.c_uint32), ("device_ms", C.c_double)]


class CvlGraphView(C.Structure):
    _fields_ = [("num_edges", C.c_int32), ("total_neighbor_pairs", C.c_int64),
                ("max_num_of_neighbors", C.c_uint32), ("truncated_anchors", C.c_uint32),
                ("neighbor_offsets", C.POINTER(C.c_int32)), ("neighbor_ids", C.POINTER(C.c_int32)),
                ("neighbor_dist2", C.POINTER(C.c_double))]


class CvlBatchStats(C.Structure):
    _fields_ = [("device_ms", C.c_double), ("num_curvelets", C.c_uint64), ("valid_pairs", C.c_uint64),
                ("total_pairs", C.c_uint64), ("close_pairs", C.c_uint64), ("max_num_of_neighbors", C.c_uint32),
                ("truncated_anchors", C.c_uint32), ("num_maps", C.c_uint32), ("launches", C.c_uint32)]


class CvlServerCfg(C.Structure):
    _fields_ = [("device", C.c_int), ("workers", C.c_int), ("mem_budget_bytes", C.c_size_t),
                ("admit_bytes_per_edge", C.c_size_t), ("max_batch_edges", C.c_int64),
                ("large_map_edges", C.c_int64), ("host_reserve_bytes", C.c_size_t),
                ("small_takes_large", C.c_int), ("large_workers", C.c_int), ("large_yield_ms", C.c_int),
                ("device_reserve_bytes", C.c_size_t), ("max_map_edges", C.c_int64), ("pairs_per_edge", C.c_double),
                ("curvelets_per_edge", C.c_double)]


class CvlServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("completed", C.c_uint64), ("failed", C.c_uint64),
                ("queued", C.c_uint64), ("in_flight", C.c_uint64), ("launches", C.c_uint64),
                ("edges_completed", C.c_uint64), ("admitted_bytes", C.c_size_t), ("p50_ms", C.c_double),
                ("p95_ms", C.c_double), ("p99_ms", C.c_double), ("max_ms", C.c_double),
                ("upload_ms", C.c_double), ("run_ms", C.c_double), ("device_ms", C.c_double),
                ("result_ms", C.c_double), ("queue_ms", C.c_double), ("device_grows", C.c_uint64),
                ("device_grow_ms", C.c_double), ("host_grows", C.c_uint64), ("host_grow_ms", C.c_double),
                ("reserved_bytes", C.c_size_t)]


class CvlRequestTimes(C.Structure):
    _fields_ = [("id", C.c_uint64), ("edges", C.c_int64), ("queue_ms", C.c_double), ("upload_ms", C.c_double),
                ("run_ms", C.c_double), ("result_ms", C.c_double), ("total_ms", C.c_double),
                ("launch_maps", C.c_int32), ("worker", C.c_int32)]


class CvlEngineGraphs(C.Structure):
    _fields_ = [("enabled", C.c_int32), ("graphs", C.c_int32), ("captures", C.c_uint64), ("replays", C.c_uint64),
                ("fallbacks", C.c_uint64)]


class CvlEngineMemory(C.Structure):
    _fields_ = [("held_bytes", C.c_size_t), ("device_grows", C.c_uint64), ("device_grow_ms", C.c_double)]


class CvlWorkspaceShape(C.Structure):
    _fields_ = [("num_edges", C.c_int64), ("num_pairs", C.c_int64), ("num_curvelets", C.c_int64),
                ("num_maps", C.c_int32), ("edge_data_sz", C.c_int32)]


class CvlTuning(C.Structure):
    _fields_ = [("cell_size", C.c_int), ("bundle_blocks_per_sm", C.c_int), ("growth_blocks_per_sm", C.c_int),
                ("seeds_per_group", C.c_int), ("anchors_per_warp", C.c_int), ("chunk_pairs", C.c_int64)]


CVL_TUNING_BUCKETS = 4


class CvlDeviceResults(C.Structure):
    _fields_ = [("num_curvelets", C.c_uint32), ("chain_width", C.c_uint32), ("chains", C.c_void_p),
                ("info", C.c_void_p), ("done_event", C.c_void_p)]


class CvlContourParams(C.Structure):
    _fields_ = [("min_group_size", C.c_uint32), ("gap", C.c_double), ("fit_polyarcs", C.c_int), ("dx", C.c_double),
                ("dt_rad", C.c_double), ("max_k", C.c_double), ("rad", C.c_double), ("token_len", C.c_double)]


class CvlContoursView(C.Structure):
    _fields_ = [("num_links", C.c_int64), ("link_parent", C.POINTER(C.c_int32)),
                ("link_child", C.POINTER(C.c_int32)), ("link_votes", C.POINTER(C.c_int32)),
                ("num_fragments", C.c_int64), ("fragment_offsets", C.POINTER(C.c_int64)),
                ("fragment_ids", C.POINTER(C.c_int32)), ("max_fragment_length", C.c_int32),
                ("num_edges", C.c_int32), ("device_ms", C.c_float), ("num_polyarcs", C.c_int64),
                ("polyarc_offsets", C.POINTER(C.c_int64)), ("polyarc_ids", C.POINTER(C.c_int32)),
                ("polyarc_info", C.POINTER(C.c_double))]

# (name, restype, argtypes) of every entry point declared in include/cvl.h
_vp = C.c_void_p
_dp = C.POINTER(C.c_double)
SIGNATURES = [
    ("cvl_params_default", None, [C.POINTER(CvlParams)]),
    ("cvl_engine_cfg_default", None, [C.POINTER(CvlEngineCfg)]),
    ("cvl_engine_create", C.c_int, [C.POINTER(CvlEngineCfg), C.POINTER(_vp)]),
    ("cvl_engine_destroy", None, [_vp]),
    ("cvl_last_error", C.c_char_p, []),
    ("cvl_version", C.c_char_p, []),
    ("cvl_run", C.c_int, [_vp, _dp, C.c_int32, C.c_int32, C.POINTER(CvlParams), C.POINTER(_vp)]),
    ("cvl_run_f32", C.c_int, [_vp, C.POINTER(C.c_float), C.c_int32, C.c_int32, C.POINTER(CvlParams), C.POINTER(_vp)]),
    ("cvl_result_get", C.c_int, [_vp, C.POINTER(CvlResultView)]),
    ("cvl_result_free", None, [_vp]),
    ("cvl_build_neighbor_graph", C.c_int, [_vp, _dp, C.c_int32, C.c_int32, C.c_double, C.c_uint, C.c_uint,
                                           C.POINTER(_vp)]),
    ("cvl_graph_get", C.c_int, [_vp, C.POINTER(CvlGraphView)]),
    ("cvl_graph_free", None, [_vp]),
    ("cvl_form_pairwise_bundles", C.c_int, [_vp, _vp, C.POINTER(CvlParams), C.POINTER(C.c_uint32)]),
    ("cvl_build_curvelets", C.c_int, [_vp, _vp, C.POINTER(CvlParams), C.POINTER(_vp)]),
    ("cvl_pair_bundles", C.c_int, [_vp, _dp, C.c_int32, C.POINTER(CvlParams), _dp, _dp,
                                   C.POINTER(C.c_uint8), C.POINTER(C.c_int32)]),
    ("cvl_engine_workspace_bytes", C.c_int, [_vp, C.POINTER(CvlWorkspaceShape), C.POINTER(CvlParams),
                                            C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    ("cvl_engine_reserve_workspace", C.c_int, [_vp, C.POINTER(CvlWorkspaceShape), C.POINTER(CvlParams)]),
    ("cvl_engine_memory_get", C.c_int, [_vp, C.POINTER(CvlEngineMemory)]),
    ("cvl_engine_warmup", C.c_int, [_vp]),
    ("cvl_engine_set_graphs", C.c_int, [_vp, C.c_int]),
    ("cvl_engine_graph_stats", C.c_int, [_vp, C.POINTER(CvlEngineGraphs)]),
    ("cvl_debug_fail_allocations", C.c_int, [C.c_int64]),
    ("cvl_check_pair_bundles_literal", C.c_int, [_vp, _dp, C.c_int32, C.POINTER(CvlParams), _dp, _dp,
                                                 C.POINTER(C.c_uint8), C.POINTER(C.c_int32)]),
    ("cvl_check_transport_cells", C.c_int, [_vp, _dp, C.c_int32, C.POINTER(CvlParams), C.c_int32, _dp,
                                            C.POINTER(C.c_int32)]),
    ("cvl_pair_bundles_noalloc", C.c_int, [_dp, C.c_int32, C.POINTER(CvlParams), _dp, _dp, C.POINTER(C.c_uint8),
                                           C.POINTER(C.c_uint32), C.POINTER(C.c_int32)]),
    ("cvl_batch_upload", C.c_int, [_vp, _dp, C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.POINTER(_vp)]),
    ("cvl_batch_refill", C.c_int, [_vp, _dp, C.POINTER(C.c_int32), C.c_int32, C.c_int32]),
    ("cvl_batch_refill_parts", C.c_int, [_vp, C.POINTER(_dp), C.POINTER(C.c_int32), C.c_int32, C.c_int32]),
    ("cvl_batch_free", None, [_vp]),
    ("cvl_batch_run", C.c_int, [_vp, _vp, C.POINTER(CvlParams), C.POINTER(_vp)]),
    ("cvl_batch_result_map", C.c_int, [_vp, C.c_int32, C.POINTER(CvlResultView)]),
    ("cvl_batch_result_take_map", C.c_int, [_vp, C.c_int32, C.POINTER(_vp)]),
    ("cvl_batch_result_stats", C.c_int, [_vp, C.POINTER(CvlBatchStats)]),
    ("cvl_batch_result_free", None, [_vp]),
    ("cvl_server_cfg_default", None, [C.POINTER(CvlServerCfg)]),
    ("cvl_server_create", C.c_int, [C.POINTER(CvlServerCfg), C.POINTER(CvlParams), C.POINTER(_vp)]),
    ("cvl_server_submit", C.c_int, [_vp, _dp, C.c_int32, C.c_int32, C.POINTER(C.c_uint64)]),
    ("cvl_server_poll", C.c_int, [_vp, C.c_uint64, C.POINTER(_vp)]),
    ("cvl_server_wait", C.c_int, [_vp, C.c_uint64, C.c_int64, C.POINTER(_vp)]),
    ("cvl_server_next", C.c_int, [_vp, C.c_int64, C.POINTER(C.c_uint64), C.POINTER(_vp)]),
    ("cvl_server_stats_get", C.c_int, [_vp, C.POINTER(CvlServerStats)]),
    ("cvl_server_request_times", C.c_int64, [_vp, C.POINTER(CvlRequestTimes), C.c_int64]),
    ("cvl_server_latencies", C.c_int64, [_vp, _dp, C.POINTER(C.c_int64), C.POINTER(C.c_uint64), C.c_int64]),
    ("cvl_server_destroy", None, [_vp]),
    ("cvl_read_edges", C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.POINTER(_dp), C.POINTER(C.c_int64)]),
    ("cvl_read_edges_f32", C.c_int, [C.c_char_p, C.c_int32, C.c_int32, C.POINTER(C.POINTER(C.c_float)),
                                     C.POINTER(C.c_int64)]),
    ("cvl_free_edges", None, [_vp]),
    ("cvl_write_edges_binary", C.c_int, [C.c_char_p, _dp, C.c_int64, C.c_int32]),
    ("cvl_tuning_bucket", C.c_int, [C.c_int64]),
    ("cvl_engine_get_tuning", C.c_int, [_vp, C.c_int, C.POINTER(CvlTuning)]),
    ("cvl_engine_set_tuning", C.c_int, [_vp, C.c_int, C.POINTER(CvlTuning)]),
    ("cvl_engine_autotune", C.c_int, [_vp, _vp, C.POINTER(CvlParams), C.c_int, C.POINTER(CvlTuning), _dp]),
    ("cvl_engine_flush_l2", C.c_int, [_vp]),
    ("cvl_engine_last_kernel_times", C.c_int, [_vp, C.POINTER(C.c_char_p), _dp, C.c_int]),
    ("cvl_engine_last_launch_count", C.c_int, [_vp]),
    ("cvl_measure_fp64_peak", C.c_int, [_vp, _dp]),
    ("cvl_run_device", C.c_int, [_vp, _vp, C.c_int32, C.c_int32, C.POINTER(CvlParams), _vp, C.POINTER(_vp)]),
    ("cvl_engine_device_results", C.c_int, [_vp, C.POINTER(CvlDeviceResults)]),
    ("cvl_run_maps", C.c_int, [_vp, _dp, C.POINTER(C.c_int32), C.c_int32, C.c_int32, C.POINTER(CvlParams),
                               C.c_int64, C.POINTER(_vp)]),
    ("cvl_contour_params_default", None, [C.POINTER(CvlContourParams)]),
    ("cvl_link_contours", C.c_int, [_vp, _dp, C.c_int32, C.c_int32, C.POINTER(C.c_uint32), C.c_int64, C.c_int32,
                                    C.POINTER(CvlContourParams), C.POINTER(_vp)]),
    ("cvl_run_contours", C.c_int, [_vp, _dp, C.c_int32, C.c_int32, C.POINTER(CvlParams),
                                   C.POINTER(CvlContourParams), C.POINTER(_vp), C.POINTER(_vp)]),
    ("cvl_contours_get", C.c_int, [_vp, C.POINTER(CvlContoursView)]),
    ("cvl_contours_free", None, [_vp]),
]

_lib = None


def load() -> C.CDLL:
    """Loads libcvl.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libcvl.so is not built ({LIB_PATH}); run "
                              "`python -m curvelet_construction_on_gpu_b200.build`")
        lib = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


class CvlError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        msg = load().cvl_last_error().decode(errors="replace")
        super().__init__(f"{what}: {ERRNAMES.get(code, code)}: {msg}")


def check(code: int, what: str) -> None:
    if code != CVL_OK:
        raise CvlError(code, what)
