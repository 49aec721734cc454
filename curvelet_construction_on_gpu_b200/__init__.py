"""cvl -- B200-native curvelet construction (the cpu_curvelet path on sm_100a).

The compute path is libcvl.so (hand-written CUDA for sm_100a behind the C ABI
in include/cvl.h). This package is its host-side mirror of the reference
interface; it has no CPU fallback.
"""
from .api import (M_PI, Batch, BatchResult, ContourParams, Contours, CurveletFormationResult, CurveletGPU,
                  CurveletParams, Engine, GPUNeighborGraph, Result, Server, build_neighbor_csr_graph, default_engine, pair_bundles_noalloc,
                  run_curvelet)
from ._abi import CvlError, load as load_library
from .data_io import (chain_to_info_filename, read_TO_edges_from_file, write_double_array_to_file,
                      write_int_array_to_file)

__all__ = ["M_PI", "Batch", "BatchResult", "ContourParams", "Contours", "CurveletFormationResult", "CurveletGPU", "CurveletParams", "Engine",
           "GPUNeighborGraph", "Result", "Server", "build_neighbor_csr_graph", "pair_bundles_noalloc", "default_engine", "run_curvelet", "CvlError",
           "load_library", "chain_to_info_filename", "read_TO_edges_from_file", "write_double_array_to_file",
           "write_int_array_to_file"]
