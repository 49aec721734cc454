"""Edge-file input and chain/info file output in the reference's formats
(cpu_curvelet/data_io.hpp:11-145)."""
from __future__ import annotations

import os

import numpy as np


def edge_input_path(filename: str, base_dir: str = "../test_files") -> str:
    """edge_input_path (data_io.hpp:11-14)."""
    return os.path.join(base_dir, filename)


def read_TO_edges_from_file(filename: str, values_per_edge: int = 4, base_dir: str = "../test_files") -> np.ndarray:
    """read_TO_edges_from_file (data_io.hpp:22-79): exactly values_per_edge numbers
    per line, no blank lines, at least one edge. Raises ValueError where the
    reference prints an error and returns false."""
    path = edge_input_path(filename, base_dir)
    if not os.path.exists(path):
        raise FileNotFoundError(f"Error: input file does not exist: {path}")
    rows = []
    with open(path) as fh:
        for ln, line in enumerate(fh, 1):
            if not line.strip(" \t\r\n"):
                raise ValueError(f"Error: blank line at line {ln} in {path} (each line must contain exactly "
                                 f"{values_per_edge} numeric values)")
            toks = line.split()
            vals = []
            for j in range(values_per_edge):
                try:
                    vals.append(float(toks[j]))
                except (IndexError, ValueError):
                    raise ValueError(f"Error: invalid edge file format in {path} at line {ln}: expected "
                                     f"{values_per_edge} numeric values per line, found {j}.") from None
            if len(toks) > values_per_edge:
                raise ValueError(f"Error: invalid edge file format in {path} at line {ln}: expected exactly "
                                 f"{values_per_edge} numeric values per line, found extra data.")
            rows.append(vals)
    if not rows:
        raise ValueError(f"Error: input file contains no valid edges: {path}")
    return np.asarray(rows, dtype=np.float64)


def _write(path: str, rows: np.ndarray, fmt) -> None:
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    with open(path, "w") as fh:
        for r in rows:
            fh.write("".join(fmt(v) + "\t" for v in r) + "\n")


def write_int_array_to_file(filename: str, data: np.ndarray, out_dir: str = "../outputs") -> str:
    """write_int_array_to_file (data_io.hpp:81-107): tab after every value, one row per line."""
    path = os.path.join(out_dir, filename)
    _write(path, np.asarray(data).astype(np.int64), lambda v: str(int(v)))
    return path


def _g6(v: float) -> str:
    # std::ostream default formatting of a double: %g with 6 significant digits
    return "%g" % v


def write_double_array_to_file(filename: str, data: np.ndarray, out_dir: str = "../outputs") -> str:
    """write_double_array_to_file (data_io.hpp:109-134)."""
    path = os.path.join(out_dir, filename)
    _write(path, np.asarray(data, dtype=np.float64), _g6)
    return path


def chain_to_info_filename(chain_file: str) -> str:
    """chain_to_info_filename (data_io.hpp:136-145)."""
    pos = chain_file.find("chain")
    if pos >= 0:
        return chain_file[:pos] + "info" + chain_file[pos + 5:]
    return "info_" + chain_file


def read_edges(path: str, values_per_edge: int = 4, nthreads: int = 0, scalar: str = "double") -> np.ndarray:
    """An edge file through cvl_read_edges: the reference's text format read on
    all cores (same values and error messages as its stream reader), or the
    binary format for a path ending in ".cvle". nthreads -1: the stream reader
    alone. scalar="float" reads as read_TO_edges_from_file<float> (each number
    straight to float32). Raises ValueError with the reference's message on bad
    input."""
    import ctypes as C

    from . import _abi
    lib = _abi.load()
    ctype, fn = (C.c_float, lib.cvl_read_edges_f32) if scalar == "float" else (C.c_double, lib.cvl_read_edges)
    ptr = C.POINTER(ctype)()
    n = C.c_int64(0)
    rc = fn(path.encode(), values_per_edge, nthreads, C.byref(ptr), C.byref(n))
    if rc != 0:
        raise ValueError(lib.cvl_last_error().decode())
    try:
        return np.ctypeslib.as_array(ptr, shape=(int(n.value) * values_per_edge,)).reshape(-1, values_per_edge).copy()
    finally:
        lib.cvl_free_edges(ptr)


def write_edges_binary(path: str, edges: np.ndarray) -> None:
    """The binary edge format (cvl_write_edges_binary): "CVLEDGE1", uint32
    values_per_edge, uint32 0, uint64 num_edges, little-endian float64 rows."""
    import ctypes as C

    from . import _abi
    e = np.ascontiguousarray(edges, dtype=np.float64)
    rc = _abi.load().cvl_write_edges_binary(path.encode(), e.ctypes.data_as(C.POINTER(C.c_double)), e.shape[0],
                                            e.shape[1])
    if rc != 0:
        raise ValueError(_abi.load().cvl_last_error().decode())
