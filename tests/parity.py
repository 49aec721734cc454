"""Comparison rules for the parity tests.

Chains (anchor, ordered edge ids, zero padding) and the forward flag must be
identical. Info columns whose arithmetic has no transcendental input (forward
flag, reference theta, theta' = To2Pi(theta + dt), length, quality) must be
bit-identical. The columns that carry sin/cos/atan2 results (k_max, k_min,
pt_x, pt_y, k) must agree within 1e-9 relative, with a floor of 1e-9 of the
column's natural scale (max_k for curvatures, 1 px for positions): the GPU's
libm and glibc differ by at most a few ulps per call, and k = (k_max + k_min)/2
cancels to values near zero where a relative bound alone is ill-conditioned.

The --float mode (the reference's run_curvelet<float>) keeps the same exact
columns and the same chains. Its sin/cos/atan2 results are float, so the
tolerant columns get 2^-20 relative (8 float ulps) with a floor of 1e-4 of the
column's scale: the curve bundle bounds divide by eq, a float difference of
terms near |tt|^2 that cancels, so an ulp of the terms becomes about 1e-5 of
max_k in k_max / k_min.
"""
from __future__ import annotations

import numpy as np

EXACT_COLS = [0, 3, 6, 8, 9]
TOL_COLS = [1, 2, 4, 5, 7]
REL_TOL = 1e-9
FLOAT_REL_TOL = 2.0 ** -20
FLOAT_FLOOR = 1e-4


def info_scales(max_k: float = 0.3) -> np.ndarray:
    s = np.ones(10)
    s[[1, 2, 7]] = max_k
    return s


def compare_info(a: np.ndarray, b: np.ndarray, max_k: float = 0.3, scalar: str = "double") -> dict:
    """Returns deviation statistics; 'ok' is the pass/fail verdict."""
    rel_tol, floor_frac = (REL_TOL, REL_TOL) if scalar == "double" else (FLOAT_REL_TOL, FLOAT_FLOOR)
    assert a.shape == b.shape, (a.shape, b.shape)
    out = {"rows": int(a.shape[0])}
    if a.shape[0] == 0:
        out.update(ok=True, exact_cols_equal=True, max_rel=0.0, bit_identical_frac=1.0)
        return out
    ex = np.array_equal(a[:, EXACT_COLS].view(np.uint64), b[:, EXACT_COLS].view(np.uint64))
    d = np.abs(a[:, TOL_COLS] - b[:, TOL_COLS])
    mag = np.maximum(np.abs(a[:, TOL_COLS]), np.abs(b[:, TOL_COLS]))
    floor = floor_frac * info_scales(max_k)[TOL_COLS]
    bound = np.maximum(rel_tol * mag, floor)
    within = bool(np.all(d <= bound))
    rel = np.where(mag > 0, d / np.where(mag > 0, mag, 1.0), 0.0)
    out.update(ok=bool(ex and within), exact_cols_equal=bool(ex), max_rel=float(rel.max()),
               max_abs=float(d.max()), within_tol=within,
               bit_identical_frac=float(np.mean(a.view(np.uint64) == b.view(np.uint64))))
    return out


def first_chain_mismatch(a: np.ndarray, b: np.ndarray) -> str:
    n = min(a.shape[0], b.shape[0])
    for i in range(n):
        if not np.array_equal(a[i], b[i]):
            return f"row {i}: gpu {a[i].tolist()} vs oracle {b[i].tolist()}"
    return f"row counts differ: gpu {a.shape[0]} vs oracle {b.shape[0]}"


def assert_same_curvelets(gpu, ref, max_k: float = 0.3, label: str = "", scalar: str = "double") -> dict:
    """gpu/ref expose .chains and .info (numpy)."""
    assert gpu.chains.shape == ref.chains.shape and np.array_equal(gpu.chains, ref.chains), \
        f"{label}: chains differ ({first_chain_mismatch(gpu.chains, ref.chains)})"
    st = compare_info(gpu.info, ref.info, max_k, scalar)
    assert st["ok"], f"{label}: info outside tolerance: {st}"
    return st
