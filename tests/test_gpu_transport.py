"""The path's bundle transport on the GPU, at the operands where its rewrite has
a special case, bit for bit.

The bundle kernel k_bundles runs bundle_column_fp64 (csrc/cvl_path.cuh): the
reference's per-cell formulas (compute_curve_bundle, cpu_curvelet.hpp:693-809)
rewritten into fewer operations with the same correctly rounded values, and one
special case: a branch-2 cell whose denominator e1 cancels to +0 negates its two
k_dx quotients, because the reference's own branch-2 denominator is -0 there
(:774). cvl_pair_bundles runs the same device function per pair, and
cvl_check_transport_cells runs it on operand sets given directly, so these tests
reach that code at chosen operands:

- operand sets (no trig, every operation IEEE): the device result equals the
  reference's expressions as written, evaluated here with one rounding per
  operation, bit for bit, on the path's operand ranges, on other grids, on cells
  built to cancel (exact +0 denominators in both branches) and on zero
  distances, with the k_dx quotient pair formed both ways the kernel forms it
  (two divisions; one reciprocal and Markstein's corrections); the number of
  branch-2 cells that take the negation is counted and must be positive;
- pairs: the reference's compute_curve_bundle on 64 pairs and on 256 pairs whose
  centre cell cancels to +0 in branch 2 (tests/golden/pair_bundles_cancel.npz):
  the path's arithmetic equals the literal two-branch form on the same device
  trig bit for bit; against the reference, pair validity, cell validity and the
  +0 cells' (+inf, -inf) are exact and the other bounds within 1e-9 relative
  (glibc and CUDA sin/cos differ by a few ulps).
"""
import os

import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def grid(sx, dx):
    P = int(2 * np.floor(dx / sx + 0.5) + 1)  # cpu_curvelet.hpp:73
    return np.array([sx * (float(i) - (float(P) - 1.0) / 2.0) for i in range(P)])  # :697


def reference_columns(ops, d2, dx, max_k):
    """cpu_curvelet.hpp:693-809 as written, for one orientation sample per row:
    numpy double arithmetic, one rounding per operation, no fused multiply-add."""
    DX, DY, tt, s_m, s_p, cm, sm, cp, sp, b1 = (ops[:, k] for k in range(10))
    b1 = b1 != 0.0
    DX2, DY2, _dx2 = DX * DX, DY * DY, dx * dx
    sin_T0pdt_times_DY, cos_T0pdt_times_DX = DY * sp, DX * cp
    sin_T0mdt_times_DY, cos_T0mdt_times_DX = DY * sm, DX * cm
    n, P = ops.shape[0], len(d2)
    bmin, bmax = np.empty((n, P)), np.empty((n, P))
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        for i, delta_x2 in enumerate(d2):
            ttmdx2 = tt - delta_x2
            lo, hi = np.full(n, -max_k), np.full(n, max_k)
            # branch 1 (:706-744)
            eq1 = (-2.0 * delta_x2 * tt + DX2 + DY2 - _dx2 + delta_x2 * delta_x2)
            k1_dx_min = 2.0 * (ttmdx2 - dx) / eq1
            k1_dx_max = 2.0 * (ttmdx2 + dx) / eq1
            # branch 2 (:770-800)
            eq2 = -(2.0 * delta_x2 * tt - DX2 - DY2 + _dx2 - delta_x2 * delta_x2) / 2.0
            k2_dx_min = (ttmdx2 - dx) / eq2
            k2_dx_max = (ttmdx2 + dx) / eq2
            k_dt_m = s_m / (-s_m * delta_x2 + cos_T0mdt_times_DX + sin_T0mdt_times_DY)
            k_dt_p = s_p / (-s_p * delta_x2 + cos_T0pdt_times_DX + sin_T0pdt_times_DY)
            kdx_min = np.where(b1, k1_dx_min, k2_dx_min)
            kdx_max = np.where(b1, k1_dx_max, k2_dx_max)
            lo = np.where(lo < kdx_min, kdx_min, lo)
            hi = np.where(hi > kdx_max, kdx_max, hi)
            kdt_min = np.where(b1, k_dt_m, k_dt_p)
            kdt_max = np.where(b1, k_dt_p, k_dt_m)
            lo = np.where(lo < kdt_min, kdt_min, lo)
            hi = np.where(hi > kdt_max, kdt_max, hi)
            bmin[:, i], bmax[:, i] = lo, hi
    return bmin, bmax


def negated_cells(ops, d2, dx):
    """Branch-2 cells whose rewritten denominator e1 is +0 (the cells the kernel negates)."""
    DX, DY, tt = ops[:, 0], ops[:, 1], ops[:, 2]
    b2 = ops[:, 9] == 0.0
    hits = 0
    for d in d2:
        e1 = (((DX * DX - (2.0 * d) * tt) + DY * DY) - dx * dx) + d * d
        hits += int(np.sum((e1 == 0.0) & b2))
    return hits


def random_ops(rng, n, scale):
    DX = rng.uniform(-scale, scale, n)
    DY = rng.uniform(-scale, scale, n)
    tt = rng.uniform(-1.5 * scale, 1.5 * scale, n)
    th = rng.uniform(-np.pi, np.pi, (n, 2))
    s = rng.uniform(-1.0, 1.0, (n, 2))
    b1 = (rng.random(n) < 0.5).astype(np.float64)
    return np.column_stack([DX, DY, tt, s[:, 0], s[:, 1], np.cos(th[:, 0]), np.sin(th[:, 0]), np.cos(th[:, 1]),
                            np.sin(th[:, 1]), b1])


def cancelling_ops(rng, n, d, dx):
    """tt chosen so that -2 d tt + DX^2 + DY^2 - dx^2 + d^2 is about 0, then moved
    by a few ulps: denominators that cancel to (nearly) zero, exact +0 included."""
    ops = random_ops(rng, n, 3.5)
    DX, DY = ops[:, 0], ops[:, 1]
    tt = (DX * DX + DY * DY - dx * dx + d * d) / (2.0 * d)
    ops[:, 2] = tt * (1.0 + rng.integers(-4, 5, n) * 2.0 ** -52)
    return ops


def check_ops(engine, ops, params):
    """Both forms of the rewrite's k_dx quotients (two divisions; one reciprocal with
    Markstein's corrections) and the literal form, against the reference, bit for bit."""
    d2 = grid(params.sx, params.dx)
    emin, emax = reference_columns(ops, d2, params.dx, params.max_k)
    for shared in (False, True):
        rmin, rmax, lmin, lmax = engine.transport_cells(ops, params, shared_quotients=shared)
        for got, want in ((rmin, emin), (rmax, emax), (lmin, emin), (lmax, emax)):
            assert got.shape == want.shape
            bad = got.view(np.uint64) != want.view(np.uint64)
            assert not bad.any(), f"shared={shared}: {int(bad.sum())} cells differ; first {np.argwhere(bad)[:3].tolist()}"
    return negated_cells(ops, d2, params.dx)


def test_transport_cells_path_ranges(engine):
    rng = np.random.default_rng(31)
    p = cvl.CurveletParams()
    for scale in (3.5, 0.9):
        check_ops(engine, random_ops(rng, 100_000, scale), p)


def test_transport_cells_other_grids(engine):
    rng = np.random.default_rng(32)
    for kw in (dict(sx=0.05, dx=0.4), dict(sx=0.3, dx=0.9), dict(sx=0.17, dx=0.6, max_k=0.7)):
        check_ops(engine, random_ops(rng, 40_000, 50.0), cvl.CurveletParams(**kw))


def test_transport_cells_cancelling_denominators(engine):
    """Cells built to cancel, in both branches: the device's rewritten arithmetic
    equals the reference's expressions bit for bit, and the branch-2 cells with
    e1 == +0 (where the kernel negates the quotients) are reached."""
    rng = np.random.default_rng(33)
    p = cvl.CurveletParams()
    hits = 0
    for d in grid(p.sx, p.dx):
        if d == 0.0:
            continue
        hits += check_ops(engine, cancelling_ops(rng, 50_000, d, p.dx), p)
    # zero distance: e1 = (((0 - 2d * 0) + 0) - dx^2) + d^2 is +0 wherever |d| == dx
    z = random_ops(rng, 2000, 1.0)
    z[:, 0] = z[:, 1] = z[:, 2] = 0.0
    hits += check_ops(engine, z, p)
    print(f"[transport] branch-2 cells with e1 == +0 reached on the device: {hits}")
    assert hits > 100


def test_pair_bundles_production_equals_literal(engine, golden_pairs):
    """cvl_pair_bundles (the path's arithmetic) and the literal two-branch form,
    on the same device trig values: bit for bit."""
    for pairs, prm in ((golden_pairs["pairs"], cvl.CurveletParams()),
                       (np.load(os.path.join(GOLDEN, "pair_bundles_cancel.npz"))["pairs"],
                        cvl.CurveletParams(sx=0.5))):
        a = engine.pair_bundles(pairs, prm)
        b = engine.pair_bundles(pairs, prm, literal=True)
        assert np.array_equal(a[2], b[2])
        assert np.array_equal(a[0].view(np.uint64), b[0].view(np.uint64))
        assert np.array_equal(a[1].view(np.uint64), b[1].view(np.uint64))


def test_pair_bundles_cancelling_cells_vs_reference(engine):
    """256 pairs whose centre cell's e1 is +0 in branch 2: the reference closes
    that cell with (+inf, -inf); the path's arithmetic on the GPU gives the same
    cell bit for bit, and the same pair and cell validity everywhere."""
    z = np.load(os.path.join(GOLDEN, "pair_bundles_cancel.npz"))
    prm = cvl.CurveletParams(sx=float(z["params"][0]))
    bmin, bmax, valid = engine.pair_bundles(z["pairs"], prm)
    rmin, rmax = z["bmin"], z["bmax"]
    n = len(valid)
    c = z["cell"]
    assert np.array_equal(bmin[np.arange(n), c], np.full(n, np.inf))
    assert np.array_equal(bmax[np.arange(n), c], np.full(n, -np.inf))
    assert np.array_equal(valid, z["valid"].astype(bool))
    assert np.array_equal(bmax > bmin, rmax > rmin)
    fin = np.isfinite(rmin) & np.isfinite(rmax)
    assert np.array_equal(np.isfinite(bmin) & np.isfinite(bmax), fin)
    for a, b in ((bmin[fin], rmin[fin]), (bmax[fin], rmax[fin])):
        assert np.all(np.abs(a - b) <= np.maximum(1e-9 * np.maximum(np.abs(a), np.abs(b)), 1e-9 * 0.3))
    same = np.mean(bmin.view(np.uint64) == rmin.view(np.uint64)), np.mean(bmax.view(np.uint64) == rmax.view(np.uint64))
    print(f"[transport] cancelling pairs: {int(valid.sum())}/{n} valid; bit-identical cells {same[0]:.4f} / {same[1]:.4f}")
