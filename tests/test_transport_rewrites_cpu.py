"""The bundle transport's exact rewrites, checked bit for bit on the CPU.

The FP64 bundle kernel (k_bundles in csrc/cvl_path.cuh, compiled with -fmad=false)
computes the per-cell curvature bounds of compute_curve_bundle
(cpu_curvelet.hpp:693-809) in fewer operations:
  e1   = (((DX2 - (2 dx2) tt) + DY2) - dx^2) + dx2^2     (branch 1's eq_denom, :711)
  k_dx = ((2 tt - 2 dx2) -+ 2 dx) / e1                   (both branches)
Branch 2's eq_denom (:774) is e1 * 0.5 and its k_dx (:777-778) equals branch 1's
form, because round-to-nearest is odd-symmetric and scaling by 2 is exact, with
one exception: where e1 cancels to +0, branch 2's own sum cancels to +0 too
(x - x is +0 in round-to-nearest), so its eq_denom is -0 and its k_dx are the
negated quotients; the kernel negates them there.
These tests evaluate the reference's expressions as written (numpy double
arithmetic, one rounding per operation, no fused multiply-add) against the
rewrite on the operand ranges of the path and beyond."""
import numpy as np


def _grid(sx=0.1, P=9):
    # delta_x2 = _sx * ((T)i - (T(P) - 1.0) / 2.0)  (:697)
    return np.array([sx * (float(i) - (float(P) - 1.0) / 2.0) for i in range(P)])


def _operands(rng, n, scale):
    DX = rng.uniform(-scale, scale, n)
    DY = rng.uniform(-scale, scale, n)
    tt = rng.uniform(-1.5 * scale, 1.5 * scale, n)
    dx = np.full(n, 0.4)
    return DX, DY, tt, dx


def _check(DX, DY, tt, dx, d2):
    DX2, DY2, _dx2 = DX * DX, DY * DY, dx * dx
    ttmdx2 = tt - d2
    # the reference, branch 1 (:711, :714-715)
    eq1 = (-2.0 * d2 * tt + DX2 + DY2 - _dx2 + d2 * d2)
    k1_min = 2.0 * (ttmdx2 - dx) / eq1
    k1_max = 2.0 * (ttmdx2 + dx) / eq1
    # the reference, branch 2 (:774, :777-778)
    eq2 = -(2.0 * d2 * tt - DX2 - DY2 + _dx2 - d2 * d2) / 2.0
    k2_min = (ttmdx2 - dx) / eq2
    k2_max = (ttmdx2 + dx) / eq2
    # the rewrite
    dx2_2 = 2.0 * d2
    e1 = (((DX2 - dx2_2 * tt) + DY2) - _dx2) + d2 * d2
    ttmdx2_2 = 2.0 * tt - dx2_2
    lo2, hi2 = ttmdx2_2 - 2.0 * dx, ttmdx2_2 + 2.0 * dx
    r_min, r_max = lo2 / e1, hi2 / e1
    # branch 2 where e1 is +0: the negated quotients
    z = e1 == 0.0
    r2_min, r2_max = np.where(z, -r_min, r_min), np.where(z, -r_max, r_max)

    def same(a, b):  # bit for bit, any NaN matching any NaN (a NaN bound never wins a clamp)
        nan = np.isnan(a) & np.isnan(b)
        return np.array_equal(a.view(np.uint64)[~nan], b.view(np.uint64)[~nan]) and \
            np.array_equal(np.isnan(a), np.isnan(b))
    assert same(e1, eq1)
    assert same(np.where(z, -0.0, e1 * 0.5), eq2)
    assert same(r_min, k1_min) and same(r_max, k1_max)
    assert same(r2_min, k2_min) and same(r2_max, k2_max)
    return int(np.sum(z))


def test_rewrites_bit_identical_on_path_ranges():
    rng = np.random.default_rng(21)
    with np.errstate(divide="ignore", invalid="ignore"):
        for d2 in _grid():
            for scale in (3.5, 0.9):
                DX, DY, tt, dx = _operands(rng, 200_000, scale)
                _check(DX, DY, tt, dx, np.full_like(DX, d2))


def test_rewrites_bit_identical_beyond_path_ranges():
    """Non-default grids and distances (sx, the uncertainty, radius up to 50 px)."""
    rng = np.random.default_rng(22)
    with np.errstate(divide="ignore", invalid="ignore", over="ignore"):
        for sx, P in ((0.05, 17), (0.3, 5), (0.17, 7)):
            for d2 in _grid(sx, P):
                DX, DY, tt, _ = _operands(rng, 50_000, 50.0)
                dx = rng.uniform(0.01, 2.0, len(DX))
                _check(DX, DY, tt, dx, np.full_like(DX, d2))


def test_rewrite_near_zero_denominator():
    """Cells whose denominator cancels to (nearly) zero, where the quotient is
    huge, infinite or NaN: the rewrite still gives the reference's bits."""
    rng = np.random.default_rng(23)
    d2 = 0.3
    DX = rng.uniform(-3.5, 3.5, 100_000)
    DY = rng.uniform(-3.5, 3.5, 100_000)
    dx = np.full_like(DX, 0.4)
    # choose tt so that -2 d2 tt + DX^2 + DY^2 - dx^2 + d2^2 is about 0
    tt = (DX * DX + DY * DY - dx * dx + d2 * d2) / (2.0 * d2)
    tt = tt * (1.0 + rng.integers(-4, 5, len(tt)) * 2.0 ** -52)
    with np.errstate(divide="ignore", invalid="ignore"):
        zeros = _check(DX, DY, tt, dx, np.full_like(DX, d2))
    assert zeros > 0  # the exception is exercised
