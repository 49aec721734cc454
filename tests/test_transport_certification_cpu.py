"""The ranges behind the bundle kernel's shared-reciprocal quotients (certify_* in
csrc/cvl_kernels.cuh, markstein_quotient in csrc/cvl_path.cuh), checked on the CPU.

A run is certified when every coordinate and the parameters dx, sx are 0 or in
[2^-40, 2^40] in magnitude (coordinates are below 1e9 in any case) and every anchor
trig value sin/cos(T2 + delta_t_j) is 0 or at least 2^-100 in magnitude. The kernel
then relies on every nonzero e1 = (((DX^2 - (2d) tt) + DY^2) - dx^2) + d^2 lying in
[2^-336, 2^94], and every numerator (2 tt - 2 d) -+ 2 dx being +0 or in [2^-243, 2^48]
(never -0), which puts both inside the [2^-500, 2^501) the quotient's proof needs.
This test evaluates those expressions as the kernel does (IEEE double, one rounding
per operation) on random and extreme certified operands, and on operands built to
cancel, and checks the ranges.
"""
import numpy as np

E1_LO, E1_HI = 2.0 ** -336, 2.0 ** 94
NUM_LO, NUM_HI = 2.0 ** -243, 2.0 ** 48


def _certified_values(rng, n, lo_exp, hi_exp, zero_frac=0.05):
    """Doubles of magnitude 0 or in [2^lo_exp, 2^hi_exp], favouring the ends."""
    e = rng.integers(lo_exp, hi_exp, n)
    ends = rng.random(n)
    e = np.where(ends < 0.2, lo_exp, np.where(ends > 0.8, hi_exp - 1, e))
    m = 1.0 + rng.random(n)
    m = np.where(rng.random(n) < 0.1, np.nextafter(2.0, 0.0), m)
    v = np.ldexp(m, e) * np.where(rng.random(n) < 0.5, -1.0, 1.0)
    return np.where(rng.random(n) < zero_frac, 0.0, v)


def _transport_operands(ax, ay, lx, ly, s, c, dx, sx, i, P):
    DX, DY = ax - lx, ay - ly
    tt = s * DX - c * DY
    d = sx * (float(i) - (float(P) - 1.0) / 2.0)
    d2_2 = 2.0 * d
    e1 = (((DX * DX - d2_2 * tt) + DY * DY) - dx * dx) + d * d
    t = 2.0 * tt - d2_2
    return e1, t - 2.0 * dx, t + 2.0 * dx


def _check(e1, lo2, hi2):
    a = np.abs(e1)
    assert np.all((a == 0.0) | ((a >= E1_LO) & (a <= E1_HI))), a[(a != 0) & ((a < E1_LO) | (a > E1_HI))][:5]
    for num in (lo2, hi2):
        b = np.abs(num)
        assert np.all((b == 0.0) | ((b >= NUM_LO) & (b <= NUM_HI)))
        assert not np.any((num == 0.0) & np.signbit(num)), "a numerator is -0"


def test_certified_ranges_random_and_extreme():
    rng = np.random.default_rng(7)
    n = 400_000
    coord_hi = 29  # |coordinate| < 1e9 < 2^30
    for _ in range(5):
        ax, ay, lx, ly = (_certified_values(rng, n, -40, coord_hi) for _ in range(4))
        s = np.clip(_certified_values(rng, n, -100, 1), -1.0, 1.0)
        c = np.clip(_certified_values(rng, n, -100, 1), -1.0, 1.0)
        dx = np.abs(_certified_values(rng, 1, -40, 40, zero_frac=0.0))[0]
        sx = np.abs(_certified_values(rng, 1, -40, 40, zero_frac=0.0))[0]
        P = int(min(2 * np.floor(dx / sx + 0.5) + 1, 127))
        for i in (0, P // 2, P - 1):
            with np.errstate(over="ignore", invalid="ignore"):
                e1, lo2, hi2 = _transport_operands(ax, ay, lx, ly, s, c, dx, sx, i, P)
            ok = np.isfinite(e1)
            _check(e1[ok], lo2[ok], hi2[ok])


def test_certified_ranges_cancelling():
    """Operands whose e1 cancels to zero or nearly (tt placed at the root of e1, then
    moved by a few ulps), at the default grid: nonzero results stay in range."""
    rng = np.random.default_rng(8)
    n = 400_000
    dx, sx = 0.4, 0.1
    P = 9
    ax = rng.uniform(0, 2000, n)
    ay = rng.uniform(0, 2000, n)
    lx = ax + rng.uniform(-3.5, 3.5, n)
    ly = ay + rng.uniform(-3.5, 3.5, n)
    th = rng.uniform(0, 2 * np.pi, n)
    s, c = np.sin(th), np.cos(th)
    for i in range(P):
        d = sx * (float(i) - (float(P) - 1.0) / 2.0)
        if d == 0.0:
            continue
        DX, DY = ax - lx, ay - ly
        root = (DX * DX + DY * DY - dx * dx + d * d) / (2.0 * d)
        # choose the anchor trig so that tt = s DX - c DY hits the root where it can
        r = np.hypot(DX, DY)
        ok = (r > np.abs(root)) & (r > 0)
        phi = np.arctan2(-DY, DX)
        ang = np.arcsin(np.clip(root / np.where(r > 0, r, 1.0), -1, 1)) - phi
        s2 = np.where(ok, np.sin(ang), s)
        c2 = np.where(ok, np.cos(ang), c)
        s2 = s2 * (1.0 + rng.integers(-4, 5, n) * 2.0 ** -52)
        s2 = np.where(np.abs(s2) < 2.0 ** -100, 0.0, s2)
        c2 = np.where(np.abs(c2) < 2.0 ** -100, 0.0, c2)
        e1, lo2, hi2 = _transport_operands(ax, ay, lx, ly, s2, c2, dx, sx, i, P)
        _check(e1, lo2, hi2)
        assert np.min(np.abs(e1[e1 != 0])) < 1e-10  # the construction does cancel
