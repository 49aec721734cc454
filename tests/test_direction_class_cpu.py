"""The direction class of a pair without the transcendental calls.

The reference classes a neighbour by the sign of
dot(To2Pi(atan2(ly - ay, lx - ax)), theta) (cpu_curvelet.hpp:459-461,
curvelet_utils.hpp:25-69), through glibc. The engine's neighbour kernel
(direction_class in csrc/cvl_kernels.cuh) takes the sign of
v = dx cos(theta) + dy sin(theta) instead whenever |v| exceeds 1e-12 (float mode:
1e-4) of |dx| + |dy|, and evaluates the reference's expression otherwise. The
engine's cos(theta) and sin(theta) are CUDA's, a few ulps from glibc's.

These tests check the margin argument against the reference's own expression:
glibc through Python's math module (double) and through ctypes (the float
functions), on random pairs and on pairs a hair away from perpendicular, with
cos(theta) and sin(theta) moved by up to 4 ulps the way another libm's could be."""
import ctypes
import math

import numpy as np

TWO_PI = 2.0 * math.pi


def _to2pi(a: float) -> float:
    # curvelet_utils.hpp:25-45, T = double
    if a >= TWO_PI:
        r = math.fmod(a, TWO_PI)
    elif a < 0:
        r = TWO_PI + math.fmod(a, TWO_PI)
    else:
        r = a
    if not (r >= 0 and r < TWO_PI):
        r = 0.0
    return r


def _ref_dot(ax, ay, lx, ly, th) -> float:
    d = _to2pi(math.atan2(ly - ay, lx - ax))
    return math.cos(d) * math.cos(th) + math.sin(d) * math.sin(th)


def _ulps(x: np.ndarray, k: np.ndarray) -> np.ndarray:
    out = x.copy()
    for step in range(int(np.max(np.abs(k))) if len(k) else 0):
        up = k > step
        dn = -k > step
        out[up] = np.nextafter(out[up], np.inf)
        out[dn] = np.nextafter(out[dn], -np.inf)
    return out


def _cases(rng, n, near):
    ax = rng.uniform(0, 2000, n)
    ay = rng.uniform(0, 2000, n)
    r = rng.uniform(0.05, 3.5, n)
    phi = rng.uniform(-math.pi, math.pi, n)
    lx = ax + r * np.cos(phi)
    ly = ay + r * np.sin(phi)
    if near:
        # theta a hair away from perpendicular to the pair's direction
        delta = np.exp(rng.uniform(math.log(1e-17), math.log(1e-6), n)) * rng.choice([-1.0, 1.0], n)
        th = np.arctan2(ly - ay, lx - ax) + rng.choice([-0.5, 0.5], n) * math.pi + delta
        th = np.where(th < -math.pi, th + TWO_PI, th)
        th = np.where(th > 3 * math.pi, th - TWO_PI, th)
    else:
        th = rng.uniform(-math.pi, 2 * math.pi, n)
    return ax, ay, lx, ly, th


def test_double_margin_gives_the_reference_sign():
    rng = np.random.default_rng(11)
    decided = agree = 0
    for near in (False, True):
        ax, ay, lx, ly, th = _cases(rng, 60_000, near)
        dx, dy = lx - ax, ly - ay
        for k in (0, 4):
            c = _ulps(np.cos(th), rng.integers(-k, k + 1, len(th)))
            s = _ulps(np.sin(th), rng.integers(-k, k + 1, len(th)))
            v = dx * c + dy * s
            margin = 1e-12 * (np.abs(dx) + np.abs(dy))
            for i in np.nonzero(np.abs(v) > margin)[0]:
                d = _ref_dot(ax[i], ay[i], lx[i], ly[i], th[i])
                decided += 1
                agree += (d > 0) == (v[i] > 0) and d != 0
    assert decided > 100_000
    assert agree == decided


def test_double_margin_is_needed_near_perpendicular():
    """Without the margin, the sign of v and the reference's sign do disagree a
    hair from perpendicular: the fallback to the reference's expression matters."""
    rng = np.random.default_rng(12)
    ax, ay, lx, ly, th = _cases(rng, 40_000, True)
    v = (lx - ax) * np.cos(th) + (ly - ay) * np.sin(th)
    diff = sum(1 for i in range(len(th)) if (_ref_dot(ax[i], ay[i], lx[i], ly[i], th[i]) > 0) != (v[i] > 0))
    assert diff > 0


def test_float_margin_gives_the_reference_sign():
    """Float mode: the reference's run_curvelet<float> evaluates atan2f, To2Pi,
    cosf and sinf in float; the engine computes v in double from the float edges
    and its float cos/sin of theta, with a margin of 1e-4 of |dx| + |dy|."""
    m = ctypes.CDLL("libm.so.6")
    for f in ("atan2f", "cosf", "sinf", "fmodf"):
        getattr(m, f).restype = ctypes.c_float
    m.atan2f.argtypes = m.fmodf.argtypes = [ctypes.c_float, ctypes.c_float]
    m.cosf.argtypes = m.sinf.argtypes = [ctypes.c_float]
    f32 = np.float32
    two_pi = f32(2) * f32(math.pi)

    def to2pi(a):
        if a >= two_pi:
            r = f32(m.fmodf(a, two_pi))
        elif a < 0:
            r = f32(two_pi + f32(m.fmodf(a, two_pi)))
        else:
            r = a
        if not (r >= 0 and r < two_pi):
            r = f32(0)
        return r

    rng = np.random.default_rng(13)
    decided = agree = 0
    for near in (False, True):
        ax, ay, lx, ly, th = (a.astype(np.float32) for a in _cases(rng, 15_000, near))
        for i in range(len(th)):
            d = to2pi(f32(m.atan2f(f32(ly[i] - ay[i]), f32(lx[i] - ax[i]))))
            cd, sd = f32(m.cosf(d)), f32(m.sinf(d))
            ct, st = f32(m.cosf(th[i])), f32(m.sinf(th[i]))
            ref = f32(f32(cd * ct) + f32(sd * st))
            for k in (0, 4):
                c = float(_ulps(np.array([ct]), np.array([rng.integers(-k, k + 1)]))[0])
                s = float(_ulps(np.array([st]), np.array([rng.integers(-k, k + 1)]))[0])
                dx, dy = float(lx[i]) - float(ax[i]), float(ly[i]) - float(ay[i])
                v = dx * c + dy * s
                if abs(v) > 1e-4 * (abs(dx) + abs(dy)):
                    decided += 1
                    agree += (ref > 0) == (v > 0) and ref != 0
    assert decided > 20_000
    assert agree == decided
