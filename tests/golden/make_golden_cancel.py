"""Generates tests/golden/pair_bundles_cancel.npz: (anchor, neighbour) pairs at
which the bundle transport's denominator cancels to exactly +0 in the second
transport branch, with the reference's own compute_curve_bundle outputs.

Why these pairs: the path's bundle kernel computes branch 2's k_dx through branch
1's denominator e1 = (((DX2 - (2 dx2) tt) + DY2) - dx^2) + dx2^2, which equals
branch 2's eq_denom times 2 everywhere except where e1 is +0; there branch 2's
eq_denom is -0 (cpu_curvelet.hpp:774) and its k_dx are infinities of the other
sign. These pairs reach that value on the device:
  - the anchor's orientation is 0, so the centre orientation sample has
    T2t = 0 + 0 and sin(T2t) = 0, cos(T2t) = 1 exactly (in glibc and on the GPU),
    and tt = 0 * DX - 1 * DY = -DY (cpu_curvelet.hpp:702-705);
  - the grid step sx = 0.5 gives P = 3 and dx2 = -0.5, 0, 0.5
    (cpu_curvelet.hpp:73, :697), so e1 can vanish for a pair that is not close
    (DX^2 + DY^2 >= 4 dx^2): DX^2 + (DY + dx2)^2 = dx^2 on a circle;
  - DX > 0 puts the pair in branch 2 (DX cos 0 + DY sin 0 >= 0, :690);
  - the anchor is at (1 + DX, 1 + DY) and the neighbour at (1, 1), with DX and
    DY multiples of 2^-52, so te - le gives DX and DY exactly.
Each pair's centre-column cell (i, (Q-1)/2) with e1 == +0 is the cell this file
is about; its index is stored.

Runs in the development container only (needs oracle/_ref/libcvlref.so, built
from the reference sources by `make -C oracle REF_DIR=<cpu_curvelet dir>`):

    python tests/golden/make_golden_cancel.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

PARAMS = dict(sx=0.5)  # dx 0.4, dt 15 deg, st 0.08, max_k 0.3: the other defaults
N_PAIRS = 256


def cancelling_pairs(rng: np.random.Generator, n: int):
    dx, u = 0.4, 2.0 ** -52
    P = int(2 * np.floor(dx / PARAMS["sx"] + 0.5) + 1)
    d2 = [PARAMS["sx"] * (float(i) - (float(P) - 1.0) / 2.0) for i in range(P)]
    out = []
    for i in (0, P - 1):
        d = d2[i]
        DY = np.round(rng.uniform(0.74, 0.89, 8000) / u) * u * (1.0 if d < 0 else -1.0)
        DX0 = np.sqrt(np.maximum(dx * dx - (DY + d) ** 2, 0.0))
        for k in range(-64, 65):
            DX = np.round(DX0 / u) * u + k * u
            tt = 0.0 * DX - 1.0 * DY
            e1 = (((DX * DX - (2.0 * d) * tt) + DY * DY) - dx * dx) + d * d
            ok = (e1 == 0.0) & (DX > 0) & ~(DX * DX + DY * DY < 4 * dx * dx)
            ok &= ((1.0 + DX) - 1.0 == DX) & ((1.0 + DY) - 1.0 == DY)
            out += [(i, a, b) for a, b in zip(DX[ok], DY[ok])]
    pick = rng.choice(len(out), size=n, replace=False)
    rows, cell_i = [], []
    for k in pick:
        i, a, b = out[k]
        T0 = rng.uniform(-np.pi, np.pi)
        rows.append((1.0 + a, 1.0 + b, 0.0, 1.0, 1.0, T0))
        cell_i.append(i)
    return np.asarray(rows), np.asarray(cell_i, dtype=np.int32)


def main() -> None:
    O.build()
    if not O.ref_available():
        raise SystemExit("reference harness not built (needs the reference sources)")
    rng = np.random.Generator(np.random.PCG64(2024))
    pairs, cell_i = cancelling_pairs(rng, N_PAIRS)
    bmin, bmax, valid = [], [], []
    for q in pairs:
        v, mn, mx = O.pair_bundle(q[:3], q[3:], use_ref=True, **PARAMS)
        valid.append(v)
        bmin.append(mn)
        bmax.append(mx)
    bmin, bmax = np.asarray(bmin), np.asarray(bmax)
    Q = 7
    cell = cell_i * Q + (Q - 1) // 2
    closed = bmax[np.arange(N_PAIRS), cell] <= bmin[np.arange(N_PAIRS), cell]
    np.savez_compressed(os.path.join(HERE, "pair_bundles_cancel.npz"), pairs=pairs, bmin=bmin, bmax=bmax,
                        valid=np.asarray(valid), cell=cell.astype(np.int32),
                        params=np.array([PARAMS["sx"]]))
    print("pairs", pairs.shape, "valid", int(np.sum(valid)), "cancel cells closed", int(closed.sum()))


if __name__ == "__main__":
    main()
