"""Generates the committed golden fixtures from the reference's own code.

Runs in the development container only (it needs the reference sources and
oracle/_ref/libcvlref.so, built by `make -C oracle`). Writes:

  tests/golden/reference_files.npz   the reference's three loadable sample edge
      files as arrays, and for each: counts, the neighbour CSR, and the chains
      and info rows (full for the two small files; SHA-256 digests for
      TO_edges.txt, whose outputs are 6.8 MB)
  tests/golden/kat_maps.npz          small hand-made maps (collinear edges, a
      radius-20 arc, a close pair, a near-perpendicular neighbour, a 150-edge
      blob that hits max_candidates, equal-distance neighbours, group_max_sz 7)
      with the reference's full outputs
  tests/golden/pair_bundles.npz      64 (anchor, neighbour) pairs with the
      reference's 63-cell bundles (compute_curve_bundle)

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402

REF_FILES = ["TO_edges_digit1.txt", "TO_edges_ABC_0006_thresh1.txt", "TO_edges.txt"]
# the reference project's sample inputs: $CVL_REFERENCE_DIR/test_files
REF_DIR = os.path.join(os.environ.get("CVL_REFERENCE_DIR", ""), "test_files")


def _need_reference() -> None:
    if not os.path.isdir(REF_DIR) or not os.environ.get("CVL_REFERENCE_DIR"):
        raise SystemExit("set CVL_REFERENCE_DIR to the reference project's root (it holds test_files/)")


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def kat_maps() -> dict[str, tuple[np.ndarray, dict]]:
    rng = np.random.Generator(np.random.PCG64(7))
    maps = {}
    # five collinear edges along y = 10, orientation 0
    e = np.array([[10.0 + k, 10.0, 0.0, 5.0] for k in range(5)])
    maps["collinear5"] = (e, {})
    # a radius-20 arc sampled every 1 px, tangent orientation
    s = np.arange(40.0)
    phi = s / 20.0
    e = np.stack([50 + 20 * np.cos(phi), 50 + 20 * np.sin(phi), phi + math.pi / 2, np.full_like(s, 9.0)], 1)
    maps["arc_r20"] = (e, {})
    # close pairs (distance < 2*dx = 0.8) inside a short line
    e = np.array([[10.0, 10.0, 0.1, 5.0], [10.5, 10.02, 0.1, 5.0], [11.0, 10.1, 0.1, 5.0], [12.0, 10.2, 0.1, 5.0],
                  [12.3, 10.25, 0.1, 5.0], [13.0, 10.3, 0.1, 5.0]])
    maps["close_pairs"] = (e, {})
    # neighbours almost perpendicular to the anchor orientation
    e = np.array([[20.0, 20.0, 0.0, 5.0], [20.0, 22.0, 0.0, 5.0], [20.0, 18.0, 0.0, 5.0], [21.0, 20.0, 0.0, 5.0],
                  [19.0, 20.0, 0.0, 5.0], [20.0 + 1e-12, 21.0, 0.0, 5.0]])
    maps["perpendicular"] = (e, {})
    # a dense blob: 150 edges within a 3 x 3 px square -> anchors reach max_candidates
    e = np.stack([30 + rng.uniform(-1.4, 1.4, 150), 30 + rng.uniform(-1.4, 1.4, 150),
                  rng.uniform(-math.pi, math.pi, 150), rng.uniform(1, 5, 150)], 1)
    maps["blob150"] = (e, {})
    # equal squared distances (ties) across cells, fewer than 16 candidates
    e = np.array([[40.0, 40.0, 0.0, 5.0], [42.0, 40.0, 0.0, 5.0], [38.0, 40.0, 0.0, 5.0], [40.0, 42.0, 0.3, 5.0],
                  [40.0, 38.0, -0.3, 5.0], [41.0, 41.0, 0.2, 5.0], [39.0, 39.0, 0.2, 5.0], [43.0, 40.0, 0.0, 5.0]])
    maps["ties"] = (e, {})
    # a noisy segment run with group_max_sz = 7 and a smaller max_candidates
    t = np.arange(30.0)
    e = np.stack([5 + t * 0.9, 5 + t * 0.3 + rng.normal(0, 0.1, 30), np.full(30, math.atan2(0.3, 0.9)) +
                  rng.normal(0, 0.03, 30), np.full(30, 4.0)], 1)
    maps["segment_gms7"] = (e, {"group_max_sz": 7, "max_candidates": 9})
    # edges with 6 values per row (extra columns ignored) and negative coordinates
    e6 = np.concatenate([np.stack([-5 + t * 0.8, -3 + t * 0.1, np.full(30, 0.12), np.full(30, 4.0)], 1),
                         rng.uniform(0, 1, (30, 2))], 1)
    maps["negative_sz6"] = (e6, {})
    return maps


def main() -> None:
    _need_reference()
    O.build()
    if not O.ref_available():
        raise SystemExit("reference harness not built (needs the reference sources)")
    out = {}
    for f in REF_FILES:
        key = f.replace(".txt", "")
        e = O.read_edge_file(os.path.join(REF_DIR, f))
        r = O.ref_run(e, nthreads=8)
        out[f"{key}/edges"] = e
        out[f"{key}/counts"] = np.array([r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs,
                                         r.max_num_of_neighbors], dtype=np.int64)
        if e.shape[0] < 10000:
            out[f"{key}/chains"] = r.chains
            out[f"{key}/info"] = r.info
            out[f"{key}/csr_offsets"] = r.csr.offsets
            out[f"{key}/csr_ids"] = r.csr.ids
            out[f"{key}/csr_dist2"] = r.csr.dist2
        out[f"{key}/digests"] = np.array([digest(r.chains), digest(r.info), digest(r.csr.offsets),
                                          digest(r.csr.ids), digest(r.csr.dist2)])
        print(f, e.shape, r.num_curvelets, r.valid_pairs)
    np.savez_compressed(os.path.join(HERE, "reference_files.npz"), **out)

    kat = {}
    for name, (e, params) in kat_maps().items():
        r = O.ref_run(e, nthreads=1, **params)
        kat[f"{name}/edges"] = e
        kat[f"{name}/params"] = np.array([params.get("group_max_sz", 4), params.get("max_candidates", 128)])
        kat[f"{name}/chains"] = r.chains
        kat[f"{name}/info"] = r.info
        kat[f"{name}/csr_offsets"] = r.csr.offsets
        kat[f"{name}/csr_ids"] = r.csr.ids
        kat[f"{name}/csr_dist2"] = r.csr.dist2
        kat[f"{name}/counts"] = np.array([r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs,
                                          r.max_num_of_neighbors], dtype=np.int64)
        print(name, e.shape, r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors)
    np.savez_compressed(os.path.join(HERE, "kat_maps.npz"), **kat)

    # pair bundles: random geometry around the radius, plus a close pair and both branches
    rng = np.random.Generator(np.random.PCG64(11))
    pairs = []
    for _ in range(60):
        r = rng.uniform(0.3, 3.5)
        a = rng.uniform(-math.pi, math.pi)
        te = (rng.uniform(0, 100), rng.uniform(0, 100), rng.uniform(-math.pi, math.pi))
        le = (te[0] + r * math.cos(a), te[1] + r * math.sin(a), te[2] + rng.normal(0, 0.3))
        pairs.append(te + le)
    pairs.append((10.0, 10.0, 0.0, 10.5, 10.0, 0.0))   # close pair
    pairs.append((10.0, 10.0, 0.0, 12.0, 10.0, 0.0))   # neighbour ahead (DX < 0: branch 1)
    pairs.append((10.0, 10.0, 0.0, 8.0, 10.0, 0.0))    # neighbour behind (branch 2)
    pairs.append((10.0, 10.0, 0.5, 11.0, 12.0, 2.0))   # strongly curved
    pairs = np.asarray(pairs, dtype=np.float64)
    bmin, bmax, valid = [], [], []
    for q in pairs:
        v, mn, mx = O.pair_bundle(q[:3], q[3:], use_ref=True)
        valid.append(v)
        bmin.append(mn)
        bmax.append(mx)
    np.savez_compressed(os.path.join(HERE, "pair_bundles.npz"), pairs=pairs, bmin=np.asarray(bmin),
                        bmax=np.asarray(bmax), valid=np.asarray(valid))
    print("pairs", pairs.shape, int(np.sum(valid)))


if __name__ == "__main__":
    main()
