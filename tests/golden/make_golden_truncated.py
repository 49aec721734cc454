"""Golden fixtures for maps whose anchors are truncated at max_candidates.

Where the cap cuts inside a pixel cell, the reference keeps the edges that its
unstable std::sort of the cell keys happens to put first (cpu_curvelet/preprocess.hpp:90-92,
:162-164), an order libstdc++ defines. The engine and the C restatement keep the
lowest edge indices instead. These fixtures give the reference's own answer for
that choice: the reference's CurveletCPU stage (form_pairwise_bundles,
build_curvelets_greedy, cpu_curvelet.hpp:305-634), compiled from its sources
into oracle/_ref/libcvlref.so, run on the lowest-index neighbour lists, in
double and in float (run_curvelet<float>, the --float mode).

The lowest-index lists come from the C restatement (oracle/cvl_oracle.c,
orc_build_csr) in double and from oracle.build_csr_f32 in float; both equal the
reference's own lists on every map without a truncated anchor
(tests/test_oracle_pinned.py).

Runs in the development container only (it needs oracle/_ref, built from the
reference sources by `make -C oracle`). Writes tests/golden/truncated_lowest.npz:

  <case>/<scalar>/edges        the map (float32 in float mode)
  <case>/<scalar>/params       group_max_sz, max_candidates
  <case>/<scalar>/csr_sha256   SHA-256 of the lowest-index offsets and ids (int32)
  <case>/<scalar>/counts       num_curvelets, valid_pairs, total pairs, max degree,
                               truncated anchors
  <case>/<scalar>/chains, info the reference stage's outputs (info row-major)
  pin_f32/<map>/csr_sha256     SHA-256 of the reference's own float CSR, with its
                               squared distances, for the maps without a truncated
                               anchor (the float KATs of make_golden_f32.py and two
                               sample files): the pin of oracle.build_csr_f32

    python tests/golden/make_golden_truncated.py
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_golden import kat_maps  # noqa: E402
from oracle import oracle as O  # noqa: E402


def blob600() -> np.ndarray:
    """600 edges in a 4 x 4 px square: every anchor has ~500 candidates."""
    rng = np.random.Generator(np.random.PCG64(3))
    return np.stack([50 + rng.uniform(-2, 2, 600), 50 + rng.uniform(-2, 2, 600), rng.uniform(-3, 3, 600),
                     rng.uniform(1, 5, 600)], 1)


def cases():
    e150, p150 = kat_maps()["blob150"]
    return {
        "blob150": (e150, dict(p150)),
        "blob600_mc128": (blob600(), dict(max_candidates=128)),
        "blob600_mc40": (blob600(), dict(max_candidates=40)),
    }


def csr_digest(offsets, ids, dist2=None) -> str:
    """SHA-256 of the offsets and ids (int32), and of the squared distances as
    float32 when given (float mode)."""
    h = hashlib.sha256()
    h.update(np.ascontiguousarray(offsets, dtype=np.int32).tobytes())
    h.update(np.ascontiguousarray(ids, dtype=np.int32).tobytes())
    if dist2 is not None:
        h.update(np.ascontiguousarray(dist2, dtype=np.float32).tobytes())
    return h.hexdigest()


def lowest_csr(e, scalar, max_candidates):
    if scalar == "float":
        return O.build_csr_f32(e, max_candidates=max_candidates)
    return O.build_csr(e, max_candidates=max_candidates)


def main() -> None:
    O.build()
    if not O.ref_available():
        raise SystemExit("reference harness not built (needs the reference sources)")
    out = {}
    for name, (e, params) in cases().items():
        gms = params.get("group_max_sz", 4)
        mc = params.get("max_candidates", 128)
        for scalar in ("double", "float"):
            ee = e.astype(np.float32) if scalar == "float" else np.ascontiguousarray(e, dtype=np.float64)
            c = lowest_csr(ee, scalar, mc)
            assert c.truncated_anchors > 0, name
            r = O.ref_run_csr(ee, c.offsets, c.ids, scalar=scalar, group_max_sz=gms, max_candidates=mc)
            k = f"{name}/{scalar}"
            out[f"{k}/edges"] = ee
            out[f"{k}/params"] = np.array([gms, mc], dtype=np.int64)
            out[f"{k}/csr_sha256"] = np.array(csr_digest(c.offsets, c.ids))
            out[f"{k}/counts"] = np.array([r.chains.shape[0], r.valid_pairs, r.total_neighbor_pairs,
                                           r.max_num_of_neighbors, c.truncated_anchors], dtype=np.int64)
            out[f"{k}/chains"] = r.chains
            out[f"{k}/info"] = r.info
            print(k, ee.shape, "curvelets", r.chains.shape[0], "valid pairs", r.valid_pairs,
                  "truncated", c.truncated_anchors)
    g32 = np.load(os.path.join(HERE, "reference_files_f32.npz"))
    pins = [k.split("/")[1] for k in g32.files if k.startswith("kat/") and k.endswith("/edges")]
    pins = [(f"kat/{n}", f"kat/{n}") for n in sorted(pins)] + \
        [(k, k) for k in ("TO_edges_digit1", "TO_edges_ABC_0006_thresh1")]
    for label, key in pins:
        e = g32[f"{key}/edges"]
        mc = int(g32[f"{key}/params"][1]) if f"{key}/params" in g32.files else 128
        r = O.ref_run(e, nthreads=8, scalar="float", max_candidates=mc)
        if int(np.diff(r.csr.offsets).max(initial=0)) >= mc:
            continue  # a truncated map: its CSR is libstdc++'s choice
        out[f"pin_f32/{label.replace('kat/', '')}/csr_sha256"] = np.array(
            csr_digest(r.csr.offsets, r.csr.ids, r.csr.dist2))
        print("pin", label, e.shape)
    np.savez_compressed(os.path.join(HERE, "truncated_lowest.npz"), **out)


if __name__ == "__main__":
    main()
