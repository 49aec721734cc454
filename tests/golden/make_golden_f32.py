"""Golden fixtures of the reference's --float mode (run_curvelet<float>,
cpu_curvelet/main.cpp:110).

Runs in the development container only: it needs the reference sources (its
sample edge files and oracle/_ref, built by `make -C oracle`). The float
instantiation of the reference's templates is run in-process through
oracle/_ref/libcvlref.so, whose float path reproduces the reference program's
`--float` output files byte for byte. Writes tests/golden/reference_files_f32.npz:

  for each of the three sample files: the edges as the reference reads them in
  float mode (strtof per token), the counts, and the chains and info rows (full
  for the two small files, SHA-256 digests for TO_edges.txt); and for the KAT
  maps of make_golden.py: their edges in float32 and the reference's outputs.

    python tests/golden/make_golden_f32.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from make_golden import REF_DIR, REF_FILES, _need_reference, digest, kat_maps  # noqa: E402
from oracle import oracle as O  # noqa: E402


def main() -> None:
    _need_reference()
    O.build()
    if not O.ref_available():
        raise SystemExit("reference harness not built (needs the reference sources)")
    out = {}
    for f in REF_FILES:
        key = f.replace(".txt", "")
        e = O.parse_edges_f32(os.path.join(REF_DIR, f))
        r = O.ref_run(e, nthreads=8, scalar="float")
        out[f"{key}/edges"] = e
        out[f"{key}/counts"] = np.array([r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs,
                                         r.max_num_of_neighbors], dtype=np.int64)
        if e.shape[0] < 10000:
            out[f"{key}/chains"] = r.chains
            out[f"{key}/info"] = r.info
        out[f"{key}/digests"] = np.array([digest(r.chains), digest(r.info)])
        print(f, e.shape, r.num_curvelets, r.valid_pairs)
    for name, (e, params) in kat_maps().items():
        e32 = e.astype(np.float32)
        r = O.ref_run(e32, nthreads=1, scalar="float", **params)
        out[f"kat/{name}/edges"] = e32
        out[f"kat/{name}/params"] = np.array([params.get("group_max_sz", 4), params.get("max_candidates", 128)])
        out[f"kat/{name}/chains"] = r.chains
        out[f"kat/{name}/info"] = r.info
        out[f"kat/{name}/counts"] = np.array([r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs,
                                              r.max_num_of_neighbors], dtype=np.int64)
        print("kat", name, r.num_curvelets, r.valid_pairs)
    np.savez_compressed(os.path.join(HERE, "reference_files_f32.npz"), **out)


if __name__ == "__main__":
    main()
