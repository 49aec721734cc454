"""Golden fixtures of the downstream stage (curvelets -> edgel link graph ->
contour fragments), made by the reference's own original_code implementation:
construct_the_link_graph and extract_regular_contours_from_the_link_graph
(original_code/form_curvelet_process.cpp:453-654), compiled from its sources by
`make -C oracle` into oracle/_ref/liborigref.so (oracle/orig_harness.cpp).

Runs in the development container only (it needs the reference sources). Writes
tests/golden/contours.npz:

  file/<name>/<mg>_<gap>/{links, frag_offsets, frag_ids}: the three sample edge
      files' curvelets (the reference's cpu_curvelet output) through the stage,
      full for the two small files, SHA-256 digests for TO_edges.txt;
  fuzz<seed>/{edges, chains} + fuzz<seed>/<mg>_<gap>/...: random curvelet sets
      (synth.contour_fuzz) with junctions, reversed links, gaps and cycles;
  rings<seed>/...: closed contours (synth.contour_rings);
  poly/<case>/{offsets, ids, info}: the C^1 polyarcs that original_code's
      fit_polyarcs_to_all_edgel_chains (form_curvelet_process.cpp:661-796) fits
      along those fragments (min_group_size 4, gap 1.5; fuzz cases also at 2, 3.5),
      read as its output type 2 (digests for TO_edges.txt).

    python tests/golden/make_golden_contours.py
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

from curvelet_construction_on_gpu_b200 import synth  # noqa: E402
from make_golden import REF_DIR, REF_FILES, _need_reference  # noqa: E402
from oracle import oracle as O  # noqa: E402

FILE_PARAMS = [(4, 1.5), (2, 1.5), (3, 2.0), (4, 1.0)]
FUZZ_PARAMS = [(4, 1.5), (2, 1.5), (3, 2.0), (2, 3.5)]


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def put(out: dict, key: str, c, full: bool) -> None:
    if full:
        out[f"{key}/links"] = c.links
        out[f"{key}/frag_offsets"] = c.frag_offsets
        out[f"{key}/frag_ids"] = c.frag_ids
    else:
        out[f"{key}/digests"] = np.array([digest(c.links), digest(c.frag_offsets), digest(c.frag_ids)])
        out[f"{key}/counts"] = np.array([c.links.shape[0], c.num_frags, c.frag_ids.shape[0]], np.int64)


def main() -> None:
    _need_reference()
    O.build()
    if not (O.ref_available() and O.orig_available()):
        raise SystemExit("reference harnesses not built (make -C oracle; needs the reference sources)")
    out = {}
    for f in REF_FILES:
        name = f.replace(".txt", "")
        e = O.read_edge_file(os.path.join(REF_DIR, f))
        r = O.ref_run(e, nthreads=8)
        fw = (r.info[:, 0] > 0).astype(np.uint8)
        for mg, gap in FILE_PARAMS:
            c = O.ref_link_contours(e, r.chains, fw, mg, gap)
            put(out, f"file/{name}/{mg}_{gap}", c, e.shape[0] < 10000)
            print(name, mg, gap, c.links.shape[0], c.num_frags)
    for seed in (0, 1):
        e, ch = synth.contour_fuzz(seed)
        out[f"fuzz{seed}/edges"], out[f"fuzz{seed}/chains"] = e, ch
        for mg, gap in FUZZ_PARAMS:
            c = O.ref_link_contours(e, ch, None, mg, gap)
            put(out, f"fuzz{seed}/{mg}_{gap}", c, True)
            print("fuzz", seed, mg, gap, c.links.shape[0], c.num_frags)
    for seed in (0, 1):
        e, ch = synth.contour_rings(seed)
        out[f"rings{seed}/edges"], out[f"rings{seed}/chains"] = e, ch
        c = O.ref_link_contours(e, ch, None, 4, 1.5)
        put(out, f"rings{seed}/4_1.5", c, True)
        print("rings", seed, c.num_frags)
    # polyarcs along the fragments
    for f in REF_FILES:
        name = f.replace(".txt", "")
        e = O.read_edge_file(os.path.join(REF_DIR, f))
        r = O.ref_run(e, nthreads=8)
        put_poly(out, f"poly/{name}", O.ref_polyarcs(e, r.chains), e.shape[0] < 10000)
    for seed in (0, 1):
        e, ch = out[f"fuzz{seed}/edges"], out[f"fuzz{seed}/chains"]
        put_poly(out, f"poly/fuzz{seed}", O.ref_polyarcs(e, ch), True)
        put_poly(out, f"poly/fuzz{seed}_2_3.5", O.ref_polyarcs(e, ch, 2, 3.5), True)
        e, ch = out[f"rings{seed}/edges"], out[f"rings{seed}/chains"]
        put_poly(out, f"poly/rings{seed}", O.ref_polyarcs(e, ch), True)
    np.savez_compressed(os.path.join(HERE, "contours.npz"), **out)


def put_poly(out: dict, key: str, p, full: bool) -> None:
    if full:
        out[f"{key}/offsets"], out[f"{key}/ids"], out[f"{key}/info"] = p.offsets, p.ids, p.info
    else:
        out[f"{key}/digests"] = np.array([digest(p.offsets), digest(p.ids)])
        out[f"{key}/info"] = p.info  # 1,466 rows for TO_edges: small enough to keep in full
    print(key, p.num)


if __name__ == "__main__":
    main()
