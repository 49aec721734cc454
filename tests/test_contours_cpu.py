"""The downstream stage's checker, pinned on the CPU: the C restatement
(oracle/cvl_oracle.c: orc_link_contours) reproduces the reference's own
original_code link graph and one-chain extraction (tests/golden/contours.npz,
made by tests/golden/make_golden_contours.py from original_code compiled as is)
bit for bit: the links with their votes in _cLinks order, and the fragments."""
import hashlib
import os

import numpy as np
import pytest

from curvelet_construction_on_gpu_b200 import synth
from curvelet_construction_on_gpu_b200.api import Contours

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gc():
    return np.load(os.path.join(GOLDEN, "contours.npz"))


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def assert_same_contours(c, gc, key):
    if f"{key}/links" in gc.files:
        assert np.array_equal(c.links, gc[f"{key}/links"]), key
        assert np.array_equal(c.frag_offsets, gc[f"{key}/frag_offsets"]), key
        assert np.array_equal(c.frag_ids, gc[f"{key}/frag_ids"]), key
    else:
        assert [c.links.shape[0], c.num_frags, c.frag_ids.shape[0]] == gc[f"{key}/counts"].tolist(), key
        assert [_digest(c.links), _digest(c.frag_offsets), _digest(c.frag_ids)] == gc[f"{key}/digests"].tolist(), key


def _params(gc, prefix):
    return sorted({k[len(prefix) + 1:].split("/")[0] for k in gc.files
                   if k.startswith(prefix + "/") and "_" in k[len(prefix) + 1:].split("/")[0]})


@pytest.mark.parametrize("name", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1"])
def test_restatement_on_reference_curvelets(oracle, gc, golden_files, name):
    e, ch = golden_files[f"{name}/edges"], golden_files[f"{name}/chains"]
    for p in _params(gc, f"file/{name}"):
        mg, gap = p.split("_")
        assert_same_contours(oracle.link_contours(e, ch, int(mg), float(gap)), gc, f"file/{name}/{p}")


def test_restatement_on_to_edges(oracle, gc, golden_files):
    e = golden_files["TO_edges/edges"]
    r = oracle.run(e, nthreads=8)  # equals the reference's curvelets (test_oracle_pinned)
    for p in _params(gc, "file/TO_edges"):
        mg, gap = p.split("_")
        assert_same_contours(oracle.link_contours(e, r.chains, int(mg), float(gap)), gc, f"file/TO_edges/{p}")


@pytest.mark.parametrize("case", ["fuzz0", "fuzz1", "rings0", "rings1"])
def test_restatement_on_fuzz_and_rings(oracle, gc, case):
    e, ch = gc[f"{case}/edges"], gc[f"{case}/chains"]
    for p in _params(gc, case):
        mg, gap = p.split("_")
        assert_same_contours(oracle.link_contours(e, ch, int(mg), float(gap)), gc, f"{case}/{p}")


def test_generators_reproduce_fixture_inputs(gc):
    for seed in (0, 1):
        e, ch = synth.contour_fuzz(seed)
        assert np.array_equal(e, gc[f"fuzz{seed}/edges"]) and np.array_equal(ch, gc[f"fuzz{seed}/chains"])
        e, ch = synth.contour_rings(seed)
        assert np.array_equal(e, gc[f"rings{seed}/edges"]) and np.array_equal(ch, gc[f"rings{seed}/chains"])


def test_restatement_matches_live_original_code(oracle):
    if not oracle.orig_available():
        pytest.skip("original_code harness not built here")
    for seed in (5, 6):
        e, ch = synth.contour_fuzz(seed, n_edges=1500, width=8)
        for mg, gap in ((2, 1.5), (5, 2.0), (0, 0.0)):
            a = oracle.link_contours(e, ch, mg, gap)
            b = oracle.ref_link_contours(e, ch, None, mg, gap)
            assert np.array_equal(a.links, b.links) and np.array_equal(a.frag_ids, b.frag_ids)
            assert np.array_equal(a.frag_offsets, b.frag_offsets)


def test_rings_close_on_themselves(gc):
    # a closed ring gives one fragment that starts and ends on its start edge
    offs, ids = gc["rings0/4_1.5/frag_offsets"], gc["rings0/4_1.5/frag_ids"]
    frags = [ids[offs[i]:offs[i + 1]] for i in range(len(offs) - 1)]
    assert any(f[0] == f[-1] and len(set(f.tolist())) == len(f) - 1 for f in frags)


def test_fragment_array_layout():
    c = Contours(np.zeros((0, 3), np.int32), np.array([0, 3, 7]), np.array([4, 5, 6, 0, 1, 2, 3], np.int32), 8)
    a = c.as_array()
    assert a.tolist() == [[5, 6, 7, 0], [1, 2, 3, 4]]
    assert [f.tolist() for f in c.fragments()] == [[4, 5, 6], [0, 1, 2, 3]]


# ---- polyarcs along the fragments (fit_polyarcs_to_all_edgel_chains) ----------
def assert_same_polyarcs(p_offsets, p_ids, p_info, gc, key):
    if f"{key}/offsets" in gc.files:
        assert np.array_equal(p_offsets, gc[f"{key}/offsets"]), key
        assert np.array_equal(p_ids, gc[f"{key}/ids"]), key
    else:
        assert [_digest(p_offsets), _digest(p_ids)] == gc[f"{key}/digests"].tolist(), key
    return gc[f"{key}/info"]


def _poly_cases():
    return [("TO_edges_digit1", None), ("TO_edges_ABC_0006_thresh1", None), ("TO_edges", None),
            ("fuzz0", (4, 1.5)), ("fuzz0_2_3.5", (2, 3.5)), ("fuzz1", (4, 1.5)), ("fuzz1_2_3.5", (2, 3.5)),
            ("rings0", (4, 1.5)), ("rings1", (4, 1.5))]


@pytest.mark.parametrize("case,params", _poly_cases())
def test_polyarc_restatement_matches_reference(oracle, gc, golden_files, case, params):
    """orc_polyarcs_fit equals original_code's fit bit for bit: chains and all 12 columns."""
    if params is None:
        e = golden_files[f"{case}/edges"]
        ch = golden_files[f"{case}/chains"] if f"{case}/chains" in golden_files.files else oracle.run(e, nthreads=8).chains
        mg, gap = 4, 1.5
    else:
        base = case.split("_")[0]
        e, ch = gc[f"{base}/edges"], gc[f"{base}/chains"]
        mg, gap = params
    c = oracle.link_contours(e, ch, mg, gap)
    p = oracle.polyarcs(e, c.frag_offsets, c.frag_ids)
    info = assert_same_polyarcs(p.offsets, p.ids, p.info, gc, f"poly/{case}")
    assert np.array_equal(p.info.view(np.uint64), info.view(np.uint64)), case


def test_polyarc_restatement_matches_live_original_code(oracle):
    if not oracle.orig_available():
        pytest.skip("original_code harness not built here")
    e, ch = synth.contour_fuzz(8, n_edges=2000, width=6)
    for mg, gap in ((2, 2.0), (3, 3.0)):
        c = oracle.link_contours(e, ch, mg, gap)
        a = oracle.polyarcs(e, c.frag_offsets, c.frag_ids, dx=0.5, max_k=0.4)
        b = oracle.ref_polyarcs(e, ch, mg, gap, dx=0.5, max_k=0.4)
        assert np.array_equal(a.ids, b.ids) and np.array_equal(a.offsets, b.offsets)
        assert np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))
