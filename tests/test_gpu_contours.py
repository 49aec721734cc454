"""The downstream stage on the GPU (cvl_link_contours / cvl_run_contours): the
edgel link graph (links, votes, _cLinks order) and the contour fragments equal
the reference's original_code output (tests/golden/contours.npz) and the pinned
C restatement, bit for bit: on the sample files' curvelets, on fuzzed curvelet
sets with junctions, reversed links, gaps and cycles, on rings, and at full
size on the 1920x1080 map through the fused edges -> contours pass."""
import os

import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import synth
from tests.test_contours_cpu import _params, assert_same_contours

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def gc():
    return np.load(os.path.join(GOLDEN, "contours.npz"))


def _cp(p):
    mg, gap = p.split("_")
    return cvl.ContourParams(int(mg), float(gap))


def _same(a, b):
    return (np.array_equal(a.links, b.links) and np.array_equal(a.frag_offsets, b.frag_offsets)
            and np.array_equal(a.frag_ids, b.frag_ids))


@pytest.mark.parametrize("name", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1"])
def test_reference_curvelets(engine, gc, golden_files, name):
    e, ch = golden_files[f"{name}/edges"], golden_files[f"{name}/chains"]
    for p in _params(gc, f"file/{name}"):
        assert_same_contours(engine.link_contours(e, ch, _cp(p)), gc, f"file/{name}/{p}")


def test_to_edges_fused_and_staged(engine, gc, golden_files):
    e = golden_files["TO_edges/edges"]
    for p in _params(gc, "file/TO_edges"):
        res, c = engine.run_contours(e, contour_params=_cp(p))
        assert res.num_curvelets == 67735
        assert_same_contours(c, gc, f"file/TO_edges/{p}")
        assert_same_contours(engine.link_contours(e, res.chains, _cp(p)), gc, f"file/TO_edges/{p}")


@pytest.mark.parametrize("case", ["fuzz0", "fuzz1", "rings0", "rings1"])
def test_fuzz_and_rings(engine, gc, case):
    e, ch = gc[f"{case}/edges"], gc[f"{case}/chains"]
    for p in _params(gc, case):
        c = engine.link_contours(e, ch, _cp(p))
        assert_same_contours(c, gc, f"{case}/{p}")
    print(f"[contours] {case}: {c.links.shape[0]} links, {c.num_frags} fragments, {c.device_ms:.3f} ms")


@pytest.mark.parametrize("seed", [11, 12, 13])
def test_fuzz_vs_restatement(engine, oracle, seed):
    e, ch = synth.contour_fuzz(seed, n_edges=4000, width=int(4 + seed % 3 * 2), max_per_anchor=6)
    for mg, gap in ((2, 1.5), (4, 2.5), (0, 1.0), (3, 0.0)):
        a = engine.link_contours(e, ch, cvl.ContourParams(mg, gap))
        b = oracle.link_contours(e, ch, mg, gap)
        assert _same(a, b), (seed, mg, gap)


def test_plain_hd_full_size(engine, oracle):
    """The 1920x1080 map (about 250k edges, 500k curvelets): fused on the device."""
    e = synth.plain_hd(1000)
    for cp in (cvl.ContourParams(), cvl.ContourParams(2, 1.5)):
        res, c = engine.run_contours(e, contour_params=cp)
        b = oracle.link_contours(e, res.chains, cp.min_group_size, cp.gap)
        assert _same(c, b)
        print(f"[contours plain_hd] mg={cp.min_group_size}: {c.links.shape[0]} links, {c.num_frags} fragments, "
              f"longest {int(np.diff(c.frag_offsets).max())}, whole path {c.device_ms:.2f} ms")
    # gap comes from CurveletParams.gap when no contour parameters are given
    _, c1 = engine.run_contours(e, cvl.CurveletParams(gap=2.0), want_curvelets=False)
    _, c2 = engine.run_contours(e, contour_params=cvl.ContourParams(4, 2.0), want_curvelets=False)
    assert _same(c1, c2)


def test_dense_map_vs_restatement(engine, oracle):
    e = synth.dense_4k(4000)[:400000]
    res, c = engine.run_contours(e, contour_params=cvl.ContourParams(2, 1.5))
    assert _same(c, oracle.link_contours(e, res.chains, 2, 1.5))


def test_edge_cases(engine):
    e, ch = synth.contour_fuzz(3, n_edges=500)
    c = engine.link_contours(e, ch[:0])  # no curvelets
    assert c.links.shape == (0, 3) and c.num_frags == 0
    c = engine.link_contours(e, ch, cvl.ContourParams(2, 0.0))  # nothing is close enough
    assert c.num_frags == 0 and c.links.shape[0] > 0
    c = engine.link_contours(e, ch, cvl.ContourParams(99, 1.5))  # no curvelet is long enough
    assert c.links.shape[0] == 0 and c.num_frags == 0
    bad = ch.copy()
    bad[5, 2] = 501  # an id past the map
    with pytest.raises(cvl.CvlError):
        engine.link_contours(e, bad)
    with pytest.raises(cvl.CvlError):
        engine.link_contours(e, ch[::-1])  # anchors out of order
    with pytest.raises(cvl.CvlError):
        engine.link_contours(e, np.zeros((3, 65), np.uint32) + 1)
    with pytest.raises(cvl.CvlError):
        engine.link_contours(e, ch, cvl.ContourParams(4, -1.0))
    # the engine stays usable after the errors
    assert engine.link_contours(e, ch).links.shape[0] > 0


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1"])
def test_cli_fragments_file(tmp_path, gc, golden_files, key):
    """CURVELET --fragments writes the fragment map (output type 1 layout) next to
    the usual outputs, which stay byte-identical to the reference program's."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cli_bin = os.path.join(root, "curvelet_construction_on_gpu_b200", "bin", "CURVELET")
    for d in ("bin", "test_files", "outputs"):
        (tmp_path / d).mkdir(exist_ok=True)
    synth.write_edge_file(str(tmp_path / "test_files" / f"{key}.txt"), golden_files[f"{key}/edges"])
    r = subprocess.run([cli_bin, "--double", "--edge-file", f"{key}.txt", "--output", f"chain_{key}.txt",
                        "--fragments", f"frag_{key}.txt", "--link-min-group", "3", "--gap", "2.0"],
                       cwd=tmp_path / "bin", capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    cli = np.load(os.path.join(GOLDEN, "cli_outputs.npz"))
    assert (tmp_path / "outputs" / f"chain_{key}.txt").read_bytes() == cli[f"{key}/chain"].tobytes()
    assert (tmp_path / "outputs" / f"info_{key}.txt").read_bytes() == cli[f"{key}/info"].tobytes()
    want = cvl.Contours(gc[f"file/{key}/3_2.0/links"], gc[f"file/{key}/3_2.0/frag_offsets"],
                        gc[f"file/{key}/3_2.0/frag_ids"], 0).as_array()
    got = (tmp_path / "outputs" / f"frag_{key}.txt").read_text()
    assert got == "".join("".join(f"{v}\t" for v in row) + "\n" for row in want.tolist())


# ---- C^1 polyarcs along the fragments --------------------------------------------
POLY_EXACT = [0, 3, 4, 5, 7, 9, 10, 11]  # no transcendental input: bit-identical
POLY_TOL = [1, 2, 6, 8]                   # the bundle's k range (sin), theta and arc length (atan2)


def assert_polyarc_info(a, b, max_k=0.3, label=""):
    assert a.shape == b.shape, label
    assert np.array_equal(a[:, POLY_EXACT].view(np.uint64), b[:, POLY_EXACT].view(np.uint64)), label
    d = np.abs(a[:, POLY_TOL] - b[:, POLY_TOL])
    mag = np.maximum(np.abs(a[:, POLY_TOL]), np.abs(b[:, POLY_TOL]))
    floor = 1e-9 * np.array([max_k, max_k, 1.0, 1.0])
    assert np.all(d <= np.maximum(1e-9 * mag, floor)), (label, d.max(0))
    return float(np.mean(a.view(np.uint64) == b.view(np.uint64)))


@pytest.mark.parametrize("case,mg,gap", [("TO_edges_digit1", 4, 1.5), ("TO_edges_ABC_0006_thresh1", 4, 1.5),
                                         ("TO_edges", 4, 1.5), ("fuzz0", 4, 1.5), ("fuzz0_2_3.5", 2, 3.5),
                                         ("fuzz1_2_3.5", 2, 3.5), ("rings0", 4, 1.5), ("rings1", 4, 1.5)])
def test_polyarcs_vs_reference(engine, gc, golden_files, case, mg, gap):
    from tests.test_contours_cpu import assert_same_polyarcs
    cp = cvl.ContourParams(mg, gap, fit_polyarcs=True)
    if case.startswith("TO_edges"):
        e = golden_files[f"{case}/edges"]
        res, c = engine.run_contours(e, contour_params=cp)
    else:
        base = case.split("_")[0]
        e, ch = gc[f"{base}/edges"], gc[f"{base}/chains"]
        c = engine.link_contours(e, ch, cp)
    info = assert_same_polyarcs(c.poly_offsets, c.poly_ids, c.poly_info, gc, f"poly/{case}")
    bit = assert_polyarc_info(c.poly_info, info, label=case)
    print(f"[polyarcs] {case}: {c.num_polyarcs} polyarcs, {bit:.4f} of info values bit-identical")


def test_polyarcs_full_size_vs_restatement(engine, oracle):
    """The 1920x1080 map fused: edges -> curvelets -> fragments -> polyarcs."""
    e = synth.plain_hd(1000)
    res, c = engine.run_contours(e, contour_params=cvl.ContourParams(fit_polyarcs=True))
    oc = oracle.link_contours(e, res.chains)
    p = oracle.polyarcs(e, oc.frag_offsets, oc.frag_ids)
    assert np.array_equal(c.poly_offsets, p.offsets) and np.array_equal(c.poly_ids, p.ids)
    bit = assert_polyarc_info(c.poly_info, p.info, label="plain_hd")
    print(f"[polyarcs plain_hd] {c.num_polyarcs} polyarcs, {bit:.4f} bit-identical, whole path {c.device_ms:.2f} ms")
    # off by default; other model parameters
    assert engine.run_contours(e, want_curvelets=False)[1].poly_offsets is None
    cp = cvl.ContourParams(2, 2.0, fit_polyarcs=True, dx=0.5, max_k=0.4)
    _, c2 = engine.run_contours(e, contour_params=cp, want_curvelets=False)
    oc2 = oracle.link_contours(e, res.chains, 2, 2.0)
    p2 = oracle.polyarcs(e, oc2.frag_offsets, oc2.frag_ids, dx=0.5, max_k=0.4)
    assert np.array_equal(c2.poly_ids, p2.ids)
    assert_polyarc_info(c2.poly_info, p2.info, max_k=0.4, label="plain_hd dx 0.5")


def test_polyarcs_edge_cases(engine):
    e, ch = synth.contour_fuzz(3, n_edges=500)
    c = engine.link_contours(e, ch[:0], cvl.ContourParams(fit_polyarcs=True))  # no fragments
    assert c.num_polyarcs == 0 and c.poly_offsets.tolist() == [0]
    with pytest.raises(cvl.CvlError):
        engine.link_contours(e, ch, cvl.ContourParams(fit_polyarcs=True, token_len=0.0))


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1"])
def test_cli_polyarcs_files(tmp_path, gc, golden_files, key):
    """CURVELET --polyarcs writes output type 2: the polyarc chains (1-based, zero-padded
    to the longest) and their 12 info columns, 6 significant digits as the reference's
    writer prints them; the usual outputs stay byte-identical."""
    import subprocess
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cli_bin = os.path.join(root, "curvelet_construction_on_gpu_b200", "bin", "CURVELET")
    for d in ("bin", "test_files", "outputs"):
        (tmp_path / d).mkdir(exist_ok=True)
    synth.write_edge_file(str(tmp_path / "test_files" / f"{key}.txt"), golden_files[f"{key}/edges"])
    r = subprocess.run([cli_bin, "--double", "--edge-file", f"{key}.txt", "--output", f"chain_{key}.txt",
                        "--polyarcs", f"chain_poly_{key}.txt"], cwd=tmp_path / "bin", capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    cli = np.load(os.path.join(GOLDEN, "cli_outputs.npz"))
    assert (tmp_path / "outputs" / f"chain_{key}.txt").read_bytes() == cli[f"{key}/chain"].tobytes()
    offs, ids, info = gc[f"poly/{key}/offsets"], gc[f"poly/{key}/ids"], gc[f"poly/{key}/info"]
    w = int(np.diff(offs).max())
    rows = [[int(v) + 1 for v in ids[offs[i]:offs[i + 1]]] + [0] * (w - (offs[i + 1] - offs[i]))
            for i in range(len(offs) - 1)]
    got = (tmp_path / "outputs" / f"chain_poly_{key}.txt").read_text()
    assert got == "".join("".join(f"{v}\t" for v in row) + "\n" for row in rows)
    printed = np.array([[float(x) for x in ln.split()] for ln in
                        (tmp_path / "outputs" / f"info_poly_{key}.txt").read_text().splitlines()])
    assert printed.shape == info.shape
    mag = np.maximum(np.abs(printed), np.abs(info))
    assert np.all(np.abs(printed - info) <= 5e-6 * mag + 1e-300)  # 6 significant digits
