"""The --float mode (the reference's run_curvelet<float>, cpu_curvelet/main.cpp:110)
on the GPU, through cvl_run_f32, against the reference's own float instantiation:
the committed fixtures of tests/golden/reference_files_f32.npz (made by
tests/golden/make_golden_f32.py), the reference harness in-process where it is
built, and the reference program's --float output files (cli_outputs.npz "f32/").

Rules (tests/parity.py): counts and chains identical, the info columns without
a transcendental input bit-identical, the others within the float tolerance.
The KAT blob150 truncates all 150 anchors at max_candidates, where the choice
inside a pixel cell follows libstdc++'s unstable sort in the reference and the
lowest edge ids here: against the whole reference run its truncation-independent
counts must agree, and against the reference's curvelet stage run on the
lowest-index lists (tests/golden/truncated_lowest.npz) everything must."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import synth
from tests.parity import assert_same_curvelets

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CLI = os.path.join(ROOT, "curvelet_construction_on_gpu_b200", "bin", "CURVELET")


class _Ref:
    def __init__(self, chains, info):
        self.chains, self.info = chains, info


@pytest.fixture(scope="module")
def g32():
    return np.load(os.path.join(GOLDEN, "reference_files_f32.npz"))


def _counts(r):
    return [r.num_curvelets, r.valid_pairs, r.total_neighbor_pairs, r.max_num_of_neighbors]


def test_float_kat_maps(engine, g32):
    names = sorted({k.split("/")[1] for k in g32.files if k.startswith("kat/")})
    assert len(names) == 8
    for name in names:
        e = g32[f"kat/{name}/edges"]
        gms, mc = g32[f"kat/{name}/params"].tolist()
        r = engine.run(e, cvl.CurveletParams(group_max_sz=gms, max_candidates=mc, edge_data_sz=e.shape[1]),
                       scalar="float")
        ref = g32[f"kat/{name}/counts"].tolist()
        if r.truncated_anchors:
            assert name == "blob150" and r.truncated_anchors == 150
            assert _counts(r)[2:] == ref[2:], name
            continue
        assert _counts(r) == ref, name
        st = assert_same_curvelets(r, _Ref(g32[f"kat/{name}/chains"], g32[f"kat/{name}/info"]),
                                   label=name, scalar="float")
        print(f"[float kat] {name}: {st}")


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1", "TO_edges"])
def test_float_sample_files(engine, g32, key):
    e = g32[f"{key}/edges"]
    assert e.dtype == np.float32
    r = engine.run(e, scalar="float")
    assert _counts(r) == g32[f"{key}/counts"].tolist()
    if f"{key}/chains" in g32.files:
        st = assert_same_curvelets(r, _Ref(g32[f"{key}/chains"], g32[f"{key}/info"]), label=key, scalar="float")
        print(f"[float file] {key}: {st}")
    else:
        assert hashlib.sha256(np.ascontiguousarray(r.chains).tobytes()).hexdigest() == str(g32[f"{key}/digests"][0])


@pytest.mark.parametrize("case", ["blob150", "blob600_mc128", "blob600_mc40"])
def test_float_truncated_vs_reference_stage(engine, golden_trunc, case):
    """Every anchor truncated: the float engine against the reference's
    run_curvelet<float> curvelet stage on the same lowest-index float lists."""
    k = f"{case}/float"
    e = golden_trunc[f"{k}/edges"]
    assert e.dtype == np.float32
    gms, mc = golden_trunc[f"{k}/params"].tolist()
    r = engine.run(e, cvl.CurveletParams(group_max_sz=gms, max_candidates=mc, edge_data_sz=e.shape[1]),
                   scalar="float")
    assert _counts(r) + [r.truncated_anchors] == golden_trunc[f"{k}/counts"].tolist()
    st = assert_same_curvelets(r, _Ref(golden_trunc[f"{k}/chains"], golden_trunc[f"{k}/info"]),
                               label=case + " f32 vs reference stage", scalar="float")
    print(f"[float truncated] {case}: {st}")


def test_float_input_checks(engine):
    # float64 edges are not converted silently: the caller says which instantiation
    e = synth.plain_small(3)
    with pytest.raises((TypeError, ValueError)):
        engine.run(e, scalar="float")
    with pytest.raises(ValueError):
        engine.run(e.astype(np.float32), scalar="half")
    # the same argument checks as cvl_run: an empty map is CVL_EINVAL
    with pytest.raises(cvl.CvlError):
        engine.run(np.zeros((0, 4), np.float32), scalar="float")
    with pytest.raises(cvl.CvlError):
        engine.run(np.zeros((5, 3), np.float32), scalar="float")


@pytest.mark.parametrize("seed", [0, 5])
def test_float_plain_small_vs_reference(engine, oracle, seed):
    if not oracle.ref_available():
        pytest.skip("reference harness not built here")
    e = synth.plain_small(seed).astype(np.float32)
    r = engine.run(e, scalar="float")
    o = oracle.ref_run(e, nthreads=16, scalar="float")
    assert _counts(r) == [o.num_curvelets, o.valid_pairs, o.total_neighbor_pairs, o.max_num_of_neighbors]
    print(f"[float plain_small {seed}]", assert_same_curvelets(r, o, label="plain_small f32", scalar="float"))


def test_float_plain_hd_full_size_vs_reference(engine, oracle):
    """The 1920x1080 map, about 250k edges, 500k curvelets."""
    if not oracle.ref_available():
        pytest.skip("reference harness not built here")
    e = synth.plain_hd(1000).astype(np.float32)
    r = engine.run(e, scalar="float")
    o = oracle.ref_run(e, nthreads=os.cpu_count() or 8, scalar="float")
    assert _counts(r) == [o.num_curvelets, o.valid_pairs, o.total_neighbor_pairs, o.max_num_of_neighbors]
    print("[float plain_hd]", assert_same_curvelets(r, o, label="plain_hd f32", scalar="float"))


def _run_cli_float(tmp_path, key, edges32):
    for d in ("bin", "test_files", "outputs"):
        (tmp_path / d).mkdir(exist_ok=True)
    # %.9g prints every float32 exactly enough that strtof gives it back
    np.savetxt(tmp_path / "test_files" / f"{key}.txt", edges32.astype(np.float64), fmt="%.9g", delimiter="\t")
    out = f"chain_{key}.txt"
    r = subprocess.run([CLI, "--float", "--edge-file", f"{key}.txt", "--output", out], cwd=tmp_path / "bin",
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "Using scalar type: float" in r.stdout
    return (tmp_path / "outputs" / out).read_bytes(), (tmp_path / "outputs" / f"info_{key}.txt").read_bytes()


def _parse_info(b):
    return np.array([[float(x) for x in ln.split()] for ln in b.decode().splitlines()])


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1", "TO_edges"])
def test_cli_float_outputs(tmp_path, g32, key):
    """Chain files byte-identical to the reference program's --float run. Info
    files print 6 significant digits; they are byte-identical unless a value
    within the float tolerance straddles a printed digit, so lines that differ
    are checked value by value against the reference's printed values."""
    cli = np.load(os.path.join(GOLDEN, "cli_outputs.npz"))
    edges = g32[f"{key}/edges"]
    chain, info = _run_cli_float(tmp_path, key, edges)
    k = "f32/" + key
    if f"{k}/chain" in cli.files:
        assert chain == cli[f"{k}/chain"].tobytes()
        ref_info = cli[f"{k}/info"].tobytes()
        if info != ref_info:
            a, b = _parse_info(info), _parse_info(ref_info)
            assert a.shape == b.shape
            diff_rows = np.any(a != b, axis=1)
            # printed values are rounded to 6 digits: allow one unit in the 6th digit
            mag = np.maximum(np.abs(a), np.abs(b))
            assert np.all(np.abs(a - b) <= np.maximum(1e-5 * mag, 1e-4 * 0.3) + 1e-12)
            print(f"[cli float] {key}: {int(diff_rows.sum())} of {a.shape[0]} info lines differ in print")
    else:
        assert len(chain) == int(cli[f"{k}/lengths"][0])
        assert hashlib.sha256(chain).hexdigest() == str(cli[f"{k}/chain_sha256"])
        same = hashlib.sha256(info).hexdigest() == str(cli[f"{k}/info_sha256"])
        print(f"[cli float] {key}: info file byte-identical: {same}")
