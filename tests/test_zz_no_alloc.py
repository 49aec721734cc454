"""cvl_pair_bundles_noalloc: pair bundles through a fixed per-device scratch,
with no engine and no device allocation, against the engine's
cvl_pair_bundles on the same pairs.

The GPU tests pass on their own in a fresh process and after the rest of the
suite; one of them also runs the calls in a child process whose first CUDA
work is the no-alloc call, so the per-device set-up runs there first."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import _abi
from curvelet_construction_on_gpu_b200.api import pair_bundles_noalloc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
MAX_PAIRS_63 = 15872  # 256 + a(48 n) + 2 a(504 n) + a(n) <= 16 MiB, a() = round up to 256


def random_pairs(n, seed):
    """(te_x, te_y, te_theta, le_x, le_y, le_theta) rows: the neighbour within the
    3.5 px radius of the anchor, about 1 in 8 closer than 2 dx (default bundle)."""
    rng = np.random.default_rng(seed)
    te = np.column_stack([rng.uniform(0, 1920, n), rng.uniform(0, 1080, n), rng.uniform(0, 2 * np.pi, n)])
    r = np.where(rng.random(n) < 0.125, rng.uniform(0.0, 0.8, n), rng.uniform(0.8, 3.5, n))
    a = rng.uniform(0, 2 * np.pi, n)
    le = np.column_stack([te[:, 0] + r * np.cos(a), te[:, 1] + r * np.sin(a), rng.uniform(0, 2 * np.pi, n)])
    return np.column_stack([te, le])


def assert_bundles_close(got, ref):
    """The no-alloc entry point and the engine's run the same kernel on the same
    pairs: validity, bounds and cell validity bit for bit."""
    bmin, bmax, valid = got[:3]
    rmin, rmax, rvalid = ref
    assert np.array_equal(valid, rvalid)
    assert np.array_equal(bmin.view(np.uint64), rmin.view(np.uint64))
    assert np.array_equal(bmax.view(np.uint64), rmax.view(np.uint64))


# ---- host-side checks (no device needed) ----------------------------------------
def test_noalloc_rejects_over_the_scratch_limit():
    lib = _abi.load()
    p = cvl.CurveletParams().to_c(0.0)
    one = np.zeros(1)
    cells = _abi.C.c_int32(0)
    count = _abi.C.c_uint32(7)
    u8 = np.zeros(1, np.uint8)
    rc = lib.cvl_pair_bundles_noalloc(one.ctypes.data_as(_abi._dp), MAX_PAIRS_63 + 1, _abi.C.byref(p),
                                      one.ctypes.data_as(_abi._dp), one.ctypes.data_as(_abi._dp),
                                      u8.ctypes.data_as(_abi.C.POINTER(_abi.C.c_uint8)), _abi.C.byref(count),
                                      _abi.C.byref(cells))
    assert rc == _abi.CVL_EOVERFLOW
    msg = lib.cvl_last_error().decode()
    assert f"at most {MAX_PAIRS_63} pairs of 63 cells" in msg, msg
    assert cells.value == 63 and count.value == 0


def test_noalloc_rejects_null_arguments():
    lib = _abi.load()
    p = cvl.CurveletParams().to_c(0.0)
    one = np.zeros(1)
    cells = _abi.C.c_int32(0)
    count = _abi.C.c_uint32(0)
    rc = lib.cvl_pair_bundles_noalloc(one.ctypes.data_as(_abi._dp), 1, _abi.C.byref(p), None,
                                      one.ctypes.data_as(_abi._dp), None, _abi.C.byref(count), _abi.C.byref(cells))
    assert rc == _abi.CVL_EINVAL


# ---- GPU ------------------------------------------------------------------------
@pytest.mark.gpu
def test_noalloc_two_calls_match_engine(engine):
    """Two calls in a row on different pairs: each equals the engine entry point,
    and each call's valid-pair count is its own (the counter is cleared)."""
    for n, seed in ((5000, 1), (3001, 2)):
        q = random_pairs(n, seed)
        got = pair_bundles_noalloc(q)
        ref = engine.pair_bundles(q)
        assert_bundles_close(got, ref)
        assert got[3] == int(ref[2].sum())
        print(f"[noalloc] n={n}: valid={got[3]}, bit-identical to the engine entry point")


@pytest.mark.gpu
def test_noalloc_reference_pairs(golden_pairs):
    bmin, bmax, valid, count = pair_bundles_noalloc(golden_pairs["pairs"])
    rmin, rmax = golden_pairs["bmin"], golden_pairs["bmax"]
    assert np.array_equal(valid, golden_pairs["valid"].astype(bool))
    assert count == int(golden_pairs["valid"].sum())
    assert np.array_equal(bmax > bmin, rmax > rmin)
    for a, b in ((bmin, rmin), (bmax, rmax)):
        assert np.all(np.abs(a - b) <= np.maximum(1e-9 * np.maximum(np.abs(a), np.abs(b)), 1e-9 * 0.3))


@pytest.mark.gpu
def test_noalloc_largest_call_and_params(engine):
    q = random_pairs(MAX_PAIRS_63, 3)
    got = pair_bundles_noalloc(q)
    assert_bundles_close(got, engine.pair_bundles(q))
    # another grid: dt = 10 deg, sx = 0.2 -> P = 5, Q = 5 (cpu_curvelet.hpp:73-74)
    prm = cvl.CurveletParams(dt_deg=10.0, sx=0.2, max_k=0.5)
    q = random_pairs(2000, 4)
    got = pair_bundles_noalloc(q, prm)
    assert got[0].shape == (2000, 25)
    assert_bundles_close(got, engine.pair_bundles(q, prm))
    assert pair_bundles_noalloc(np.zeros((0, 6)))[3] == 0


@pytest.mark.gpu
def test_noalloc_first_in_a_fresh_process():
    """A child process whose first CUDA work is the no-alloc call (set-up on the
    device), then a second call, then the engine entry point to compare with.
    The same child checks that the calls allocate no device memory: the device's
    free memory is the same before and after further calls, the largest one
    included."""
    code = textwrap.dedent("""
        import numpy as np, sys
        sys.path.insert(0, %r)
        from tests.test_zz_no_alloc import random_pairs, assert_bundles_close, MAX_PAIRS_63
        import curvelet_construction_on_gpu_b200 as cvl
        from curvelet_construction_on_gpu_b200.api import pair_bundles_noalloc
        a, b = random_pairs(4000, 11), random_pairs(2500, 12)
        ga, gb = pair_bundles_noalloc(a), pair_bundles_noalloc(b)
        import torch
        free0 = torch.cuda.mem_get_info(0)[0]
        free0 = torch.cuda.mem_get_info(0)[0]
        big = random_pairs(MAX_PAIRS_63, 13)
        for q in (big, a, big):
            pair_bundles_noalloc(q)
        free1 = torch.cuda.mem_get_info(0)[0]
        assert free1 == free0, ("device memory changed", free0, free1)
        eng = cvl.Engine()
        for q, g in ((a, ga), (b, gb)):
            ref = eng.pair_bundles(q)
            assert_bundles_close(g, ref)
            assert g[3] == int(ref[2].sum())
        eng.close()
        print("fresh-process noalloc ok", ga[3], gb[3], "free bytes", free0, free1)
    """ % ROOT)
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "fresh-process noalloc ok" in r.stdout
    print(r.stdout.strip())
