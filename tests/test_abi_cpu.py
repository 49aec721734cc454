"""C ABI checks that need no GPU: the library loads, exports every entry point
include/cvl.h declares, keeps the reference defaults, rejects bad arguments
before touching a device, and fails loudly (no CPU fallback) without a GPU."""
import ctypes as C
import os
import re
import subprocess

import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h")]


def _declared():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"\b(cvl_[a-z0-9_]+)\s*\(", src):
            names.add(m.group(1))
    return sorted(names)


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(_abi.LIB_PATH)
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers all of them
    bound = {n for n, _, _ in _abi.SIGNATURES}
    assert set(names) <= bound, sorted(set(names) - bound)


def test_param_defaults_match_reference():
    p = _abi.CvlParams()
    _abi.load().cvl_params_default(C.byref(p))
    # cpu_curvelet/param_settings.hpp:11-23
    assert (p.nrad, p.gap, p.dx, p.dt_deg, p.max_k) == (3.5, 1.5, 0.4, 15.0, 0.3)
    assert (p.curvelet_style, p.group_max_sz, p.out_type) == (2, 4, 0)
    assert (p.sx, p.st, p.edge_data_sz, p.max_candidates) == (0.1, 0.08, 4, 128)
    assert p.dt_rad == 0.0
    py = cvl.CurveletParams()
    assert (py.nrad, py.dx, py.dt_deg, py.max_k, py.group_max_sz, py.sx, py.st, py.max_candidates) == \
        (3.5, 0.4, 15.0, 0.3, 4, 0.1, 0.08, 128)


def test_null_arguments_are_rejected():
    lib = _abi.load()
    r = C.c_void_p()
    assert lib.cvl_run(None, None, 0, 4, None, C.byref(r)) == _abi.CVL_EINVAL
    assert lib.cvl_result_get(None, None) == _abi.CVL_EINVAL
    assert lib.cvl_engine_create(None, None) == _abi.CVL_EINVAL
    assert lib.cvl_engine_warmup(None) == _abi.CVL_EINVAL
    assert "NULL" in lib.cvl_last_error().decode()
    assert lib.cvl_version().decode().startswith("cvl ")


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_no_gpu_fails_loudly():
    with pytest.raises(cvl.CvlError) as ei:
        cvl.Engine()
    assert ei.value.code == _abi.CVL_ENODEV


def test_cli_flags_without_gpu(tmp_path):
    cli = os.path.join(ROOT, "curvelet_construction_on_gpu_b200", "bin", "CURVELET")
    assert os.path.exists(cli), "CLI not built"
    r = subprocess.run([cli, "--help"], capture_output=True, text=True)
    assert r.returncode == 0 and "--max-candidates" in r.stderr
    r = subprocess.run([cli, "--bogus"], capture_output=True, text=True)
    assert r.returncode == 1 and "Unknown argument: --bogus" in r.stderr
    r = subprocess.run([cli, "--nrad", "abc"], capture_output=True, text=True)
    assert r.returncode == 1 and "invalid value for --nrad" in r.stderr
    # missing input file is reported before any device work (data_io.hpp:27-31)
    run_dir = tmp_path / "run"
    run_dir.mkdir()
    r = subprocess.run([cli, "--edge-file", "nope.txt"], capture_output=True, text=True, cwd=run_dir)
    assert r.returncode == 1 and "input file does not exist: ../test_files/nope.txt" in r.stderr


def test_server_defaults_and_argument_checks():
    lib = _abi.load()
    cfg = _abi.CvlServerCfg()
    lib.cvl_server_cfg_default(C.byref(cfg))
    assert (cfg.device, cfg.workers, cfg.mem_budget_bytes) == (0, 4, 40 << 30)
    # admission by the workspace formula (admit_bytes_per_edge 0)
    assert (cfg.admit_bytes_per_edge, cfg.max_batch_edges, cfg.large_map_edges) == (0, 2 << 20, 1_000_000)
    assert cfg.host_reserve_bytes == 2 << 30 and cfg.small_takes_large == 0 and cfg.large_workers == 0
    assert cfg.large_yield_ms == 10 and cfg.device_reserve_bytes == 0
    assert (cfg.max_map_edges, cfg.pairs_per_edge, cfg.curvelets_per_edge) == (4 << 20, 40.0, 8.0)
    ec = _abi.CvlEngineCfg()
    lib.cvl_engine_cfg_default(C.byref(ec))
    assert ec.stream_priority == 0
    h = C.c_void_p()
    p = cvl.CurveletParams().to_c()
    assert lib.cvl_server_create(C.byref(cfg), None, C.byref(h)) == _abi.CVL_EINVAL
    bad = _abi.CvlServerCfg()
    lib.cvl_server_cfg_default(C.byref(bad))
    bad.workers = 0
    assert lib.cvl_server_create(C.byref(bad), C.byref(p), C.byref(h)) == _abi.CVL_EINVAL
    lib.cvl_server_cfg_default(C.byref(bad))
    bad.pairs_per_edge = -1.0
    assert lib.cvl_server_create(C.byref(bad), C.byref(p), C.byref(h)) == _abi.CVL_EINVAL
    shp = _abi.CvlWorkspaceShape(1000, 16000, 3000, 1, 4)
    tot = C.c_size_t(0)
    assert lib.cvl_engine_workspace_bytes(None, C.byref(shp), C.byref(p), C.byref(tot), None) == _abi.CVL_EINVAL
    assert lib.cvl_engine_reserve_workspace(None, C.byref(shp), C.byref(p)) == _abi.CVL_EINVAL
    rid = C.c_uint64(0)
    assert lib.cvl_server_submit(None, None, 1, 4, C.byref(rid)) == _abi.CVL_EINVAL
    assert lib.cvl_server_wait(None, 1, 0, C.byref(h)) == _abi.CVL_EINVAL


@pytest.mark.skipif(_has_gpu(), reason="checks the no-GPU failure path")
def test_server_without_gpu_fails_loudly():
    with pytest.raises(cvl.CvlError) as ei:
        cvl.Server()
    assert ei.value.code == _abi.CVL_ENODEV


def test_tuning_buckets():
    lib = _abi.load()
    assert [lib.cvl_tuning_bucket(n) for n in (1, 64 << 10, (64 << 10) + 1, 512 << 10, (512 << 10) + 1,
                                                 4 << 20, (4 << 20) + 1, 1 << 30)] == [0, 0, 1, 1, 2, 2, 3, 3]
    t = _abi.CvlTuning()
    assert lib.cvl_engine_set_tuning(None, 0, C.byref(t)) == _abi.CVL_EINVAL
    assert lib.cvl_engine_get_tuning(None, 0, C.byref(t)) == _abi.CVL_EINVAL


def test_allocation_injector_arms_and_disarms():
    """The injector is host state: arming and disarming need no device."""
    lib = _abi.load()
    assert lib.cvl_debug_fail_allocations(5) == _abi.CVL_OK
    assert lib.cvl_debug_fail_allocations(-1) == _abi.CVL_OK
    assert lib.cvl_debug_fail_allocations(-2) == _abi.CVL_EINVAL
