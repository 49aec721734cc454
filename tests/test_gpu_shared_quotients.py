"""Markstein's shared-reciprocal quotient pair against two IEEE divisions, on the
device: the probe (tests/probes/shared_quotients.cu, built here with nvcc), and the
bundle kernel's use of it against an engine that divides.

The bundle transport's two k_dx bounds share their divisor e1 in every cell. The
probe computes a1 / b and a2 / b from one correctly rounded reciprocal with two
residual corrections each, with the operands its proof does not cover (the four
largest significands, magnitudes outside [2^-500, 2^501), zeros, subnormals,
infinities, NaN) sent to '/'. It must equal '/' bit for bit on 6.2e9 operand
pairs over five operand families. The probe's timings compare the guarded form
(every operand checked) with two divisions; the bundle kernel checks only e1's
significand per cell, its runs certifying the other ranges once (certify_* in
csrc/cvl_kernels.cuh).
"""
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

import curvelet_construction_on_gpu_b200 as cvl
from curvelet_construction_on_gpu_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "probes", "shared_quotients.cu")


def _nvcc():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    pytest.skip("nvcc not found")


def test_shared_quotients_equal_ieee_division(tmp_path):
    exe = str(tmp_path / "shared_quotients")
    subprocess.run([_nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-fmad=false",
                    "-prec-div=true", "-o", exe, SRC], check=True, capture_output=True, text=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    checks = re.findall(r"check mode (\d) operands (\d+) mismatches (\d+)", out.stdout)
    assert len(checks) == 5
    for mode, n, bad in checks:
        assert int(n) > 10**9 and int(bad) == 0, (mode, n, bad)
    times = dict(re.findall(r"time (\w+) ([0-9.]+) ms", out.stdout))
    assert set(times) == {"two_divisions", "shared_two_corrections", "shared_one_correction", "shared_guarded"}


def _same(a, b):
    return (np.array_equal(a.chains, b.chains) and np.array_equal(a.info.view(np.uint64), b.info.view(np.uint64))
            and a.valid_pairs == b.valid_pairs and a.total_neighbor_pairs == b.total_neighbor_pairs)


def test_engine_shared_quotients_equal_divisions(engine, monkeypatch):
    """The bundle kernel's shared-reciprocal quotients (certified runs) against an
    engine that divides (CVL_NO_SHARED_QUOTIENTS): identical chains and info, bit
    for bit, through the kernel-by-kernel path, both graph buckets and a batch; and
    on a map with coordinates below 2^-40, which the run does not certify."""
    monkeypatch.setenv("CVL_NO_SHARED_QUOTIENTS", "1")
    divide = cvl.Engine()
    monkeypatch.delenv("CVL_NO_SHARED_QUOTIENTS")
    try:
        tiny = synth.plain_small(5).copy()
        tiny[:40, 0] = np.ldexp(tiny[:40, 0] - np.floor(tiny[:40, 0]), -45)  # x below 2^-40: uncertified
        maps = [synth.plain_hd(1000), synth.plain_small(3), synth.mixed_map(2041), tiny]
        for m in maps:
            assert _same(engine.run(m), divide.run(m))
        got, want = engine.run_maps(maps[1:]), divide.run_maps(maps[1:])
        assert all(_same(a, b) for a, b in zip(got, want))
    finally:
        divide.close()


def test_sincos_equals_sin_and_cos(tmp_path):
    """The neighbour kernel's anchor trig row comes from sincos (tests/probes/
    sincos_identity.cu): bit for bit the values of sin and cos, in double and float."""
    exe = str(tmp_path / "sincos_identity")
    subprocess.run([_nvcc(), "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-fmad=false",
                    "-o", exe, os.path.join(HERE, "probes", "sincos_identity.cu")], check=True,
                   capture_output=True, text=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=300)
    print(out.stdout)
    assert out.returncode == 0, out.stdout + out.stderr
    checks = re.findall(r"check mode (\d) arguments (\d+) mismatches (\d+)", out.stdout)
    assert len(checks) == 3
    for mode, n, bad in checks:
        assert int(n) > 10**8 and int(bad) == 0, (mode, n, bad)
