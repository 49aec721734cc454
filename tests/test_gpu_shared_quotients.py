"""Markstein's shared-reciprocal quotient pair against two IEEE divisions, on the
device (tests/probes/shared_quotients.cu, built here with nvcc).

The bundle transport's two k_dx bounds share their divisor e1 in every cell. The
probe computes a1 / b and a2 / b from one correctly rounded reciprocal with two
residual corrections each, with the operands its proof does not cover (the four
largest significands, magnitudes outside [2^-500, 2^501), zeros, subnormals,
infinities, NaN) sent to '/'. It must equal '/' bit for bit on 6.2e9 operand
pairs over five operand families; the timings say what the shared reciprocal
would save in the transport (the engine keeps '/', see the printed times).
"""
import os
import re
import shutil
import subprocess

import pytest

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
