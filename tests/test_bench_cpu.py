"""Host-side logic of bench.py that needs no GPU: the whole-path HBM roofline
arithmetic, the clock-sample summary that decides whether a run saw throttling,
and the command line."""
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def bench():
    sys.path.insert(0, ROOT)
    import bench as b
    return b


def test_path_hbm_arithmetic(bench):
    peaks = {"hbm_gbs": 6500.0}
    r = bench.path_hbm(1_000_000, 2_000_000, 10.0, peaks)
    # 32 B per edge in + 100 B per curvelet out, over 10 ms
    assert r["bytes_per_step"] == 32e6 + 200e6
    assert r["achieved"] == pytest.approx(232e6 / 0.010 / 1e9)
    assert r["frac"] == pytest.approx(r["achieved"] / 6500.0)
    assert r["peak_source"].startswith("MEASURED_PEAKS.json")
    # six values per edge, and the fallback peak when none was measured
    r6 = bench.path_hbm(10, 0, 1.0, {}, edge_bytes=48)
    assert r6["bytes_per_step"] == 480.0 and r6["peak"] == 6650.0 and "fallback" in r6["peak_source"]
    assert bench.path_hbm(10, 10, 0.0, peaks)["achieved"] == 0.0


def test_clocks_summary(bench, tmp_path, monkeypatch):
    monkeypatch.setenv("CVL_BENCH_OUT", str(tmp_path))
    c = bench._Clocks(0)
    # index, clocks.sm, clocks.max.sm, power, active mask, hw_slowdown, hw_thermal, sw_thermal, sw_power_cap
    rows = ["0, 1965, 1965, 700.1, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
            "0, 1950, 1965, 990.5, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
            "0, 1965, 1965, 720.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active"]
    (tmp_path / "clocks_rank0.csv").write_text("\n".join(rows) + "\n")
    s = c.summary()
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0 and s["samples"] == 3
    assert s["reasons"] == ["sw_power_cap"]
    rows.append("0, 1200, 1965, 500.0, 0x0000000000000040, Not Active, Active, Not Active, Not Active")
    (tmp_path / "clocks_rank0.csv").write_text("\n".join(rows) + "\n")
    assert c.summary()["reasons"] == ["hw_thermal_slowdown", "sw_power_cap"]
    # no sampler output at all
    os.remove(tmp_path / "clocks_rank0.csv")
    assert c.summary()["reasons"] == ["unsampled"]


def test_bench_command_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--help"], capture_output=True, text=True,
                       timeout=120)
    assert r.returncode == 0
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--workload"):
        assert flag in r.stdout
