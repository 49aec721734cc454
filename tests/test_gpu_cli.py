"""The drop-in CURVELET program on the GPU: run the way the reference's is (from
bin/, input in ../test_files/, output in ../outputs/), its chain and info files
equal the ones the reference program wrote for the same edges, byte for byte
(tests/golden/cli_outputs.npz; digests for TO_edges.txt)."""
import hashlib
import os
import subprocess

import numpy as np
import pytest

from curvelet_construction_on_gpu_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
CLI = os.path.join(ROOT, "curvelet_construction_on_gpu_b200", "bin", "CURVELET")


def _run_cli(tmp_path, key, edges):
    for d in ("bin", "test_files", "outputs"):
        (tmp_path / d).mkdir(exist_ok=True)
    synth.write_edge_file(str(tmp_path / "test_files" / f"{key}.txt"), edges)  # %.17g: the same doubles
    out = f"chain_{key}.txt"
    r = subprocess.run([CLI, "--double", "--edge-file", f"{key}.txt", "--output", out], cwd=tmp_path / "bin",
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    return (tmp_path / "outputs" / out).read_bytes(), (tmp_path / "outputs" / f"info_{key}.txt").read_bytes()


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1", "TO_edges"])
def test_cli_outputs_byte_identical(tmp_path, key):
    ref = np.load(os.path.join(GOLDEN, "reference_files.npz"))
    cli = np.load(os.path.join(GOLDEN, "cli_outputs.npz"))
    chain, info = _run_cli(tmp_path, key, ref[f"{key}/edges"])
    if f"{key}/chain" in cli.files:
        assert chain == cli[f"{key}/chain"].tobytes()
        assert info == cli[f"{key}/info"].tobytes()
    else:
        assert [len(chain), len(info)] == cli[f"{key}/lengths"].tolist()
        assert hashlib.sha256(chain).hexdigest() == str(cli[f"{key}/chain_sha256"])
        assert hashlib.sha256(info).hexdigest() == str(cli[f"{key}/info_sha256"])
