"""Golden output files of the reference's own CURVELET program.

Runs in the development container only: it needs the reference's sample edge
files and oracle/_ref/CURVELET (built from the reference sources by
`make -C oracle`). For each sample file it runs that program the way its README
does (from a bin/ directory, input in ../test_files/, output in ../outputs/)
and keeps the exact bytes of the chain and info files it writes
(data_io.hpp:81-145), once with --double and once with --float (keys "f32/…"). For TO_edges.txt, whose outputs are 6.8 MB, it keeps the
SHA-256 digest and length of each file.

    python tests/golden/make_cli_golden.py  ->  tests/golden/cli_outputs.npz
"""
from __future__ import annotations

import hashlib
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
# the reference project's sample inputs: $CVL_REFERENCE_DIR/test_files
REF_DIR = os.path.join(os.environ.get("CVL_REFERENCE_DIR", ""), "test_files")


def _need_reference() -> None:
    if not os.path.isdir(REF_DIR) or not os.environ.get("CVL_REFERENCE_DIR"):
        raise SystemExit("set CVL_REFERENCE_DIR to the reference project's root (it holds test_files/)")
REF_CLI = os.path.join(ROOT, "oracle", "_ref", "CURVELET")
FILES = {"TO_edges_digit1": "full", "TO_edges_ABC_0006_thresh1": "full", "TO_edges": "digest"}


def run_reference(name: str, work: str, scalar: str = "--double") -> tuple[bytes, bytes]:
    for d in ("bin", "test_files", "outputs"):
        os.makedirs(os.path.join(work, d), exist_ok=True)
    shutil.copy(os.path.join(REF_DIR, name + ".txt"), os.path.join(work, "test_files", name + ".txt"))
    out = f"chain_{name}.txt"
    r = subprocess.run([REF_CLI, scalar, "--nthreads", str(os.cpu_count() or 1), "--edge-file", name + ".txt",
                        "--output", out], cwd=os.path.join(work, "bin"), capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(r.stdout + r.stderr)
    with open(os.path.join(work, "outputs", out), "rb") as fh:
        chain = fh.read()
    with open(os.path.join(work, "outputs", out.replace("chain", "info")), "rb") as fh:
        info = fh.read()
    return chain, info


def main() -> None:
    _need_reference()
    if not os.path.exists(REF_CLI):
        sys.exit("oracle/_ref/CURVELET is not built (make -C oracle)")
    out = {}
    with tempfile.TemporaryDirectory() as work:
        for scalar, tag in (("--double", ""), ("--float", "f32/")):
            for name, kind in FILES.items():
                chain, info = run_reference(name, os.path.join(work, tag + name), scalar)
                key = tag + name
                if kind == "full":
                    out[f"{key}/chain"] = np.frombuffer(chain, np.uint8)
                    out[f"{key}/info"] = np.frombuffer(info, np.uint8)
                else:
                    out[f"{key}/chain_sha256"] = np.array(hashlib.sha256(chain).hexdigest())
                    out[f"{key}/info_sha256"] = np.array(hashlib.sha256(info).hexdigest())
                    out[f"{key}/lengths"] = np.array([len(chain), len(info)], np.int64)
                print(scalar, name, len(chain), len(info))
    np.savez_compressed(os.path.join(HERE, "cli_outputs.npz"), **out)


if __name__ == "__main__":
    main()
