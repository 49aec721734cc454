"""The output file format (data_io.hpp:81-145), checked on the CPU: the
Python writers, fed the reference's own chains and info rows, reproduce the
files that the reference's CURVELET program wrote, byte for byte
(tests/golden/cli_outputs.npz, made by tests/golden/make_cli_golden.py)."""
import os

import numpy as np
import pytest

from curvelet_construction_on_gpu_b200 import data_io

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1"])
def test_writers_match_reference_files(tmp_path, key):
    ref = np.load(os.path.join(GOLDEN, "reference_files.npz"))
    cli = np.load(os.path.join(GOLDEN, "cli_outputs.npz"))
    out = f"chain_{key}.txt"
    data_io.write_int_array_to_file(out, ref[f"{key}/chains"], str(tmp_path))
    data_io.write_double_array_to_file(data_io.chain_to_info_filename(out), ref[f"{key}/info"], str(tmp_path))
    assert (tmp_path / out).read_bytes() == cli[f"{key}/chain"].tobytes()
    assert (tmp_path / f"info_{key}.txt").read_bytes() == cli[f"{key}/info"].tobytes()


@pytest.mark.parametrize("key", ["TO_edges_digit1", "TO_edges_ABC_0006_thresh1"])
def test_writers_match_reference_float_files(tmp_path, key):
    """The float fixtures (the reference's run_curvelet<float> in-process, made by
    make_golden_f32.py) written out equal the reference program's --float files:
    the in-process float instantiation is the program's."""
    ref = np.load(os.path.join(GOLDEN, "reference_files_f32.npz"))
    cli = np.load(os.path.join(GOLDEN, "cli_outputs.npz"))
    out = f"chain_{key}.txt"
    data_io.write_int_array_to_file(out, ref[f"{key}/chains"], str(tmp_path))
    data_io.write_double_array_to_file(data_io.chain_to_info_filename(out), ref[f"{key}/info"], str(tmp_path))
    assert (tmp_path / out).read_bytes() == cli[f"f32/{key}/chain"].tobytes()
    assert (tmp_path / f"info_{key}.txt").read_bytes() == cli[f"f32/{key}/info"].tobytes()
