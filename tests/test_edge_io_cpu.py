"""Edge files on the CPU (cvl_read_edges / cvl_write_edges_binary): the
multi-threaded reader gives the same values, bit for bit, and the same error
messages as the reference's line-by-line stream reader (read_TO_edges_from_file,
data_io.hpp:22-79; nthreads -1 runs that loop) on plain and on unusual input;
the binary format round-trips."""
import numpy as np
import pytest

from curvelet_construction_on_gpu_b200 import data_io


def _both(path, vpe=4):
    """(values or error) of the parallel reader and of the stream reader."""
    out = []
    for nt in (8, -1):
        try:
            out.append(("ok", data_io.read_edges(str(path), vpe, nt)))
        except ValueError as e:
            out.append(("err", str(e)))
    return out


def _same(path, vpe=4):
    (k1, v1), (k2, v2) = _both(path, vpe)
    assert k1 == k2, (v1, v2)
    if k1 == "ok":
        assert v1.shape == v2.shape and np.array_equal(v1.view(np.uint64), v2.view(np.uint64))
    else:
        assert v1 == v2
    return k1, v1


@pytest.mark.parametrize("fmt", ["%.17g", "%.6f", "%.10e", "%g"])
def test_plain_files_match_the_stream_reader(tmp_path, fmt):
    rng = np.random.default_rng(11)
    e = np.column_stack([rng.uniform(-5000, 5000, 30000), rng.uniform(0, 3000, 30000),
                         rng.uniform(-np.pi, np.pi, 30000), rng.uniform(0, 1e-3, 30000)])
    p = tmp_path / "plain.txt"
    np.savetxt(p, e, fmt=fmt, delimiter="\t")
    kind, v = _same(p)
    assert kind == "ok" and v.shape == (30000, 4)
    p2 = tmp_path / "spaces.txt"
    p2.write_text("".join("  " + "   ".join(fmt % x for x in r) + " \t\n" for r in e[:5000]))
    _same(p2)


UNUSUAL = {
    "plus_sign": "+1.5 2 3 4\n5 6 7 8\n",
    "inf": "1 2 inf 4\n",
    "nan": "1 nan 3 4\n",
    "hex": "0x10 2 3 4\n",
    "junk_after_number": "1.5x 2 3 4\n",
    "exponent_without_digits": "1e 2 3 4\n",
    "two_points": "1.5.3 2 3\n",
    "crlf": "1 2 3 4\r\n5 6 7 8\r\n",
    "no_final_newline": "1 2 3 4\n5 6 7 8",
    "trailing_empty_line": "1 2 3 4\n\n",
    "blank_line_inside": "1 2 3 4\n\n5 6 7 8\n",
    "whitespace_line": "1 2 3 4\n \t \n5 6 7 8\n",
    "missing_value": "1 2 3\n",
    "extra_value": "1 2 3 4 5\n",
    "text": "a b c d\n",
    "empty_file": "",
    "only_newlines": "\n\n",
    "overflow": "1e400 2 3 4\n",
    "underflow": "1e-400 2 3 4\n",
    "subnormal": "4.9e-324 2 3 4\n",
    "negative_zero": "-0 -0.0 0 1\n",
    "leading_point": "-.5 .25 5. 1\n",
    "vertical_tab": "1\v2 3 4\n",
}


@pytest.mark.parametrize("name", sorted(UNUSUAL))
def test_unusual_input_matches_the_stream_reader(tmp_path, name):
    p = tmp_path / f"{name}.txt"
    p.write_bytes(UNUSUAL[name].encode())
    _same(p)


def test_errors_at_chunk_boundaries(tmp_path):
    # a blank line or a bad value anywhere in a large file, including right at the
    # points where the reader splits the file over threads
    rng = np.random.default_rng(2)
    rows = ["%.17g\t%.17g\t%.17g\t%.17g" % tuple(r) for r in rng.uniform(0, 100, (20000, 4))]
    for k, bad in ((2500, ""), (10000, ""), (19999, "1 2 3"), (7, "x 1 2 3"), (15000, "1 2 3 4 5")):
        p = tmp_path / f"bad{k}.txt"
        p.write_text("\n".join(rows[:k] + [bad] + rows[k:]) + "\n")
        kind, msg = _same(p)
        assert kind == "err" and f"line {k + 1}" in msg


def test_missing_file_message(tmp_path):
    with pytest.raises(ValueError) as ei:
        data_io.read_edges(str(tmp_path / "nope.txt"))
    assert "Error: input file does not exist: " in str(ei.value)


def test_binary_round_trip_and_checks(tmp_path):
    rng = np.random.default_rng(4)
    e = rng.normal(size=(1234, 6))
    p = tmp_path / "m.cvle"
    data_io.write_edges_binary(str(p), e)
    assert np.array_equal(data_io.read_edges(str(p), 6).view(np.uint64), e.view(np.uint64))
    with pytest.raises(ValueError) as ei:
        data_io.read_edges(str(p), 4)
    assert "has 6 values per edge, expected 4" in str(ei.value)
    raw = p.read_bytes()
    (tmp_path / "t.cvle").write_bytes(raw[:-8])
    with pytest.raises(ValueError) as ei:
        data_io.read_edges(str(tmp_path / "t.cvle"), 6)
    assert "truncated" in str(ei.value)
    (tmp_path / "x.cvle").write_bytes(b"NOTEDGES" + raw[8:])
    with pytest.raises(ValueError) as ei:
        data_io.read_edges(str(tmp_path / "x.cvle"), 6)
    assert "not a binary edge file" in str(ei.value)


# ---- --float mode: read_TO_edges_from_file<float> reads each number straight to float ----
def _both_f32(path, vpe=4):
    out = []
    for nt in (8, -1):
        try:
            out.append(("ok", data_io.read_edges(str(path), vpe, nt, scalar="float")))
        except ValueError as e:
            out.append(("err", str(e)))
    (k1, v1), (k2, v2) = out
    assert k1 == k2, (v1, v2)
    if k1 == "ok":
        assert v1.dtype == np.float32 and v1.shape == v2.shape
        assert np.array_equal(v1.view(np.uint32), v2.view(np.uint32))
    else:
        assert v1 == v2
    return k1, v1


def test_float_reader_matches_strtof(tmp_path):
    """Each token rounded once, to nearest float (strtof), on all threads and in
    the stream reader; 17-digit tokens include values between two floats that a
    read through double would round twice."""
    from oracle import oracle as O
    rng = np.random.default_rng(12)
    e = np.column_stack([rng.uniform(-5000, 5000, 20000), rng.uniform(0, 3000, 20000),
                         rng.uniform(-np.pi, np.pi, 20000), rng.uniform(0, 1e-3, 20000)])
    # midpoints between adjacent floats, nudged by one double ulp either way
    f = rng.uniform(1, 2000, 4000).astype(np.float32)
    mid = (f.astype(np.float64) + np.nextafter(f, np.float32(np.inf)).astype(np.float64)) / 2
    e[:4000, 0] = np.nextafter(mid, np.inf)
    e[4000:8000, 1] = np.nextafter(mid, -np.inf)
    for fmt in ("%.17g", "%.6f", "%g"):
        p = tmp_path / "f.txt"
        np.savetxt(p, e, fmt=fmt, delimiter="\t")
        kind, v = _both_f32(p)
        assert kind == "ok"
        assert np.array_equal(v.view(np.uint32), O.parse_edges_f32(str(p)).view(np.uint32))


@pytest.mark.parametrize("name", ["plus_sign", "inf", "nan", "overflow", "underflow", "negative_zero",
                                  "leading_point", "missing_value", "text", "trailing_empty_line",
                                  "blank_line_inside", "crlf"])
def test_float_reader_unusual_input(tmp_path, name):
    p = tmp_path / f"{name}.txt"
    p.write_bytes(UNUSUAL[name].encode())
    _both_f32(p)


def test_float_reader_rejects_binary(tmp_path):
    p = tmp_path / "m.cvle"
    data_io.write_edges_binary(str(p), np.zeros((3, 4)))
    with pytest.raises(ValueError):
        data_io.read_edges(str(p), 4, scalar="float")
