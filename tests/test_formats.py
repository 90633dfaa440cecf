"""The reference's CSV input and binary result layout (no GPU needed)."""
from __future__ import annotations

import struct

import numpy as np

from conftest import load_package


def test_csv_round_trip_with_and_without_cluster(tmp_path):
    f = load_package().formats
    rng = np.random.Generator(np.random.PCG64(1))
    x = rng.standard_normal((17, 5), dtype=np.float32)
    lab = rng.integers(0, 4, 17).astype(np.int32)
    p = str(tmp_path / "a.csv")
    f.write_csv(p, x, lab)
    assert f.read_header(p) == (17, 5)
    y, l2 = f.read_csv(p, klaster=True)
    np.testing.assert_array_equal(x, y)
    np.testing.assert_array_equal(lab, l2)
    f.write_csv(p, x)
    y, l2 = f.read_csv(p, klaster=False)
    np.testing.assert_array_equal(x, y)
    assert not l2.any()


def test_csv_strtok_and_trim_semantics(tmp_path):
    """Spaces around tokens are trimmed and empty tokens vanish (strtok)."""
    f = load_package().formats
    p = tmp_path / "b.csv"
    p.write_text("2\n3\n 1.5 ,, 2 ,3\n4,5,6,\n")
    x, _ = f.read_csv(str(p))
    np.testing.assert_array_equal(x, np.array([[1.5, 2, 3], [4, 5, 6]], dtype=np.float32))


def test_result_layout_bytes(tmp_path):
    """Header "N;k;8\\n", long 0x01020304, then k records per point whose low 4
    bytes are the int32 id and high 4 bytes the float32 stored distance."""
    f = load_package().formats
    idx = np.array([[1, 2], [0, 2], [1, 0]], dtype=np.int32)
    dist = np.array([[1.0, 2.0], [1.0, 3.0], [3.0, 2.0]], dtype=np.float32)
    p = str(tmp_path / "out.bin")
    f.write_result(p, idx, dist, metric=0)
    raw = open(p, "rb").read()
    assert raw.startswith(b"3;2;8\n")
    off = len(b"3;2;8\n")
    assert struct.unpack("<q", raw[off:off + 8])[0] == 0x01020304
    rec = raw[off + 8:]
    assert len(rec) == 3 * 2 * 8
    i0, d0 = struct.unpack("<if", rec[:8])
    assert (i0, d0) == (1, 1.0)
    n, k, ri, rd = f.read_result(p)
    assert (n, k) == (3, 2)
    np.testing.assert_array_equal(ri, idx)
    np.testing.assert_array_equal(rd, dist)
    assert open(p + "VALIDATION").read() == "Everything is OK."


def test_stored_distance_conventions():
    f = load_package().formats
    d = np.array([4.0, 0.25], dtype=np.float32)
    np.testing.assert_array_equal(f.stored_distance(d, 0), d)            # L2 as is
    np.testing.assert_array_equal(f.stored_distance(d, 1), [2.0, 0.5])   # sqrt(L1)
    np.testing.assert_array_equal(f.stored_distance(d, 2), [-3.0, 0.75])  # similarity


def test_debug_side_file(tmp_path):
    f = load_package().formats
    p = str(tmp_path / "o")
    f.write_result(p, np.array([[1], [0]], dtype=np.int32), np.array([[0.5], [0.5]], np.float32),
                   metric=0, debug=True)
    assert open(p + "DEBUG").read() == "NEAR: <0, 1>(0.5) ;\nNEAR: <1, 0>(0.5) ;\n"
