"""The .mda boundary format, pinned against files written by the reference's
own Python writer (tests/golden/make_golden.py)."""
import json
import os
import struct

import numpy as np
import pytest

from mountainsort_b200 import mdaio

GOLD = os.path.join(os.path.dirname(__file__), "golden")
DTYPES = ["uint8", "int16", "uint16", "float32", "int32", "uint32", "float64"]


def expected():
    with open(os.path.join(GOLD, "mda_expected.json")) as f:
        return json.load(f)


@pytest.mark.parametrize("dt", DTYPES)
def test_read_reference_written_files(dt):
    e = expected()
    X = mdaio.readmda(os.path.join(GOLD, f"mda_{dt}.mda"))
    assert X.dtype == np.dtype(dt)
    assert X.shape == (e["M"], e["N"])
    np.testing.assert_array_equal(X, np.array(e["values"]).astype(dt))
    np.testing.assert_array_equal(X, np.array(e["reference_readmda"][dt]))


@pytest.mark.parametrize("dt", DTYPES)
def test_write_is_byte_identical_to_reference_writer(dt, tmp_path):
    e = expected()
    X = np.array(e["values"])
    p = str(tmp_path / "x.mda")
    mdaio.writemda(X, p, dtype=dt)
    with open(p, "rb") as f, open(os.path.join(GOLD, f"mda_{dt}.mda"), "rb") as g:
        assert f.read() == g.read()


def test_chunked_writer_and_64bit_dims():
    e = expected()
    X = np.array(e["values"], dtype=np.float32)
    np.testing.assert_array_equal(mdaio.readmda(os.path.join(GOLD, "mda_chunked_float32.mda")), X)
    p = os.path.join(GOLD, "mda_dims64_float32.mda")
    h = mdaio.read_header_path(p)
    assert h.uses64bitdims and h.dims == (4, 12) and h.header_size == 28
    np.testing.assert_array_equal(mdaio.readmda(p), X)


def test_64bit_dims_round_trip(tmp_path):
    X = np.arange(24, dtype=np.float32).reshape(4, 6, order="F")
    p = str(tmp_path / "d64.mda")
    mdaio.writemda(X, p, uses64bitdims=True)
    with open(p, "rb") as f:
        code, nb, nd = struct.unpack("<iii", f.read(12))
    assert (code, nb, nd) == (-3, 4, -2)
    np.testing.assert_array_equal(mdaio.readmda(p), X)
    with open(os.path.join(GOLD, "mda_dims64_float32.mda"), "rb") as g, open(p, "rb") as f:
        assert f.read()[:28] == g.read()[:28][:12] + struct.pack("<qq", 4, 6)


def test_float_to_int_truncates(tmp_path):
    p = str(tmp_path / "t.mda")
    mdaio.writemda(np.array([[1.7, -1.7, 2.5, -0.2]], dtype=np.float32), p, dtype="int16")
    np.testing.assert_array_equal(mdaio.readmda(p), np.array([[1, -1, 2, 0]], dtype=np.int16))


@pytest.mark.parametrize("blob,msg", [
    (b"\x01\x00", "truncated"),
    (struct.pack("<iii", -9, 4, 2) + struct.pack("<ii", 1, 1), "data type"),
    (struct.pack("<iii", -3, 4, 0), "dims"),
    (struct.pack("<iii", -3, 4, 2) + struct.pack("<i", 3), "truncated"),
])
def test_corrupt_headers_rejected(tmp_path, blob, msg):
    p = str(tmp_path / "bad.mda")
    with open(p, "wb") as f:
        f.write(blob)
    with pytest.raises(mdaio.MdaError, match=msg):
        mdaio.readmda(p)


def test_short_file_rejected(tmp_path):
    p = str(tmp_path / "short.mda")
    with open(p, "wb") as f:
        f.write(struct.pack("<iiiii", -3, 4, 2, 4, 10) + b"\x00" * 12)
    with pytest.raises(mdaio.MdaError, match="short"):
        mdaio.readmda(p)


def test_atomic_write_leaves_no_tmp(tmp_path):
    p = str(tmp_path / "a.mda")
    mdaio.writemda(np.zeros((2, 3), np.float32), p)
    assert os.path.exists(p) and not os.path.exists(p + ".tmp")


@pytest.mark.parametrize("dt", [np.float32, np.int16])
def test_rows_view_and_block_writer(tmp_path, dt):
    """The streaming processors' file access: a memory map of an input's
    rows, and an output written block by block into a preallocated .tmp file
    (unwritten timepoints zero), renamed when closed or removed when aborted."""
    M, N = 5, 1001
    X = (np.arange(M * N).reshape(N, M) % 3000).astype(dt)
    src = str(tmp_path / "in.mda")
    mdaio.writemda(X.T, src)
    m, n, rows = mdaio.timeseries_rows_view(src)
    assert (m, n) == (M, N) and rows.dtype == dt
    np.testing.assert_array_equal(rows[10:20], X[10:20])
    out = str(tmp_path / "out.mda")
    w = mdaio.TimeseriesWriter(out, dt, M, N)
    assert os.path.exists(out + ".tmp") and not os.path.exists(out)
    w.write(0, X[:400])
    w.write(600, X[600:])
    w.close()
    assert not os.path.exists(out + ".tmp")
    Y = mdaio.readmda(out).T
    np.testing.assert_array_equal(Y[:400], X[:400])
    np.testing.assert_array_equal(Y[600:], X[600:])
    assert not Y[400:600].any()
    w = mdaio.TimeseriesWriter(str(tmp_path / "gone.mda"), dt, M, N)
    w.abort()
    assert not os.path.exists(str(tmp_path / "gone.mda.tmp"))
    # an empty timeseries is a header only
    e = str(tmp_path / "empty.mda")
    w = mdaio.TimeseriesWriter(e, dt, M, 0)
    w.close()
    assert mdaio.readmda(e).shape == (M, 0)
