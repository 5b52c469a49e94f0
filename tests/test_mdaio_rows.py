"""Block I/O of the processor executable (RowReader / RowWriter in
mountainsort_b200/csrc/mdaio.cpp), compiled with a small driver and checked
against numpy on the CPU: rows of a file or of a directory's files
concatenated in time, other data types converted to float32 as mdaReadData
converts them, int16 kept as int16, large blocks read by several threads,
and outputs written into a preallocated .tmp file that is renamed on commit
and removed otherwise."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from mountainsort_b200 import mdaio

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mountainsort_b200", "csrc")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("drv") / "mdaio_rows_driver")
    r = subprocess.run([gxx, "-O1", "-std=c++17", "-pthread", "-I", CSRC,
                        os.path.join(ROOT, "tests", "cpp", "mdaio_rows_driver.cpp"), os.path.join(CSRC, "mdaio.cpp"),
                        "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def _run(driver, *args):
    return subprocess.run([driver, *map(str, args)], capture_output=True, text=True, timeout=120)


def _read(driver, tmp_path, path, as_type, t0, nt, M):
    out = tmp_path / "blk.bin"
    r = _run(driver, "read", path, as_type, t0, nt, out)
    assert r.returncode == 0, r.stderr
    dt = np.int16 if as_type == "i16" else np.float32
    return np.fromfile(out, dtype=dt).reshape(nt, M)


def test_file_rows_and_conversions(driver, tmp_path):
    rng = np.random.default_rng(0)
    M, N = 5, 3001
    for dt in [np.float32, np.float64, np.int16, np.int32, np.uint16, np.uint8]:
        X = (rng.standard_normal((N, M)) * 100).astype(dt) if np.issubdtype(dt, np.floating) else \
            rng.integers(0, 200, (N, M)).astype(dt)
        p = str(tmp_path / f"x_{np.dtype(dt).name}.mda")
        mdaio.writemda(X.T, p)
        got = _read(driver, tmp_path, p, "f32", 17, 1000, M)
        np.testing.assert_array_equal(got, X[17:1017].astype(np.float32))
    # int16 stays int16
    X16 = rng.integers(-30000, 30000, (N, M)).astype(np.int16)
    p = str(tmp_path / "x16.mda")
    mdaio.writemda(X16.T, p)
    np.testing.assert_array_equal(_read(driver, tmp_path, p, "i16", 2000, 1001, M), X16[2000:3001])
    assert _run(driver, "info", p).stdout.split() == [str(M), str(N), "-4"]
    # float32 data cannot be read as int16; reads past the end fail
    p32 = str(tmp_path / "x_float32.mda")
    assert _run(driver, "read", p32, "i16", 0, 10, tmp_path / "o.bin").returncode != 0
    assert _run(driver, "read", p32, "f32", 3000, 2, tmp_path / "o.bin").returncode != 0


def test_large_block_read_by_threads(driver, tmp_path):
    # 96 MB: read in several parts by threads
    M, N = 64, 400_000
    X = np.arange(M * N, dtype=np.float32).reshape(N, M)
    p = str(tmp_path / "big.mda")
    mdaio.writemda(X.T, p)
    got = _read(driver, tmp_path, p, "f32", 1, N - 1, M)
    np.testing.assert_array_equal(got, X[1:])


def test_directory_rows_span_files(driver, tmp_path):
    rng = np.random.default_rng(1)
    M = 3
    d = tmp_path / "parts"
    d.mkdir()
    parts = [rng.standard_normal((n, M)).astype(np.float32) for n in (100, 1, 250)]
    for k, P in enumerate(parts):
        mdaio.writemda((P.astype(np.float64) if k == 1 else P).T, str(d / f"p{k}.mda"))
    X = np.concatenate(parts)
    assert _run(driver, "info", d).stdout.split() == ["3", "351", "0"]  # mixed types
    np.testing.assert_array_equal(_read(driver, tmp_path, d, "f32", 90, 200, M), X[90:290])


@pytest.mark.parametrize("dt", ["f32", "i16"])
def test_block_writer_preallocates_and_renames(driver, tmp_path, dt):
    M, N = 4, 50
    npdt = np.int16 if dt == "i16" else np.float32
    blk = (np.arange(10 * M) + 1).astype(npdt).reshape(10, M)
    src = tmp_path / "blk.bin"
    blk.tofile(src)
    out = str(tmp_path / f"out_{dt}.mda")
    r = _run(driver, "write", out, dt, M, N, 20, src)
    assert r.returncode == 0, r.stderr
    assert not os.path.exists(out + ".tmp")
    Y = mdaio.readmda(out).T
    assert Y.dtype == npdt and Y.shape == (N, M)
    np.testing.assert_array_equal(Y[20:30], blk)
    assert not Y[:20].any() and not Y[30:].any()
    # without commit the .tmp file is removed and nothing is renamed
    gone = str(tmp_path / f"gone_{dt}.mda")
    assert _run(driver, "write", gone, dt, M, N, 0, src, "abort").returncode == 0
    assert not os.path.exists(gone) and not os.path.exists(gone + ".tmp")
    # a block past the end is refused
    assert _run(driver, "write", str(tmp_path / "bad.mda"), dt, M, N, 45, src).returncode != 0
