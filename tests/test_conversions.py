"""The integer conversions of the int16 outputs (mountainsort_b200/csrc/common.cuh:
x86_float_to_int16, x86_double_to_int32; __host__ __device__, the same source
the GPU's output stores use), run on the CPU through tests/cpp/conv_driver.cu.

The reference writes int16 outputs with std::copy from float
(packages/ms3/mda/mdaio.cpp:232-243) and scales with (int)(x / q + 0.5)
(p_whiten.cpp, p_bandpass_filter.cpp), which on x86-64 are cvttss2si /
cvttsd2si: truncation toward zero, 0x80000000 for NaN and out-of-range
values, and for int16 the low 16 bits.  The GPU has no such instruction
(its conversions saturate), so the product spells the rule out; here it is
checked against the x86 instructions themselves (numpy's casts on this
host) and the known answers the oracle's own test pins."""
import os
import platform
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mountainsort_b200", "csrc")

x86 = pytest.mark.skipif(platform.machine() not in ("x86_64", "AMD64"),
                         reason="numpy's casts follow the x86 conversion instructions only on x86-64")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)
    if nvcc is None:
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("conv") / "conv_driver")
    r = subprocess.run([nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-I", os.path.join(ROOT, "include"), "-I", CSRC,
                        os.path.join(ROOT, "tests", "cpp", "conv_driver.cu"), "-o", exe],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return exe


def _run(driver, tmp_path, mode, x, out_dtype):
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    x.tofile(src)
    r = subprocess.run([driver, mode, str(src), str(dst)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return np.fromfile(dst, out_dtype)


def _floats(rng, n):
    x = (rng.standard_normal(n) * np.exp(rng.uniform(0, 25, n))).astype(np.float32)
    edges = np.array([0.0, -0.0, 0.5, -0.5, 0.999999, -0.999999, 32767.0, 32767.99, 32768.0, -32768.0,
                      -32768.99, -32769.0, 65535.0, 65536.0, 2147483520.0, 2147483648.0, -2147483648.0,
                      -2147483904.0, 3e9, -3e9, 1e38, -1e38, np.inf, -np.inf, np.nan, 1e-45], np.float32)
    return np.concatenate([edges, x])


def test_known_answers(driver, tmp_path):
    v = np.array([1.9, -1.9, 32767.5, 32768.0, -32769.0, 70000.0, 3e9, np.nan], np.float32)
    got = _run(driver, tmp_path, "f2i16", v, np.int16)
    np.testing.assert_array_equal(got, np.array([1, -1, 32767, -32768, 32767, 4464, 0, 0], np.int16))


@x86
def test_float_to_int16_is_the_x86_conversion(driver, tmp_path):
    x = _floats(np.random.default_rng(0), 400000)
    got = _run(driver, tmp_path, "f2i16", x, np.int16)
    with np.errstate(invalid="ignore"):
        want = x.astype(np.int32).astype(np.int16)  # cvttss2si, then the low 16 bits
    np.testing.assert_array_equal(got, want)


@x86
def test_double_to_int32_is_the_x86_conversion(driver, tmp_path):
    rng = np.random.default_rng(1)
    d = rng.standard_normal(400000) * np.exp(rng.uniform(0, 25, 400000))
    edges = np.array([0.0, -0.0, 0.5, -0.5, 2147483647.0, 2147483647.9, 2147483648.0, -2147483648.0,
                      -2147483648.9, -2147483649.0, 1e300, -1e300, np.inf, -np.inf, np.nan, 5e-324])
    d = np.concatenate([edges, d])
    got = _run(driver, tmp_path, "d2i32", d, np.int32)
    with np.errstate(invalid="ignore"):
        want = d.astype(np.int32)  # cvttsd2si
    np.testing.assert_array_equal(got, want)
    for v in (1e300, -2147483649.0, np.nan):  # 0x80000000, not saturated
        assert got[int(np.flatnonzero((edges == v) | (np.isnan(edges) & np.isnan(v)))[0])] == np.iinfo(np.int32).min
