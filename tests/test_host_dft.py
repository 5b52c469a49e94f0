"""The bandpass plan's FP64 host transforms (mountainsort_b200/csrc/host_dft.h)
run on the CPU through tests/cpp/host_dft_driver.cpp and checked against
numpy's FFT: the mixed-radix path (every prime factor at most 64) and
Bluestein's chirp-z path (a larger prime factor), including the window
lengths that need it (466033, a prime: 6 channels at 16 threads; 1398101 =
23 * 89 * 683: 4 channels at 8 threads), and the 5-smooth length rule the
padded plans and Bluestein's convolution use."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mountainsort_b200", "csrc")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = str(tmp_path_factory.mktemp("hostdft") / "host_dft_driver")
    r = subprocess.run([gxx, "-O2", "-std=c++17", "-I", CSRC, os.path.join(ROOT, "tests", "cpp", "host_dft_driver.cpp"),
                        "-o", exe], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return exe


def _dft(driver, tmp_path, x, s):
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    np.ascontiguousarray(x, np.complex128).tofile(src)
    r = subprocess.run([driver, "dft", str(s), str(src), str(dst)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return np.fromfile(dst, np.complex128)


@pytest.mark.parametrize("n", [1, 2, 7, 64, 97, 480, 500, 1009, 3410, 240000, 466033, 1398101])
@pytest.mark.parametrize("s", [-1, 1])
def test_host_dft_matches_numpy(driver, tmp_path, n, s):
    rng = np.random.default_rng(n + (s > 0))
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    got = _dft(driver, tmp_path, x, s)
    want = np.fft.fft(x) if s < 0 else np.fft.ifft(x) * n
    err = np.linalg.norm(got - want) / np.linalg.norm(want)
    assert err <= 1e-13, (n, s, err)


def test_real_even_kernel_stays_real_and_even(driver, tmp_path):
    # the padded plans transform real even taps: the spectrum must be real and even
    n = 466033
    rng = np.random.default_rng(4)
    g = np.zeros(n)
    g[: n // 2 + 1] = rng.standard_normal(n // 2 + 1)
    g[n // 2 + 1:] = g[1: n - n // 2][::-1]
    G = _dft(driver, tmp_path, g.astype(np.complex128), -1)
    assert np.abs(G.imag).max() <= 1e-10 * np.abs(G.real).max()
    assert np.abs(G[1:] - G[1:][::-1]).max() <= 1e-10 * np.abs(G).max()


def test_next_smooth5(driver):
    def smooth(n):
        r = subprocess.run([driver, "smooth", str(n)], capture_output=True, text=True, timeout=60)
        assert r.returncode == 0
        return int(r.stdout)

    for n in [1, 7, 11, 97, 931, 932065, 2796201, 480001]:
        m = smooth(n)
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        assert m >= n and k == 1
        assert all(not _is_smooth(j) for j in range(n, m))


def _is_smooth(j):
    for p in (2, 3, 5):
        while j % p == 0:
            j //= p
    return j == 1
