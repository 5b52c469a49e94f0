"""The register DFTs of mountainsort_b200/csrc/fft_reg.cuh run on the CPU.

RegDft<N, INV> and the compile-time twiddle tables are __host__ __device__,
so tests/cpp/regdft_driver.cu compiles the same header for the host (nvcc,
no GPU needed) and runs it on seeded complex vectors.  Checked against
numpy's FFT in FP64: every size the bandpass kernels unroll (16 and 30 for
the 480-point column passes, 20 and 25 for the 500-point row pass) and the
butterflies and composite steps they are built from, both directions; and
the twiddle tables (Taylor series in double, reduced to an octant, rounded
once to float) against the correctly rounded float of cos / sin."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mountainsort_b200", "csrc")
SIZES = [2, 3, 4, 5, 8, 15, 16, 20, 25, 30]


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    nvcc = shutil.which("nvcc") or ("/usr/local/cuda/bin/nvcc" if os.path.exists("/usr/local/cuda/bin/nvcc") else None)
    if nvcc is None:
        pytest.skip("nvcc not available")
    exe = str(tmp_path_factory.mktemp("regdft") / "regdft_driver")
    r = subprocess.run([nvcc, "-O2", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-I", CSRC,
                        os.path.join(ROOT, "tests", "cpp", "regdft_driver.cu"), "-o", exe],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    return exe


def _dft(driver, tmp_path, z, inv):
    count, n = z.shape
    src, dst = tmp_path / "in.bin", tmp_path / "out.bin"
    np.ascontiguousarray(z, np.complex64).tofile(src)
    r = subprocess.run([driver, "dft", str(n), str(int(inv)), str(src), str(dst), str(count)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    return np.fromfile(dst, np.complex64).reshape(count, n)


@pytest.mark.parametrize("n", SIZES)
@pytest.mark.parametrize("inv", [False, True])
def test_register_dft_matches_numpy(driver, tmp_path, n, inv):
    rng = np.random.default_rng(n * 2 + inv)
    z = (rng.standard_normal((3000, n)) + 1j * rng.standard_normal((3000, n))).astype(np.complex64)
    got = _dft(driver, tmp_path, z, inv).astype(np.complex128)
    zz = z.astype(np.complex128)
    want = np.fft.ifft(zz, axis=1) * n if inv else np.fft.fft(zz, axis=1)
    err = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
    # FP32 butterflies: a few units of 2^-24 per stage
    assert err.max() <= 1e-6, err.max()
    assert np.median(err) <= 2.5e-7, np.median(err)


def test_inverse_undoes_forward(driver, tmp_path):
    rng = np.random.default_rng(3)
    for n in (20, 25, 16, 30):
        z = (rng.standard_normal((500, n)) + 1j * rng.standard_normal((500, n))).astype(np.complex64)
        back = _dft(driver, tmp_path, _dft(driver, tmp_path, z, False), True) / n
        assert np.abs(back - z).max() <= 2e-6 * np.abs(z).max()


@pytest.mark.parametrize("n", [15, 16, 20, 25, 30])
def test_twiddle_tables_are_correctly_rounded(driver, tmp_path, n):
    out = tmp_path / "roots.bin"
    r = subprocess.run([driver, "roots", str(n), str(out)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    t = np.fromfile(out, np.float32).reshape(n, 2)
    a = 2 * np.pi * np.arange(n) / n
    for got, want in ((t[:, 0], np.cos(a)), (t[:, 1], -np.sin(a))):
        # correctly rounded: within half a float ulp of the FP64 value (whose own
        # error, ~1e-16, is what separates an exact zero from sin(pi) in FP64)
        half_ulp = 0.5 * np.spacing(np.abs(got))
        assert np.all(np.abs(got.astype(np.float64) - want) <= half_ulp + 1e-15)
    # the quarter turns are exact
    q = np.arange(0, n, n // 4) if n % 4 == 0 else np.array([0])
    assert set(np.abs(t[q]).ravel().tolist()) <= {0.0, 1.0}
