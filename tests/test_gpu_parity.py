"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Gates (written in each test):
  * filtered output vs ref32: relative L2 <= 1e-5 (plain FP32 form);
  * whitened output vs ref32: relative L2 <= 1e-5 (it is rounded to 1e-4, so
    differences are whole rounding steps at rounding boundaries);
  * covariance and whitening matrix vs the oracle: relative <= 1e-8 / 1e-10;
  * int16 outputs: identical except at truncation boundaries.
"""
import ctypes
import os
import subprocess
import sys

import numpy as np
import pytest

from mountainsort_b200 import _lib, api, mdaio, synth
from oracle import oracle64 as o64

pytestmark = pytest.mark.gpu

FS, FMIN, FMAX, FWID = 30000.0, 300.0, 6000.0, 1000.0
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def rel(a, b):
    return o64.rel_l2(a, b)


@pytest.fixture(scope="module")
def rec32():
    return synth.generate_numpy(32, 360000, K=12, seed=0, sites=(3, 6))


# (M, N, T): T chosen to exercise the canonical L = 240000 and odd windows
BP_CASES = [
    (32, 360000, 16),   # L = 240000, 3 whole chunks
    (12, 250000, 16),   # L = 240000, last chunk partial
    (7, 1000, 27),      # N shorter than one chunk, odd M (last pair padded)
    (1, 5000, 187),     # a single channel
    (3, 130000, 63),    # odd M
    (4, 150000, 16),    # L = 699050 = 2*5^2*11*31*41: generic radices
    (64, 240000, 16),   # 2 groups of 16 channel pairs
]


@pytest.mark.parametrize("M,N,T", BP_CASES)
def test_bandpass_parity(gpu_lib, ref32, M, N, T):
    X = synth.generate_numpy(M, N, K=max(1, M // 3), seed=M + N, sites=(1, min(M, 4)))
    ref = ref32.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=T)
    got = api.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=T)
    assert got.shape == ref.shape and got.dtype == np.float32
    assert rel(got, ref) <= 1e-5  # gate: plain FP32 form
    assert rel(got, ref) <= 2e-6  # what accurate FP32 FFTs give


def test_bandpass_generic_path_matches_register_path(gpu_lib, ref32, rec32):
    # L = 240000 runs the register-pass kernels; MS3GPU_BP_GENERIC=1 forces the
    # generic shared-memory Stockham kernels on the same window (fresh plan:
    # a different freq_wid keys a new plan).
    ref = ref32.bandpass_filter(rec32, FS, FMIN, FMAX, 999.0, num_threads=16)
    fast = api.bandpass_filter(rec32, FS, FMIN, FMAX, 999.0, num_threads=16)
    os.environ["MS3GPU_BP_GENERIC"] = "1"
    try:
        gen = api.bandpass_filter(rec32, FS, FMIN, FMAX, 998.0, num_threads=16)
    finally:
        del os.environ["MS3GPU_BP_GENERIC"]
    ref2 = ref32.bandpass_filter(rec32, FS, FMIN, FMAX, 998.0, num_threads=16)
    assert rel(fast, ref) <= 2e-6
    assert rel(gen, ref2) <= 2e-6


def test_bandpass_device_pointers_and_determinism(gpu_lib, rec32):
    import torch

    Xd = torch.from_numpy(rec32).cuda()
    a = api.bandpass_filter(Xd, FS, FMIN, FMAX, FWID, num_threads=16)
    b = api.bandpass_filter(Xd, FS, FMIN, FMAX, FWID, num_threads=16)
    h = api.bandpass_filter(rec32, FS, FMIN, FMAX, FWID, num_threads=16)
    assert a.is_cuda
    assert torch.equal(a, b)
    np.testing.assert_array_equal(a.cpu().numpy(), h)


def test_fused_call_repeats_bit_for_bit_at_16_channels(gpu_lib):
    """16 channels: the apply's 128-channel tiles have three wholly clipped
    32-column blocks per row, which are neither staged nor stored; repeated
    calls must give the same bits (a staging buffer reused while its store
    still reads it would not)."""
    import torch

    X = torch.from_numpy(synth.generate_numpy(16, 200_000, K=4, seed=16)).cuda()
    ref = api.bandpass_whiten(X, FS, FMIN, FMAX, FWID, num_threads=16)
    for _ in range(6):
        assert torch.equal(api.bandpass_whiten(X, FS, FMIN, FMAX, FWID, num_threads=16), ref)


def test_bandpass_no_lowcut(gpu_lib, ref32):
    X = synth.generate_numpy(16, 200000, K=3, seed=11)
    ref = ref32.bandpass_filter(X, FS, 0.0, FMAX, FWID, num_threads=16)
    got = api.bandpass_filter(X, FS, 0.0, FMAX, FWID, num_threads=16)
    assert rel(got, ref) <= 1e-5


@pytest.mark.parametrize("q", [0.5, 2.0])
def test_bandpass_int16(gpu_lib, ref32, rec32, q):
    ref = ref32.bandpass_filter(rec32, FS, FMIN, FMAX, FWID, quantization_unit=q, num_threads=16)
    got = api.bandpass_filter(rec32, FS, FMIN, FMAX, FWID, quantization_unit=q, num_threads=16)
    assert got.dtype == np.int16 and got.shape == ref.shape
    d = np.abs(got.astype(np.int32) - ref.astype(np.int32))
    assert d.max() <= 1  # truncation boundaries only
    assert np.mean(d) < 1e-4


@pytest.mark.parametrize("sub", [3, 7])
def test_bandpass_subsample(gpu_lib, ref32, sub):
    X = synth.generate_numpy(10, 250000, K=3, seed=5)
    ref = ref32.bandpass_filter(X, FS, FMIN, FMAX, FWID, subsample_factor=sub, num_threads=19)
    got = api.bandpass_filter(X, FS, FMIN, FMAX, FWID, subsample_factor=sub, num_threads=19)
    assert got.shape == ref.shape
    assert rel(got, ref) <= 1e-5


def test_bandpass_copy_when_freq_max_zero(gpu_lib, rec32):
    got = api.bandpass_filter(rec32[:1000], FS, FMIN, 0.0, FWID, num_threads=16)
    np.testing.assert_array_equal(got, rec32[:1000])


@pytest.mark.parametrize("M", [8, 32, 64, 100])
def test_whiten_stages_parity(gpu_lib, ref32, M):
    X = synth.generate_numpy(M, 120000, K=M // 2, seed=M)
    F = ref32.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=max(16, 187 // M + 1))
    C_ref = ref32.whiten_xxt(F)
    C = api.whiten_covariance(F)
    assert rel(C, C_ref) <= 1e-8
    np.testing.assert_array_equal(C, C.T)
    W_ref, comps_ref, sig_ref = ref32.whitening_matrix(C_ref)
    W, comps, sig = api.whitening_matrix(C_ref, return_components=True)
    assert rel(W, W_ref) <= 1e-10
    assert rel(sig, sig_ref) <= 1e-10
    pre_ref, _, _ = ref32.whiten(F)
    pre = api.whiten(F)
    assert rel(pre, pre_ref) <= 1e-5  # gate
    # values are multiples of 1e-4 like the reference's
    assert np.max(np.abs(pre.astype(np.float64) * 1e4 - np.round(pre.astype(np.float64) * 1e4))) < 1e-2


def _cov(M, seed):
    rng = np.random.default_rng(seed)
    A = np.eye(M) + 0.3 * rng.standard_normal((M, M)) / np.sqrt(M)
    return A @ A.T * 37.0


def test_whitening_matrix_m500_cluster16(gpu_lib):
    # 500 channels: rows in a 16-CTA cluster's shared memory.  The reference's
    # 10-step power iteration moves W by ~8e-10 under 1e-15 perturbations of
    # XXt at this size, so FP64 reorderings agree to ~1e-9.
    C = _cov(500, 500)
    W64, _, sig64 = o64.whitening_matrix(C)
    W, comps, sig = api.whitening_matrix(C, return_components=True)
    assert rel(W, W64) <= 1e-8
    assert rel(sig, sig64) <= 1e-8


@pytest.mark.parametrize("M", [1, 2, 31, 33, 100, 128, 129, 200, 256, 257, 300, 383, 384])
def test_whitening_matrix_register_kernel_matches_shared(gpu_lib, M):
    # Up to 384 channels the working matrix lives in registers and every
    # norm is formed per warp; the sums keep the shared-memory kernel's order,
    # so components, sigma and W are bit-identical to it.
    C = _cov(M, M + 7)
    W_r, comps_r, sig_r = api.whitening_matrix(C, return_components=True)
    os.environ["MS3GPU_PCA_KERNEL"] = "smem"
    try:
        W_s, comps_s, sig_s = api.whitening_matrix(C, return_components=True)
    finally:
        del os.environ["MS3GPU_PCA_KERNEL"]
    np.testing.assert_array_equal(sig_r, sig_s)
    np.testing.assert_array_equal(comps_r, comps_s)
    np.testing.assert_array_equal(W_r, W_s)


@pytest.mark.parametrize("M", [384, 700])
def test_whitening_matrix_global_rows_match_shared(gpu_lib, M):
    # The global-memory variant (rows that do not fit shared memory) runs the
    # same arithmetic in the same order: bit-identical to the shared-memory
    # variant at 384; at 700 (where it is the only variant) it is compared with
    # the FP64 oracle within the algorithm's own sensitivity there (a 1e-15
    # perturbation of XXt moves W by ~2e-4: the 10-step iteration does not
    # converge for the late, nearly degenerate components).
    C = _cov(M, M)
    if M == 384:
        W_s = api.whitening_matrix(C)
        os.environ["MS3GPU_PCA_ROWS_GLOBAL"] = "1"
        try:
            W_g = api.whitening_matrix(C)
        finally:
            del os.environ["MS3GPU_PCA_ROWS_GLOBAL"]
        np.testing.assert_array_equal(W_g, W_s)
        W64, _, _ = o64.whitening_matrix(C)
        assert rel(W_s, W64) <= 1e-8
    else:
        W64, _, sig64 = o64.whitening_matrix(C)
        W, _, sig = api.whitening_matrix(C, return_components=True)
        assert rel(W, W64) <= 2e-3
        assert rel(sig, sig64) <= 2e-4
        np.testing.assert_allclose(W, W.T, rtol=0, atol=1e-12 * np.abs(W).max())


def test_apply_plain_and_mixed_at_384(gpu_lib, ref32):
    # 384 channels (the benchmark's shape).  Plain form (FP32 FMA): within
    # 1e-5 of ref32's apply.  Mixed form (tcgen05, 3-term TF32, FP32
    # accumulation in TMEM): within 1e-4 of the FP64 apply.
    M, N = 384, 20000
    X = synth.generate_numpy(M, N, K=40, seed=384, sites=(6, 12))
    C = o64.xxt(X)
    W, _, _ = o64.whitening_matrix(C)
    ref = ref32.whiten_apply(X, W)
    exact = o64.quantize(X.astype(np.float64) @ W)
    plain = api.apply_whitening_matrix(X, W)  # tcgen05 with drained accumulators
    mixed = api.apply_whitening_matrix(X, W, precision="mixed")
    os.environ["MS3GPU_APPLY_FFMA"] = "1"
    try:
        ffma = api.apply_whitening_matrix(X, W)
    finally:
        del os.environ["MS3GPU_APPLY_FFMA"]
    e_plain, e_ffma = rel(plain, ref), rel(ffma, ref)
    e_mixed, e_mixed64 = rel(mixed, ref), rel(mixed, exact)
    print(f"apply rel L2 vs ref32: plain tensor-core {e_plain:.3e}, plain FMA {e_ffma:.3e}, "
          f"mixed {e_mixed:.3e} (mixed vs FP64 {e_mixed64:.3e})")
    assert e_plain <= 1e-5
    assert e_ffma <= 1e-5
    assert e_mixed64 <= 1e-4


def test_mixed_pipeline_vs_fp64_oracle(gpu_lib, rec32):
    # the mixed-precision form on the 32ch x 1.8M geometry, gated against the FP64 oracle
    pre = api.bandpass_whiten(rec32, FS, FMIN, FMAX, FWID, num_threads=16, precision="mixed")
    y, q64, _, _ = o64.whiten(o64.bandpass_filter(rec32, FS, FMIN, FMAX, FWID, num_threads=16))
    err = rel(pre, q64)
    print(f"mixed pipeline rel L2 vs FP64 oracle {err:.3e}, max-abs {np.max(np.abs(pre - q64)):.3e}")
    assert err <= 1e-4


def test_whiten_int16(gpu_lib, ref32, rec32):
    F = ref32.bandpass_filter(rec32, FS, FMIN, FMAX, FWID, num_threads=16)
    ref, _, _ = ref32.whiten(F, quantization_unit=0.01)
    got = api.whiten(F, quantization_unit=0.01)
    assert got.dtype == np.int16
    d = np.abs(got.astype(np.int32) - ref.astype(np.int32))
    assert d.max() <= 1 and np.mean(d) < 1e-3


def test_fused_pipeline_32ch_geometry(gpu_lib, ref32, rec32):
    """ms3.bandpass_filter then ms3.whiten, as mountainsort3.mlp runs them."""
    filt_ref = ref32.bandpass_filter(rec32, FS, FMIN, FMAX, FWID, num_threads=16)
    pre_ref, _, _ = ref32.whiten(filt_ref)
    filt, pre = api.bandpass_whiten(rec32, FS, FMIN, FMAX, FWID, num_threads=16, want_filt=True)
    assert rel(filt, filt_ref) <= 1e-5
    assert rel(pre, pre_ref) <= 1e-5
    pre_only = api.bandpass_whiten(rec32, FS, FMIN, FMAX, FWID, num_threads=16)
    np.testing.assert_array_equal(pre_only, pre)
    # against the FP64 oracle too (the floor of the FP32 forms)
    y, q64, _, _ = o64.whiten(o64.bandpass_filter(rec32, FS, FMIN, FMAX, FWID, num_threads=16))
    assert rel(pre, q64) <= 1e-4


@pytest.mark.parametrize("M,N,T", [
    (6, 700000, 16),    # L = 466033, a prime: zero-padded to a 5-smooth FFT of >= 2L - 1 points
    (4, 1500000, 8),    # L = 1398101 = 23 * 89 * 683 (tetrodes at 8 threads)
    (5, 300000, 16),    # L = 559240 = 2^3 * 5 * 11 * 31 * 41: factors <= 64, direct
    (3, 400000, 27),    # odd M (the last pair padded), L = 552336 = 2^4 * 3 * 37 * 311: zero-padded
])
def test_bandpass_any_window_length(gpu_lib, ref32, M, N, T):
    X = synth.generate_numpy(M, N, K=2, seed=M * 13 + T)
    ref = ref32.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=T)
    got = api.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=T)
    e = rel(got, ref)
    print(f"M={M} T={T} L={ref32.chunk_size(M, T) + 120000}: rel L2 vs ref32 {e:.3e}")
    assert got.shape == ref.shape
    assert e <= 1e-5  # gate: plain FP32 form
    pre = api.whiten(got)
    pre_ref, _, _ = ref32.whiten(ref)
    assert rel(pre, pre_ref) <= 1e-5


def test_out_of_memory_hook_reports_nomem(gpu_lib):
    code = (
        "import numpy as np, sys; sys.path.insert(0, %r)\n"
        "from mountainsort_b200 import api, _lib\n"
        "try:\n"
        "    api.whiten(np.ones((1000, 4), np.float32))\n"
        "    print('NOERR')\n"
        "except _lib.Ms3GpuError as e:\n"
        "    print('CODE', e.code)\n"
        "api_ok = True\n" % ROOT)
    env = dict(os.environ, MS3GPU_FAIL_ALLOC_AFTER="0")
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, env=env, timeout=300)
    assert "CODE %d" % _lib.ERR_NOMEM in r.stdout, r.stdout + r.stderr


def test_processor_executable_end_to_end(gpu_lib, ref32, tmp_path):
    X = synth.generate_numpy(16, 200000, K=4, seed=21)
    raw = str(tmp_path / "raw.mda")
    mdaio.writemda(X.T, raw)  # M x N column-major
    filt, pre = str(tmp_path / "filt.mda"), str(tmp_path / "pre.mda")
    exe = os.path.join(ROOT, "mountainsort_b200", "ms3gpu.mp")
    r = subprocess.run([exe, "ms3.bandpass_filter", f"--timeseries={raw}", f"--timeseries_out={filt}",
                        "--samplerate=30000", "--freq_min=300", "--freq_max=6000", "--_request_num_threads=16"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([exe, "ms3.whiten", f"--timeseries={filt}", f"--timeseries_out={pre}"],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    F = mdaio.readmda(filt)
    P = mdaio.readmda(pre)
    assert F.shape == (16, 200000) and F.dtype == np.float32
    filt_ref = ref32.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=16)
    pre_ref, _, _ = ref32.whiten(filt_ref)
    assert rel(F.T, filt_ref) <= 1e-5
    assert rel(P.T, pre_ref) <= 1e-5
