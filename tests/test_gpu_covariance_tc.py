"""Whiten pass 1 on the tensor cores (the exact int8 digit products of
mountainsort_b200/csrc/cov_i8.cu, used for M >= 128 channels) against the
oracle's pass 1 (p_whiten.cpp:64-118: float products summed in double).

Gate: relative L2 (Frobenius) <= 1e-8 vs ref32, the covariance tolerance of
the other tests; the matrix is exactly symmetric and repeat calls are
bit-identical.  Edge cases: a partial last run and a partial last channel
block, a channel of zeros, a channel of tiny values next to a large
transient, a device buffer that is not 16-byte aligned (the kernel works on
an aligned copy), and a non-finite value (its channel's row and column
become NaN, as the reference's double sums would)."""
import numpy as np
import pytest

from mountainsort_b200 import api, synth
from oracle import oracle64 as o64

pytestmark = pytest.mark.gpu

FS, FMIN, FMAX, FWID = 30000.0, 300.0, 6000.0, 1000.0


def _filtered(M, N, seed):
    X = synth.generate_torch(M, N, K=max(1, M // 3), seed=seed, sites=(6, 12)).cpu().numpy()
    return api.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=16)


@pytest.mark.parametrize("M,N", [(128, 100000), (200, 70001), (384, 120000), (512, 50003)])
def test_tc_covariance_vs_oracle(gpu_lib, ref32, M, N):
    F = _filtered(M, N, seed=M + 7)
    C = api.whiten_covariance(F)
    C_ref = ref32.whiten_xxt(F)
    e = o64.rel_l2(C, C_ref)
    print(f"M={M} N={N}: tensor-core covariance vs ref32 rel L2 {e:.3e}, vs FP64 {o64.rel_l2(C, o64.xxt(F)):.3e}")
    assert e <= 1e-8
    np.testing.assert_array_equal(C, C.T)
    np.testing.assert_array_equal(C, api.whiten_covariance(F))  # deterministic


def test_tc_covariance_awkward_values_and_alignment(gpu_lib, ref32):
    import torch

    M, N = 256, 90000
    F = _filtered(M, N, seed=3)
    F[1000:1050, :] -= 20000.0           # a transient on every channel
    F[:, 5] = 0.0                        # a silent channel
    F[:, 17] *= 1e-6                     # tiny values ...
    F[40000:40300, 17] += 2000.0         # ... with one large transient in their run
    C = api.whiten_covariance(F)
    C_ref = ref32.whiten_xxt(F)
    assert o64.rel_l2(C, C_ref) <= 1e-8
    assert np.all(C[5] == 0) and np.all(C[:, 5] == 0)
    # a device buffer 4 bytes past a 16-byte boundary
    flat = torch.empty(N * M + 1, dtype=torch.float32, device="cuda")
    Xd = flat[1:].view(N, M)
    Xd.copy_(torch.from_numpy(F))
    assert Xd.data_ptr() % 16 != 0
    np.testing.assert_array_equal(api.whiten_covariance(Xd).cpu().numpy(), C)


def test_tc_covariance_non_finite_channel(gpu_lib):
    M, N = 128, 40000
    F = _filtered(M, N, seed=9)
    F[123, 7] = np.inf
    C = api.whiten_covariance(F)
    assert np.all(np.isnan(C[7])) and np.all(np.isnan(C[:, 7]))
    others = np.delete(np.delete(C, 7, axis=0), 7, axis=1)
    assert np.all(np.isfinite(others))
    G = np.delete(F, 7, axis=1)
    assert o64.rel_l2(others, o64.xxt(G)) <= 1e-8
