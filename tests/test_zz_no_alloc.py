"""ms3gpu_whiten_covariance_noalloc: whiten pass 1 without any allocation.

This entry point is for callers that cannot let the library call cudaMalloc
-- applications that give the whole GPU to their own memory pool before
processing starts, and streaming loops that must not stall on a device
allocation.  It keeps its partial sums in a fixed 16 MiB array inside the
library's device image.  These tests call it through the C ABI with device
buffers and compare it, on two calls in a row, with the allocating entry
point (ms3gpu_whiten_covariance) and with the oracle's covariance pass on the
same input, both within 1e-8 relative, the covariance tolerance of the other
tests (from 128 channels on the allocating entry point sums on the tensor
cores with its own exact-integer arithmetic, so the two are not bit-equal).  The call
only queues its work on the stream, so the tests read the result after the
stream has reached it.  The file sorts last so that a run stopping at its
first failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from mountainsort_b200 import _lib, api, synth
from oracle import oracle64 as o64

pytestmark = pytest.mark.gpu


def _noalloc(L, X, out, stream):
    N, M = X.shape
    return L.ms3gpu_whiten_covariance_noalloc(X.data_ptr(), M, N, out.data_ptr(), stream)


@pytest.mark.parametrize("M,N", [(64, 200000), (384, 60000)])
def test_noalloc_covariance_matches_allocating_entry_point(gpu_lib, ref32, M, N):
    import torch

    L = gpu_lib
    Xh = synth.generate_numpy(M, N, K=4, seed=M)
    X = torch.from_numpy(Xh).cuda()
    ref = api.whiten_covariance(X).cpu().numpy()  # allocating entry point, matrix notation
    oracle = ref32.whiten_xxt(Xh)  # the oracle's pass 1 (float products summed in double)
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):  # the second call runs on the array the first one left behind
        out = torch.full((M, M), float("nan"), dtype=torch.float64, device="cuda")
        assert _noalloc(L, X, out, stream) == _lib.OK, _lib.last_error()
        torch.cuda.current_stream().synchronize()  # the call returns before its work is done
        got = out.cpu().numpy().T  # column-major buffer -> matrix notation
        assert np.all(np.isfinite(got))
        assert o64.rel_l2(got, ref) <= 1e-8
        assert o64.rel_l2(got, oracle) <= 1e-8
        np.testing.assert_array_equal(got, got.T)


def test_noalloc_covariance_rejects_what_it_cannot_do_without_allocating(gpu_lib):
    import torch

    L = gpu_lib
    Xh = np.zeros((100, 8), np.float32)
    out = torch.zeros((8, 8), dtype=torch.float64, device="cuda")
    # host input would need a staging allocation
    rc = L.ms3gpu_whiten_covariance_noalloc(Xh.ctypes.data, 8, 100, out.data_ptr(), None)
    assert rc == _lib.ERR_INVALID and "device memory" in _lib.last_error()
    # more channels than the fixed scratch holds
    big = torch.zeros((2, 2048), dtype=torch.float32, device="cuda")
    out2 = torch.zeros((2048, 2048), dtype=torch.float64, device="cuda")
    rc = L.ms3gpu_whiten_covariance_noalloc(big.data_ptr(), 2048, 2, out2.data_ptr(), None)
    assert rc == _lib.ERR_INVALID and "1984" in _lib.last_error()
