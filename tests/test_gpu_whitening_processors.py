"""ms3.compute_whitening_matrix, ms3.apply_whitening_matrix and
ms3.whiten_clips on the GPU (through the C ABI and the executable) against
the oracle (ref32, p_whiten.cpp:208-417).

Gates:
  * W from compute_whitening_matrix vs ref32's: relative <= 1e-6.  Both run
    the same power iteration on XXt matrices that differ by ~1e-9 (FP32 runs
    of 32 timepoints here, float products summed in double there); W moves by
    about that much times the iteration's sensitivity at these small M.
  * whitened timeseries / clips vs ref32 with the same W: relative L2 <= 1e-5
    (plain FP32 form); int16 outputs identical except at truncation
    boundaries (differences of at most 1).
"""
import os
import subprocess

import numpy as np
import pytest

from mountainsort_b200 import api, mdaio, synth
from oracle import oracle64 as o64

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "mountainsort_b200", "ms3gpu.mp")


def rel(a, b):
    return o64.rel_l2(a, b)


@pytest.fixture(scope="module")
def recs():
    A = synth.generate_numpy(16, 150000, K=8, seed=11)
    B = synth.generate_numpy(16, 90001, K=8, seed=12)
    return A, B


def test_compute_whitening_matrix_list_and_channels(gpu_lib, ref32, recs):
    A, B = recs
    ch = [3, 1, 16, 7, 9, 2]
    W = api.compute_whitening_matrix([A, B], channels=ch)
    W_ref, C_ref = ref32.compute_whitening_matrix([A, B], channels=ch)
    assert W.shape == (len(ch), len(ch))
    assert rel(W, W_ref) <= 1e-6
    np.testing.assert_allclose(W, W.T, rtol=0, atol=1e-12 * np.abs(W).max())
    # the same as whitening the concatenated channel subset with the stage entry points
    X = np.ascontiguousarray(np.concatenate([A, B])[:, [c - 1 for c in ch]])
    W2 = api.whitening_matrix(api.whiten_covariance(X))
    assert rel(W, W2) <= 1e-9


def test_compute_whitening_matrix_all_channels_device_inputs(gpu_lib, ref32, recs):
    import torch

    A, B = recs
    W = api.compute_whitening_matrix([torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()])
    assert isinstance(W, torch.Tensor) and W.is_cuda
    W_ref, _ = ref32.compute_whitening_matrix([A, B])
    assert rel(W.cpu().numpy(), W_ref) <= 1e-6
    # applied to the recording it gives the oracle's whitened output
    X = np.concatenate([A, B])
    pre = api.apply_whitening_matrix(X, W.cpu().numpy())
    assert rel(pre, ref32.whiten_apply(X, W_ref)) <= 1e-5


def test_compute_whitening_matrix_rejects_bad_channels(gpu_lib, recs):
    from mountainsort_b200 import _lib

    with pytest.raises(_lib.Ms3GpuError):
        api.compute_whitening_matrix([recs[0]], channels=[17])


def test_whiten_clips_parity(gpu_lib, ref32, recs):
    A, _ = recs
    W_ref, _ = ref32.compute_whitening_matrix([A])
    # clips: (L, T, M) = 300 clips of 50 timepoints cut from the recording
    clips = np.ascontiguousarray(A[: 300 * 50].reshape(300, 50, 16))
    got = api.whiten_clips(clips, W_ref)
    ref = ref32.whiten_clips(clips, W_ref)
    assert got.shape == clips.shape and got.dtype == np.float32
    assert rel(got, ref) <= 1e-5  # gate: plain FP32 form, no 1e-4 rounding
    exact = np.einsum("ltm,mk->ltk", clips.astype(np.float64), W_ref)
    assert rel(api.whiten_clips(clips, W_ref, precision="mixed"), exact) <= 1e-4
    q = 0.05
    got16 = api.whiten_clips(clips, W_ref, quantization_unit=q)
    ref16 = ref32.whiten_clips(clips, W_ref, quantization_unit=q)
    assert got16.dtype == np.int16
    d = np.abs(got16.astype(np.int32) - ref16.astype(np.int32))
    assert d.max() <= 1 and np.mean(d) < 1e-3


def _run(*args):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=600)


def test_processors_end_to_end(gpu_lib, ref32, recs, tmp_path):
    A, B = recs
    pa, pb = str(tmp_path / "a.mda"), str(tmp_path / "b.mda")
    mdaio.writemda(A.T, pa)
    mdaio.writemda(B.T, pb)
    pw = str(tmp_path / "w.mda")
    r = _run("ms3.compute_whitening_matrix", f"--timeseries_list={pa}", "--timeseries_list", pb, "--channels=2,4,6,8",
             f"--whitening_matrix_out={pw}")
    assert r.returncode == 0, r.stderr
    Wf = mdaio.readmda(pw)
    assert Wf.dtype == np.float64 and Wf.shape == (4, 4)
    W_ref, _ = ref32.compute_whitening_matrix([A, B], channels=[2, 4, 6, 8])
    assert rel(Wf, W_ref) <= 1e-6

    # apply a full 16 x 16 matrix, written as float64 like compute_whitening_matrix writes it
    W16, _ = ref32.compute_whitening_matrix([A])
    pw16 = str(tmp_path / "w16.mda")
    mdaio.writemda(W16, pw16, dtype="float64")
    po = str(tmp_path / "pre.mda")
    r = _run("ms3.apply_whitening_matrix", f"--timeseries={pa}", f"--whitening_matrix={pw16}",
             f"--timeseries_out={po}")
    assert r.returncode == 0, r.stderr
    P = mdaio.readmda(po)
    assert P.dtype == np.float32
    assert rel(P.T, ref32.whiten_apply(A, W16)) <= 1e-5
    po16 = str(tmp_path / "pre16.mda")
    r = _run("ms3.apply_whitening_matrix", f"--timeseries={pa}", f"--whitening_matrix={pw16}",
             f"--timeseries_out={po16}", "--quantization_unit=0.01")
    assert r.returncode == 0, r.stderr
    P16 = mdaio.readmda(po16)
    assert P16.dtype == np.int16
    ref16 = ref32.float_to_int16(ref32.whiten_apply(A[:20000], W16, quantization_unit=0.01))
    d = np.abs(P16.T[:20000].astype(np.int32) - ref16.astype(np.int32))
    assert d.max() <= 1 and np.mean(d) < 1e-3

    # clips M x T x L
    clips = np.ascontiguousarray(A[: 200 * 40].reshape(200, 40, 16))
    pc, pco = str(tmp_path / "clips.mda"), str(tmp_path / "clips_out.mda")
    mdaio.writemda(clips.transpose(2, 1, 0), pc)
    r = _run("ms3.whiten_clips", f"--clips={pc}", f"--whitening_matrix={pw16}", f"--clips_out={pco}")
    assert r.returncode == 0, r.stderr
    Co = mdaio.readmda(pco)
    assert Co.shape == (16, 40, 200) and Co.dtype == np.float32
    assert rel(Co.transpose(2, 1, 0), ref32.whiten_clips(clips, W16)) <= 1e-5
    # a wrong-sized matrix is an error and leaves no output
    bad = str(tmp_path / "bad_out.mda")
    r = _run("ms3.whiten_clips", f"--clips={pc}", f"--whitening_matrix={pw}", f"--clips_out={bad}")
    assert r.returncode == 255 and not os.path.exists(bad)
