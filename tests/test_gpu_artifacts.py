"""ms3.mask_out_artifacts on the GPU vs the oracle (p_mask_out_artifacts.cpp:
24-104).  The interval norms and the per-channel statistics are formed in
double in the reference's order, so the masking decisions -- and with them
the whole output -- are identical to ref32's (gate: bit-for-bit)."""
import os
import subprocess

import numpy as np
import pytest

from mountainsort_b200 import _lib, api, mdaio, synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "mountainsort_b200", "ms3gpu.mp")


def _with_artifacts(M, N, seed):
    X = synth.generate_numpy(M, N, K=max(1, M // 2), seed=seed)
    rng = np.random.default_rng(seed)
    for t in rng.integers(0, N, 6):
        X[t:t + 300, :] += rng.uniform(500, 3000)  # broadband transients on all channels
    X[5, 0] += 5000.0  # one in the first interval
    return X


@pytest.mark.parametrize("M,N,I,thr", [(32, 400037, 2000, 6.0), (7, 120000, 777, 4.0), (64, 100000, 2000, 3.0)])
def test_mask_out_artifacts_matches_oracle(gpu_lib, ref32, M, N, I, thr):
    X = _with_artifacts(M, N, seed=M)
    got, kept = api.mask_out_artifacts(X, threshold=thr, interval_size=I, return_kept=True)
    ref, kept_ref = ref32.mask_out_artifacts(X, threshold=thr, interval_size=I)
    np.testing.assert_array_equal(got, ref)
    assert kept == kept_ref and 0 < kept < (N // I) * I


def test_mask_out_artifacts_device_and_errors(gpu_lib, ref32):
    import torch

    X = _with_artifacts(16, 200000, seed=3)
    got = api.mask_out_artifacts(torch.from_numpy(X).cuda())
    ref, _ = ref32.mask_out_artifacts(X)
    np.testing.assert_array_equal(got.cpu().numpy(), ref)
    with pytest.raises(_lib.Ms3GpuError):
        api.mask_out_artifacts(X, threshold=0)
    with pytest.raises(_lib.Ms3GpuError):
        api.mask_out_artifacts(X, interval_size=0)


def test_mask_out_artifacts_processor(gpu_lib, ref32, tmp_path):
    X = _with_artifacts(32, 300000, seed=9)
    p, o = str(tmp_path / "x.mda"), str(tmp_path / "o.mda")
    mdaio.writemda(X.T, p)
    r = subprocess.run([EXE, "ms3.mask_out_artifacts", f"--timeseries={p}", f"--timeseries_out={o}",
                        "--threshold=5", "--interval_size=1500"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "Using" in r.stdout and "of all timepoints" in r.stdout
    ref, _ = ref32.mask_out_artifacts(X, threshold=5, interval_size=1500)
    np.testing.assert_array_equal(mdaio.readmda(o).T, ref)


def test_mask_out_artifacts_more_intervals_than_a_grid_row(gpu_lib, ref32):
    """More than 65535 intervals (the largest grid y extent): the norm kernel
    strides over them, in memory and in one streamed slab."""
    M, N, I = 1, 140_001, 2  # 70000 intervals
    X = _with_artifacts(M, N, seed=11)
    ref, kept_ref = ref32.mask_out_artifacts(X, threshold=4.0, interval_size=I)
    got, kept = api.mask_out_artifacts(X, threshold=4.0, interval_size=I, return_kept=True)
    np.testing.assert_array_equal(got, ref)
    assert kept == kept_ref and 0 < kept < (N // I) * I
    Y = np.full_like(X, 7.0)

    def source(t0, nt):
        return X[t0:t0 + nt]

    def sink(t0, rows):
        Y[t0:t0 + len(rows)] = rows

    kept_s = api.mask_out_artifacts_stream(source, sink, M, N, 4.0, I)
    assert kept_s == kept_ref
    np.testing.assert_array_equal(Y, ref)
