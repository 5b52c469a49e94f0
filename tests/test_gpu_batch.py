"""ms3gpu_bandpass_whiten_batch: recordings of different channel counts,
lengths and sample rates in one call (the batched uneven workload of the
benchmark configurations, at test size).

Gates: every job's output equals the single-recording call's bit-for-bit
(same kernels, same reduction orders; only the streams differ); outputs vs
ref32 relative L2 <= 1e-5 (plain FP32 form); a failing job reports its own
status and does not stop the others."""
import ctypes

import numpy as np
import pytest

from mountainsort_b200 import _lib, api, synth
from oracle import oracle64 as o64

pytestmark = pytest.mark.gpu


def _recordings():
    rng = np.random.default_rng(1)
    recs = []
    for k, M in enumerate([16, 32, 64, 128, 16, 384]):
        fs = [20000.0, 30000.0][k % 2]
        N = int(rng.integers(100_000, 400_000))
        X = synth.generate_numpy(M, N, K=max(2, M // 4), seed=100 + k)
        recs.append(dict(X=X, samplerate=fs, freq_min=300.0, freq_max=min(6000.0, 0.4 * fs), num_threads=16))
    return recs


def test_batch_equals_single_calls_and_reference(gpu_lib, ref32):
    recs = _recordings()
    outs = api.bandpass_whiten_batch(recs)
    for k, (r, out) in enumerate(zip(recs, outs)):
        single = api.bandpass_whiten(r["X"], r["samplerate"], r["freq_min"], r["freq_max"],
                                     num_threads=r["num_threads"])
        np.testing.assert_array_equal(out, single, err_msg=f"job {k}")
    for k in (0, 3):
        r = recs[k]
        filt = ref32.bandpass_filter(r["X"], r["samplerate"], r["freq_min"], r["freq_max"], 1000.0,
                                     num_threads=r["num_threads"])
        pre_ref, _, _ = ref32.whiten(filt)
        assert o64.rel_l2(outs[k], pre_ref) <= 1e-5


def test_batch_failing_job_is_isolated(gpu_lib):
    L = _lib.load()
    recs = _recordings()[:3]
    jobs = (_lib.Job * 3)()
    keep, outs = [], []
    for k, r in enumerate(recs):
        X = np.ascontiguousarray(r["X"], dtype=np.float32)
        out = np.full_like(X, np.nan)
        keep.append(X)
        outs.append(out)
        jobs[k].timeseries = X.ctypes.data
        jobs[k].M, jobs[k].N = X.shape[1], X.shape[0]
        jobs[k].pre_out = out.ctypes.data
        jobs[k].bp = api.bandpass_opts(r["samplerate"], r["freq_min"], r["freq_max"], num_threads=16)
        jobs[k].wh = _lib.WhitenOpts(0.0, _lib.PRECISION_PLAIN)
    jobs[1].bp.num_threads = 0  # invalid: the geometry needs T >= 1
    rc = L.ms3gpu_bandpass_whiten_batch(jobs, 3, None)
    assert rc == _lib.ERR_INVALID and "job 1" in _lib.last_error()
    assert [jobs[k].status for k in range(3)] == [_lib.OK, _lib.ERR_INVALID, _lib.OK]
    for k in (0, 2):
        assert np.all(np.isfinite(outs[k]))
    assert np.all(np.isnan(outs[1]))


def test_filtered_signal_in_the_output_buffer_gives_the_same_values(gpu_lib, monkeypatch):
    """When the library's filtered-signal buffer does not fit beside the
    caller's buffers, a float32 output buffer holds the filtered signal and
    is whitened in place in slabs (forced here with MS3GPU_FILT_IN_PLACE):
    the outputs must be those of the ordinary path, for single calls on
    device buffers and for a batch."""
    import torch

    recs = _recordings()[2:]
    dev = torch.device("cuda", 0)
    base = []
    for r in recs:
        Xd = torch.from_numpy(r["X"]).to(dev)
        base.append(api.bandpass_whiten(Xd, r["samplerate"], r["freq_min"], r["freq_max"],
                                        num_threads=r["num_threads"]).cpu().numpy())
    base_batch = api.bandpass_whiten_batch(recs)
    monkeypatch.setenv("MS3GPU_FILT_IN_PLACE", "1")
    for k, r in enumerate(recs):
        Xd = torch.from_numpy(r["X"]).to(dev)
        got = api.bandpass_whiten(Xd, r["samplerate"], r["freq_min"], r["freq_max"],
                                  num_threads=r["num_threads"]).cpu().numpy()
        np.testing.assert_array_equal(got, base[k], err_msg=f"single {k}")
    for k, (got, want) in enumerate(zip(api.bandpass_whiten_batch(recs), base_batch)):
        np.testing.assert_array_equal(got, want, err_msg=f"batch job {k}")


def test_many_small_recordings_in_one_batch(gpu_lib):
    """24 short recordings of 16-100 channels in one batch: their power
    iterations run concurrently on the batch's streams with most CTAs of each
    cluster owning no rows.  Every job must succeed and equal its single
    call bit for bit."""
    rng = np.random.default_rng(7)
    recs = []
    for k in range(24):
        M = int([16, 32, 40, 64, 100][k % 5])
        N = int(rng.integers(130_000, 250_000))
        recs.append(dict(X=synth.generate_numpy(M, N, K=4, seed=300 + k), samplerate=30000.0, freq_min=300.0,
                         freq_max=6000.0, num_threads=16))
    outs = api.bandpass_whiten_batch(recs)
    for k, (r, out) in enumerate(zip(recs, outs)):
        single = api.bandpass_whiten(r["X"], r["samplerate"], r["freq_min"], r["freq_max"],
                                     num_threads=r["num_threads"])
        np.testing.assert_array_equal(out, single, err_msg=f"job {k}")
