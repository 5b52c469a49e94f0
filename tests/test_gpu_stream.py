"""The streaming forms of ms3.bandpass_filter and ms3.whiten on the GPU:
recordings read and written block by block through callbacks, as the
reference's processors read them (DiskReadMda32::readChunk,
mda/diskreadmda32.cpp:615-661; p_bandpass_filter.cpp:160-220; the two input
passes of p_whiten.cpp:64-206).

Gates: every streamed output equals the in-memory call's bit for bit (the
same kernels on the same windows; the covariance summed over the same
slices), for one block and for many; a slab smaller than one covariance
slice changes only the FP64 summation order (relative L2 <= 1e-6 against
the in-memory result); the streamed bandpass against ref32 at <= 1e-5
relative L2; callback failures end the call with the callback's exception and
leave the library usable."""
import os
import subprocess

import numpy as np
import pytest

from mountainsort_b200 import _lib, api, mdaio, synth
from oracle import oracle64 as o64

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "mountainsort_b200", "ms3gpu.mp")
FS, FMIN, FMAX, FWID = 30000.0, 300.0, 6000.0, 1000.0


class Recorder:
    """A source over an in-memory (N, M) array that logs its reads, and a
    sink that assembles the output and checks the blocks come in order
    without overlap."""

    def __init__(self, X, N_out, M, out_dtype):
        self.X = X
        self.reads = []
        self.Y = np.full((N_out, M), 7, dtype=out_dtype)  # non-zero: gaps must be written as zero
        self.written = np.zeros(N_out, dtype=bool)
        self.last = -1

    def source(self, t0, nt):
        assert 0 <= t0 and t0 + nt <= len(self.X)
        self.reads.append((t0, nt))
        return self.X[t0:t0 + nt]

    def sink(self, t0, rows):
        assert t0 > self.last
        assert not self.written[t0:t0 + len(rows)].any()
        self.Y[t0:t0 + len(rows)] = rows
        self.written[t0:t0 + len(rows)] = True
        self.last = t0


def _bandpass_both(X, M, slab_bytes, in_dtype=np.float32, **kw):
    N = len(X)
    sub = kw.get("subsample_factor", 1)
    q = kw.get("quantization_unit", 0.0)
    out_dt = np.int16 if q != 0 else np.float32
    rec = Recorder(X, N // sub, M, out_dt)
    api.bandpass_filter_stream(rec.source, rec.sink, M, N, FS, FMIN, FMAX, FWID, in_dtype=in_dtype,
                               slab_bytes=slab_bytes, **kw)
    ref = api.bandpass_filter(X, FS, FMIN, FMAX, FWID, **kw)
    # output timepoints no window writes (gaps between subsampled chunks) are zero
    rec.Y[~rec.written] = 0
    return rec, ref


@pytest.mark.parametrize("slab_bytes", [1, 0])
def test_bandpass_stream_equals_in_memory(gpu_lib, ref32, slab_bytes):
    M, N = 32, 1000000
    X = synth.generate_numpy(M, N, K=8, seed=11)
    rec, ref = _bandpass_both(X, M, slab_bytes, num_threads=16)
    np.testing.assert_array_equal(rec.Y, ref)
    assert rec.written.all()
    if slab_bytes == 1:  # one window per block: 9 windows, each read with its 60000-row halos
        assert len(rec.reads) == 9
        assert rec.reads[0] == (0, 180000) and rec.reads[1] == (60000, 240000)
    else:
        assert rec.reads == [(0, N)]
    gold = ref32.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=16)
    assert o64.rel_l2(rec.Y, gold) <= 1e-5


def test_bandpass_stream_int16_subsampled_quantized(gpu_lib):
    # odd M (unpaired loads), int16 input, subsample 7 with chunk % 7 != 0
    # (gaps of zeros), int16 output
    M, N = 7, 700001
    X = synth.generate_numpy(M, N, K=3, seed=5)
    X16 = np.clip(np.round(X / 0.195), -32768, 32767).astype(np.int16)
    T = 187 // M + 1
    rec, ref = _bandpass_both(X16, M, 240000 * M * 2, in_dtype=np.int16, subsample_factor=7,
                              quantization_unit=0.5, num_threads=T)
    assert ref.dtype == np.int16
    np.testing.assert_array_equal(rec.Y, ref)
    assert len(rec.reads) > 1


def test_bandpass_stream_wide_slabs_and_copy(gpu_lib):
    M, N = 384, 600000
    X = synth.generate_numpy(M, N, K=12, seed=2)
    rec, ref = _bandpass_both(X, M, 2 * 120000 * M * 4, num_threads=16)  # two windows per block
    np.testing.assert_array_equal(rec.Y, ref)
    assert len(rec.reads) == 3
    # freq_max = 0 copies the rows unchanged, block by block
    out = np.zeros_like(X)
    api.bandpass_filter_stream(lambda t0, nt: X[t0:t0 + nt], lambda t0, r: out.__setitem__(slice(t0, t0 + len(r)), r),
                               M, N, FS, FMIN, 0.0, slab_bytes=100000 * M * 4)
    np.testing.assert_array_equal(out, X)


@pytest.mark.parametrize("M,N,q,precision", [(32, 1000000, 0.0, "plain"), (384, 600000, 0.0, "plain"),
                                             (384, 600000, 0.0, "mixed"), (64, 400000, 0.05, "plain")])
def test_whiten_stream_equals_in_memory(gpu_lib, M, N, q, precision):
    X = synth.generate_numpy(M, N, K=max(1, M // 4), seed=M + 1)
    X = api.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=16)
    ref = api.whiten(X, quantization_unit=q, precision=precision)
    out_dt = np.int16 if q > 0 else np.float32
    for slab_bytes in [0, 3 * N * M * 4 // 10]:  # one block; about 4 blocks of whole covariance slices
        rec = Recorder(X, N, M, out_dt)
        api.whiten_stream(rec.source, rec.sink, M, N, quantization_unit=q, slab_bytes=slab_bytes,
                          precision=precision)
        np.testing.assert_array_equal(rec.Y, ref)
        assert rec.written.all()
        # two passes over the input, each in increasing order
        half = len(rec.reads) // 2
        assert rec.reads[:half] == rec.reads[half:] and len(rec.reads) == 2 * half
        assert sum(nt for _, nt in rec.reads[:half]) == N
        if slab_bytes:
            assert half >= 3


def test_whiten_stream_slab_below_one_slice(gpu_lib):
    # blocks of 1024 timepoints, below one covariance run of the whole
    # recording: the runs shrink to the block, so each channel's fixed-point
    # scale is taken over 1024 timepoints instead of a whole run.  The
    # covariance stays within its 1e-8 tolerance; at 384 channels the
    # whitening matrix amplifies such differences (~30x) and the 1e-4
    # rounding turns them into whole rounding steps, so the outputs agree to
    # the plain-form tolerance rather than bit for bit.
    M, N = 384, 300000
    X = api.bandpass_filter(synth.generate_numpy(M, N, K=10, seed=9), FS, FMIN, FMAX, FWID, num_threads=16)
    ref = api.whiten(X)
    rec = Recorder(X, N, M, np.float32)
    api.whiten_stream(rec.source, rec.sink, M, N, slab_bytes=1024 * M * 4)
    assert rec.written.all()
    assert o64.rel_l2(rec.Y, ref) <= 1e-5


def test_stream_callback_failures(gpu_lib):
    M, N = 16, 500000
    X = synth.generate_numpy(M, N, K=4, seed=1)
    calls = {"n": 0}

    def bad_source(t0, nt):
        calls["n"] += 1
        if calls["n"] == 3:
            raise KeyError("disk gone")
        return X[t0:t0 + nt]

    with pytest.raises(KeyError):
        api.bandpass_filter_stream(bad_source, lambda t0, r: None, M, N, FS, FMIN, FMAX, slab_bytes=1,
                                   num_threads=16)

    def bad_sink(t0, rows):
        raise OSError("disk full")

    with pytest.raises(OSError):
        api.whiten_stream(lambda t0, nt: X[t0:t0 + nt], bad_sink, M, N, slab_bytes=100000 * M * 4)
    # a short block is an error of the source, reported as such
    with pytest.raises(ValueError):
        api.whiten_stream(lambda t0, nt: X[t0:t0 + nt - 1], lambda t0, r: None, M, N)
    # the library is still usable, and the C status of a failed callback is MS3GPU_ERR_IO
    rec, ref = _bandpass_both(X, M, 1, num_threads=16)
    np.testing.assert_array_equal(rec.Y, ref)
    import ctypes

    io = _lib.StreamIO(_lib.READ_FN(lambda c, t0, nt, d: 1), None, _lib.WRITE_FN(lambda c, t0, nt, s: 0), None, 0)
    o = api.bandpass_opts(FS, FMIN, FMAX, num_threads=16)
    rc = gpu_lib.ms3gpu_bandpass_filter_stream(M, N, _lib.DTYPE_FLOAT32, ctypes.byref(io), ctypes.byref(o), None)
    assert rc == _lib.ERR_IO
    assert "read callback failed" in _lib.last_error()


def _run(*args):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=600)


def test_executable_streams_in_blocks(gpu_lib, tmp_path):
    # the processors with 1 MB blocks give the files of the in-memory calls
    M, N = 64, 900000
    X = synth.generate_numpy(M, N, K=10, seed=4)
    raw, filt, pre = (str(tmp_path / n) for n in ("raw.mda", "filt.mda", "pre.mda"))
    mdaio.writemda(X.T, raw)
    r = _run("ms3.bandpass_filter", f"--timeseries={raw}", f"--timeseries_out={filt}", "--samplerate=30000",
             "--freq_min=300", "--freq_max=6000", "--_request_num_threads=16", "--_slab_mb=1")
    assert r.returncode == 0, r.stderr
    F = api.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=16)
    np.testing.assert_array_equal(mdaio.readmda(filt).T, F)
    r = _run("ms3.whiten", f"--timeseries={filt}", f"--timeseries_out={pre}", "--_slab_mb=1")
    assert r.returncode == 0, r.stderr
    # 1 MB blocks hold whole covariance slices (768 timepoints): the same sums
    np.testing.assert_array_equal(mdaio.readmda(pre).T, api.whiten(F))
    assert not os.path.exists(pre + ".tmp")


def test_executable_streams_directories_of_mixed_and_int16_files(gpu_lib, tmp_path):
    # a directory's files are concatenated in time; float64 / float32 parts
    # are read as float32, an all-int16 directory goes to the GPU as int16
    M, N = 32, 500000
    X = synth.generate_numpy(M, N, K=6, seed=8)
    X16 = np.clip(np.round(X / 0.195), -32768, 32767).astype(np.int16)
    cuts = [0, 130000, 131000, 500000]
    mixed, ints = tmp_path / "mixed", tmp_path / "ints"
    mixed.mkdir()
    ints.mkdir()
    for k, dt in enumerate([np.float64, np.float32, np.float64]):
        part = X[cuts[k]:cuts[k + 1]]
        mdaio.writemda(part.astype(dt).T, str(mixed / f"p{k}.mda"))
        mdaio.writemda(X16[cuts[k]:cuts[k + 1]].T, str(ints / f"p{k}.mda"))
    args = ["--samplerate=30000", "--freq_min=300", "--freq_max=6000", "--_request_num_threads=16", "--_slab_mb=8"]
    for d, ref_in in [(mixed, X.astype(np.float64).astype(np.float32)), (ints, X16)]:
        out = str(tmp_path / f"{d.name}_filt.mda")
        r = _run("ms3.bandpass_filter", f"--timeseries={d}", f"--timeseries_out={out}", *args)
        assert r.returncode == 0, r.stderr
        ref = api.bandpass_filter(ref_in, FS, FMIN, FMAX, FWID, num_threads=16)
        np.testing.assert_array_equal(mdaio.readmda(out).T, ref)
    # whiten of a directory input streams it twice
    pre = str(tmp_path / "pre.mda")
    r = _run("ms3.whiten", f"--timeseries={mixed}", f"--timeseries_out={pre}", "--quantization_unit=0.1",
             "--_slab_mb=8")
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(mdaio.readmda(pre).T, api.whiten(X.astype(np.float32), quantization_unit=0.1))


@pytest.mark.parametrize("M,N", [(1, 50000), (3, 7), (16, 1), (8, 0), (0, 100)])
def test_stream_edge_shapes(gpu_lib, M, N):
    # one channel, recordings shorter than a window's halo, a single
    # timepoint, empty recordings: the same values as the in-memory calls
    X = (np.random.default_rng(M * 1000 + N).standard_normal((N, M)) * 20).astype(np.float32)
    T = max(16, 187 // max(M, 1) + 1)
    rec = Recorder(X, N, M, np.float32)
    api.bandpass_filter_stream(rec.source, rec.sink, M, N, FS, FMIN, FMAX, FWID, num_threads=T, slab_bytes=1)
    if M * N:
        np.testing.assert_array_equal(rec.Y, api.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=T))
    else:
        assert rec.reads == [] and not rec.written.any()
    # one slab: the in-memory covariance slices (blocks smaller than a slice
    # change only the FP64 summation order, tested above)
    rec = Recorder(X, N, M, np.float32)
    api.whiten_stream(rec.source, rec.sink, M, N)
    if M * N:
        np.testing.assert_array_equal(rec.Y, api.whiten(X))


def test_executable_whitening_matrix_processors_in_blocks(gpu_lib, ref32, tmp_path):
    # ms3.compute_whitening_matrix sums x x^T block by block over the list;
    # ms3.apply_whitening_matrix whitens block by block (values of one call)
    M = 16
    A = api.bandpass_filter(synth.generate_numpy(M, 300000, K=4, seed=31), FS, FMIN, FMAX, FWID, num_threads=16)
    B = api.bandpass_filter(synth.generate_numpy(M, 170001, K=4, seed=32), FS, FMIN, FMAX, FWID, num_threads=16)
    pa, pb, pw, po = (str(tmp_path / n) for n in ("a.mda", "b.mda", "W.mda", "o.mda"))
    mdaio.writemda(A.T, pa)
    mdaio.writemda(B.T, pb)
    for chans, sel in [("", list(range(M))), ("--channels=3,1,16,8", [2, 0, 15, 7])]:
        args = ["ms3.compute_whitening_matrix", f"--timeseries_list={pa}", "--timeseries_list", pb,
                f"--whitening_matrix_out={pw}", "--_slab_mb=1"] + ([chans] if chans else [])
        r = _run(*args)
        assert r.returncode == 0, r.stderr
        W = mdaio.readmda(pw)
        W_mem = api.compute_whitening_matrix([A, B], channels=[c + 1 for c in sel] if chans else None)
        assert o64.rel_l2(W, W_mem) <= 1e-9
        W_ref, _ = ref32.compute_whitening_matrix([A, B], channels=[c + 1 for c in sel] if chans else None)
        assert o64.rel_l2(W, W_ref) <= 1e-6
    r = _run("ms3.compute_whitening_matrix", f"--timeseries_list={pa}", f"--whitening_matrix_out={pw}",
             "--channels=0,2")
    assert r.returncode != 0
    # the apply with the all-channel W, in 1 MB blocks, int16 output
    r = _run("ms3.compute_whitening_matrix", f"--timeseries_list={pa}", f"--whitening_matrix_out={pw}")
    assert r.returncode == 0, r.stderr
    W = mdaio.readmda(pw)
    r = _run("ms3.apply_whitening_matrix", f"--timeseries={pa}", f"--whitening_matrix={pw}",
             f"--timeseries_out={po}", "--quantization_unit=0.05", "--_slab_mb=1")
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(mdaio.readmda(po).T, api.apply_whitening_matrix(A, W, quantization_unit=0.05))


@pytest.mark.parametrize("M,N,I,slab", [(32, 1_000_000, 2000, 1), (7, 300_123, 777, 5 * 777 * 7 * 4), (16, 1500, 2000, 1)])
def test_mask_out_artifacts_stream_equals_in_memory(gpu_lib, M, N, I, slab):
    X = api.bandpass_filter(synth.generate_numpy(M, N, K=2, seed=N % 97), FS, FMIN, FMAX, FWID,
                            num_threads=max(16, 187 // M + 1))
    rng = np.random.default_rng(5)
    for t in rng.integers(0, max(1, N - 500), 6):  # artifacts to mask
        X[t:t + 300, rng.integers(0, M)] += 5000.0
    ref, kept_ref = api.mask_out_artifacts(X, 6.0, I, return_kept=True)
    rec = Recorder(X, N, M, np.float32)
    kept = api.mask_out_artifacts_stream(rec.source, rec.sink, M, N, 6.0, I, slab_bytes=slab)
    assert kept == kept_ref
    assert rec.written.all()
    np.testing.assert_array_equal(rec.Y, ref)
    # two passes: the norms read only whole intervals, then every timepoint
    nint = N // I
    assert sum(nt for t0, nt in rec.reads) == nint * I + N


def test_executable_masks_in_blocks(gpu_lib, tmp_path):
    M, N = 16, 400_000
    X = api.bandpass_filter(synth.generate_numpy(M, N, K=3, seed=77), FS, FMIN, FMAX, FWID, num_threads=16)
    X[123456:124000, 3] += 4000.0
    pin, pout = str(tmp_path / "f.mda"), str(tmp_path / "m.mda")
    mdaio.writemda(X.T, pin)
    r = _run("ms3.mask_out_artifacts", f"--timeseries={pin}", f"--timeseries_out={pout}", "--threshold=6",
             "--interval_size=2000", "--_slab_mb=1")
    assert r.returncode == 0, r.stderr
    ref, kept = api.mask_out_artifacts(X, 6.0, 2000, return_kept=True)
    np.testing.assert_array_equal(mdaio.readmda(pout).T, ref)
    assert f"Using {kept * 100.0 / (N // 2000 * 2000):.2f}% of all timepoints" in r.stdout


def test_python_mask_processor_streams_files(gpu_lib, tmp_path):
    from mountainsort_b200 import processors

    M, N = 8, 120_000
    X = api.bandpass_filter(synth.generate_numpy(M, N, K=2, seed=3), FS, FMIN, FMAX, FWID, num_threads=24)
    X[50000:50400, 2] += 3000.0
    pin, pout = str(tmp_path / "f.mda"), str(tmp_path / "m.mda")
    mdaio.writemda(X.T, pin)
    assert processors.run("ms3.mask_out_artifacts", timeseries=pin, timeseries_out=pout, threshold=6,
                          interval_size=1000)
    np.testing.assert_array_equal(mdaio.readmda(pout).T, api.mask_out_artifacts(X, 6.0, 1000))
