"""The CPU oracle (oracle/ref32: C++ restatement of the reference; oracle/
oracle64: FP64 numpy) checked against known answers and against each other.
These pin the checker that the GPU parity tests use."""
import json
import os

import numpy as np
import pytest
from scipy.special import erf

from oracle import oracle64 as o64

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def rel(a, b):
    return o64.rel_l2(a, b)


@pytest.mark.parametrize("L", [1, 2, 3, 5, 8, 30, 97, 480, 500, 3410, 240000])
def test_fft_matches_numpy(ref32, L):
    rng = np.random.default_rng(L)
    z = (rng.standard_normal((L, 3)) + 1j * rng.standard_normal((L, 3))).astype(np.complex64)
    f = ref32.fft(z, -1)
    b = ref32.fft(z, +1)
    zz = z.astype(np.complex128)
    assert rel(f, np.fft.fft(zz, axis=0)) < 3e-7
    assert rel(b, np.fft.ifft(zz, axis=0) * L) < 3e-7


def test_kernel_formula(ref32):
    # define_kernel (p_bandpass_filter.cpp:421-447) against an independent FP64 formula
    L, fs = 240000, 30000.0
    K = ref32.define_kernel(L, fs, 300.0, 6000.0, 1000.0)
    i = np.arange(L)
    f = np.where(i <= (L + 1) // 2, i * fs / L, (i - L) * fs / L)
    a = np.abs(f)
    v = (1 + erf(3 * (a - 300) / 300)) / 2 * (1 - erf((a - 6000) / 1000)) / 2
    v[0] = 0.0
    # 1 - erf(x) loses ~12 digits in the high-frequency tail: libm vs scipy differ there
    np.testing.assert_allclose(K, np.sqrt(v), rtol=1e-10, atol=1e-300)
    assert K[0] == 0.0
    # even kernel for even L (two channels may share one complex transform)
    np.testing.assert_array_equal(K[1:], K[1:][::-1])
    with open(os.path.join(GOLD, "oracle_vectors.json")) as fh:
        g = json.load(fh)["kernel_240000"]
    np.testing.assert_array_equal(K[g["index"]], np.array(g["value"]))


def test_kernel_no_lowcut_keeps_dc(ref32):
    K = ref32.define_kernel(1000, 1000.0, 0.0, 100.0, 10.0)
    assert K[0] > 0.99


def test_chunk_geometry(ref32):
    with open(os.path.join(GOLD, "oracle_vectors.json")) as fh:
        rows = json.load(fh)["chunk_size"]
    for M, T, c in rows:
        assert ref32.chunk_size(M, T) == c == o64.chunk_size(M, T)
    # T >= 12 and M >= 16 always give the canonical 120000 (L = 240000)
    for M in (16, 32, 384):
        for T in (12, 16, 64):
            assert ref32.chunk_size(M, T) == 120000


def test_bandpass_odd_geometry_vs_fp64(ref32):
    # M=6, T=16: chunk 346033, L = 466033 (prime) -> Bluestein in the oracle
    from mountainsort_b200 import synth

    X = synth.generate_numpy(6, 120000, K=2, seed=4, sites=(2, 3))
    assert ref32.chunk_size(6, 16) == 346033
    F = ref32.bandpass_filter(X, 30000, 300, 6000, 1000, num_threads=16)
    F64 = o64.bandpass_filter(X, 30000, 300, 6000, 1000, num_threads=16)
    assert rel(F, F64) < 1e-6


def test_bandpass_ref32_vs_fp64(ref32):
    from mountainsort_b200 import synth

    X = synth.generate_numpy(6, 260000, K=4, seed=1, sites=(2, 3))
    F = ref32.bandpass_filter(X, 30000, 300, 6000, 1000, num_threads=32)
    F64 = o64.bandpass_filter(X, 30000, 300, 6000, 1000, num_threads=32)
    assert F.shape == X.shape and F.dtype == np.float32
    assert rel(F, F64) < 5e-7


def test_bandpass_dc_kill_and_tone(ref32):
    N, fs = 480000, 30000.0
    const = np.full((N, 2), 5.0, np.float32)
    F = ref32.bandpass_filter(const, fs, 300, 6000, 1000, num_threads=94)
    # interior windows see a constant: only the DC bin, which is killed exactly
    assert np.max(np.abs(F[120000:360000])) < 1e-5
    # a tone at a bin frequency of the L = 240000 window passes with gain kernel(f)
    f0 = 1000.0
    t = np.arange(N)
    tone = np.sin(2 * np.pi * f0 * t / fs).astype(np.float32)[:, None]
    F = ref32.bandpass_filter(tone, fs, 300, 6000, 1000, num_threads=187)
    K = ref32.define_kernel(240000, fs, 300, 6000, 1000)
    g = K[int(f0 * 240000 / fs)]
    np.testing.assert_allclose(F[120000:360000, 0], g * tone[120000:360000, 0], atol=2e-5)


def test_bandpass_impulse_is_windowed_kernel(ref32):
    N = 240000
    x = np.zeros((N, 1), np.float32)
    x[100000, 0] = 1.0
    F = ref32.bandpass_filter(x, 30000, 300, 6000, 1000, num_threads=187)
    # chunk 0 covers [0, 120000): window starts at -60000; impulse at window index 160000
    K = ref32.define_kernel(240000, 30000, 300, 6000, 1000)
    h = np.fft.ifft(K).real  # circular impulse response
    expect = np.roll(h, 160000)[60000:180000]
    np.testing.assert_allclose(F[:120000, 0], expect, atol=1e-7)


def test_bandpass_quantized_and_subsampled(ref32):
    from mountainsort_b200 import synth

    X = synth.generate_numpy(3, 250000, K=2, seed=2, sites=(1, 2))
    F = ref32.bandpass_filter(X, 30000, 300, 6000, 1000, num_threads=63)
    Q = ref32.bandpass_filter(X, 30000, 300, 6000, 1000, quantization_unit=0.5, num_threads=63)
    assert Q.dtype == np.int16
    np.testing.assert_array_equal(Q, np.trunc(F.astype(np.float64) * 2.0).astype(np.int16))
    S = ref32.bandpass_filter(X, 30000, 300, 6000, 1000, subsample_factor=3, num_threads=63)
    assert S.shape == (250000 // 3, 3)
    # chunk 120000 is a multiple of 3: rows are every third filtered sample
    np.testing.assert_array_equal(S, F[: 3 * (250000 // 3):3])


def test_bandpass_freq_max_zero_copies(ref32):
    X = np.random.default_rng(0).standard_normal((100, 3)).astype(np.float32)
    np.testing.assert_array_equal(ref32.bandpass_filter(X, 30000, 300, 0, 1000), X)


def test_whiten_components(ref32):
    rng = np.random.default_rng(5)
    X = (rng.standard_normal((5000, 12)) @ (np.eye(12) + 0.3 * rng.standard_normal((12, 12)))).astype(np.float32)
    C = ref32.whiten_xxt(X)
    C64 = o64.xxt(X)
    assert rel(C, C64) < 1e-9
    np.testing.assert_array_equal(C, C.T)
    W, comps, sig = ref32.whitening_matrix(C)
    W64, comps64, sig64 = o64.whitening_matrix(C)
    assert rel(W, W64) < 1e-12
    assert rel(sig, sig64) < 1e-12
    # whitened covariance is near identity but not exact (10 power iterations)
    Y = ref32.whiten_apply(X, W)
    assert np.abs(o64.xxt(Y) - np.eye(12)).max() < 0.5


def test_whitening_matrix_golden(ref32):
    with open(os.path.join(GOLD, "oracle_vectors.json")) as fh:
        g = json.load(fh)["whitening_6"]
    W, comps, sig = ref32.whitening_matrix(np.array(g["XXt"]))
    np.testing.assert_array_equal(W, np.array(g["W"]))
    np.testing.assert_array_equal(sig, np.array(g["sigma"]))


def test_whitening_matrix_separated_diagonal(ref32):
    d = 10.0 ** np.arange(0, 12, 2)[::-1]
    W, comps, sig = ref32.whitening_matrix(np.diag(d))
    np.testing.assert_allclose(W, np.diag(1 / np.sqrt(d)), rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(sig, d, rtol=1e-12)


def test_whitening_zero_matrix(ref32):
    W, comps, sig = ref32.whitening_matrix(np.zeros((4, 4)))
    assert np.all(W == 0) and np.all(sig == 0)


def test_whiten_rounding_and_int16(ref32):
    rng = np.random.default_rng(9)
    X = rng.standard_normal((20000, 8)).astype(np.float32)
    out, C, W = ref32.whiten(X)
    q = np.round(out.astype(np.float64) / 1e-4)
    assert np.max(np.abs(out / 1e-4 - q)) < 1e-2  # multiples of 1e-4 (as float32)
    y, qd, _, _ = o64.whiten(X)
    assert rel(out, qd) < 5e-6
    o16, _, _ = ref32.whiten(X, quantization_unit=0.01)
    assert o16.dtype == np.int16
    # (int)(y/q + 0.5) truncates toward zero (p_whiten.cpp:445-451)
    expect = np.trunc(out.astype(np.float64) / 0.01 + 0.5)
    np.testing.assert_array_equal(o16, expect.astype(np.int16))


def test_small_case_golden(ref32):
    d = np.load(os.path.join(GOLD, "small_case.npz"))
    filt = ref32.bandpass_filter(d["raw"], 30000, 300, 6000, 1000, num_threads=16)
    np.testing.assert_array_equal(filt, d["filt"])
    pre, xxt, W = ref32.whiten(filt)
    np.testing.assert_array_equal(pre, d["pre"])


def test_float_to_int16_x86(ref32):
    v = np.array([1.9, -1.9, 32767.5, 32768.0, -32769.0, 70000.0, 3e9, np.nan], np.float32)
    got = ref32.float_to_int16(v)
    np.testing.assert_array_equal(got, np.array([1, -1, 32767, -32768, 32767, 4464, 0, 0], np.int16))


def test_compute_whitening_matrix_oracle_concatenates_and_selects_channels(ref32):
    # ms3.compute_whitening_matrix (p_whiten.cpp:208-298): recordings concatenated
    # in time, 1-based channel subset, XXt / (N - 1), then the power-iteration W
    from mountainsort_b200 import synth
    A = synth.generate_numpy(12, 30000, K=6, seed=3)
    B = synth.generate_numpy(12, 17001, K=6, seed=4)
    ch = [3, 1, 12, 7]
    W, C = ref32.compute_whitening_matrix([A, B], channels=ch)
    X = np.concatenate([A, B])[:, [c - 1 for c in ch]].astype(np.float64)
    assert o64.rel_l2(C, X.T @ X / (X.shape[0] - 1)) <= 1e-9
    W64 = o64.whitening_matrix(C)
    W64 = W64[0] if isinstance(W64, tuple) else W64
    assert o64.rel_l2(W, W64) <= 1e-12
    # no subset = all channels, and the same XXt as ms3.whiten's pass 1 on the concatenation
    W_all, C_all = ref32.compute_whitening_matrix([A, B])
    assert o64.rel_l2(C_all, ref32.whiten_xxt(np.concatenate([A, B]))) <= 1e-12
    with pytest.raises(ValueError):
        ref32.compute_whitening_matrix([A], channels=[0])


def test_whiten_clips_oracle_has_no_1e4_rounding(ref32):
    rng = np.random.default_rng(5)
    clips = rng.standard_normal((20, 40, 12)).astype(np.float32)
    A = rng.standard_normal((12, 12))
    W = (A + A.T) / 24
    out = ref32.whiten_clips(clips, W)
    exact = np.einsum("ltm,mk->ltk", clips.astype(np.float64), W)  # out(m1) = sum_m2 x(m2) W(m2, m1)
    assert o64.rel_l2(out, exact) <= 1e-6
    assert np.abs(out * 1e4 - np.round(out * 1e4)).max() > 1e-2  # not multiples of 1e-4
    q = 0.5
    out16 = ref32.whiten_clips(clips, W, quantization_unit=q)
    assert out16.dtype == np.int16
    assert np.abs(out16.astype(np.float64) - np.trunc(out.astype(np.float64) / q + 0.5)).max() <= 1


def test_mask_out_artifacts_oracle(ref32):
    # p_mask_out_artifacts.cpp:24-104 restated in numpy
    rng = np.random.default_rng(2)
    M, I, nint = 6, 100, 40
    N = nint * I + 37  # a tail beyond the last whole interval
    X = rng.standard_normal((N, M)).astype(np.float32)
    X[5 * I + 10, 2] = 80.0  # artifact in interval 5
    X[3, 4] = 80.0  # artifact in interval 0 (the reference also writes use_it[-1])
    out, kept = ref32.mask_out_artifacts(X, threshold=6, interval_size=I)
    norms = np.sqrt((X[: nint * I].astype(np.float64) ** 2).reshape(nint, I, M).sum(axis=1))
    use = np.ones(nint + 1, bool)
    for m in range(M):
        v = norms[:, m]
        lim = v.mean() + v.std(ddof=1) * 6
        for i in np.nonzero(v > lim)[0]:
            use[max(i - 1, 0):i + 2] = False
    assert not use[0] and not use[1] and not use[4] and not use[5] and not use[6] and use[2] and use[7]
    expect = np.zeros_like(X)
    for i in range(nint):
        if use[i]:
            expect[i * I:(i + 1) * I] = X[i * I:(i + 1) * I]
    np.testing.assert_array_equal(out, expect)
    assert kept == use[:nint].sum() * I
    with pytest.raises(ValueError):
        ref32.mask_out_artifacts(X, threshold=0)


def test_detect_events_oracle_on_planted_spikes(ref32):
    # detect_events.cpp:69-135: above threshold*stdev, strongest within detect_interval
    rng = np.random.default_rng(4)
    N, M = 60000, 3
    X = rng.standard_normal((N, M)).astype(np.float32)
    X[1000, 0] = -30.0                   # isolated negative spike
    X[5000, 0], X[5006, 0] = 20.0, 25.0  # two within 10 samples: the stronger wins
    X[9000, 1] = 40.0
    times = ref32.detect_events(X, detect_threshold=8, detect_interval=10, detect_sign=0, chunk_size=20000)
    assert list(times[0]) == [1000, 5006] and list(times[1]) == [9000] and len(times[2]) == 0
    neg = ref32.detect_events(X, detect_threshold=8, detect_interval=10, detect_sign=-1, chunk_size=20000)
    assert list(neg[0]) == [1000]
    pos = ref32.detect_events(X, detect_threshold=8, detect_interval=10, detect_sign=1, chunk_size=20000)
    assert list(pos[0]) == [5006] and list(pos[1]) == [9000]
