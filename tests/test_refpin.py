"""The oracle (ref32, the C++ restatement) pinned to the reference's own code.

oracle/_ref/libmsref.so is the reference's packages/ms3/p_bandpass_filter.cpp,
p_whiten.cpp, pca.cpp, p_mask_out_artifacts.cpp and mda/ classes compiled
from the reference checkout (`make -C oracle ref`) against a Qt subset and an
FFTW interface over the oracle's FFT (FFTW itself is a third-party library the
reference does not vendor).  ref32 must reproduce it bit for bit:

  * against tests/golden/ref_golden.npz, produced by that library with
    tests/golden/make_ref_golden.py -- runs everywhere;
  * against the library itself on more shapes (chunk geometries of several
    thread counts, odd channel counts, a recording shorter than one chunk,
    no low cut, subsampling, int16 outputs, the whitening processors, the
    artifact mask) -- runs where the library was built, skipped elsewhere.
"""
import hashlib
import os

import numpy as np
import pytest

from mountainsort_b200 import synth
from oracle import refpin

HERE = os.path.dirname(os.path.abspath(__file__))
FS, FMIN, FMAX, FWID = 30000.0, 300.0, 6000.0, 1000.0

needs_ref = pytest.mark.skipif(not refpin.available(), reason="oracle/_ref not built (no reference checkout)")


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.fixture(scope="module")
def golden():
    return np.load(os.path.join(HERE, "golden", "ref_golden.npz"))


def _check(g, name, a):
    assert tuple(a.shape) == tuple(g[name + "_shape"])
    assert str(a.dtype) == str(g[name + "_dtype"])
    np.testing.assert_array_equal(a.ravel()[:64], g[name + "_head"])
    assert _sha(a) == str(g[name + "_sha256"])


def test_ref32_reproduces_the_reference_golden_vectors(ref32, golden):
    g = golden
    Xf = g["X16"].astype(np.float32)  # the reference converts int16 to float on read
    bp = ref32.bandpass_filter(Xf, FS, FMIN, FMAX, FWID, num_threads=16)
    _check(g, "bp16", bp)
    _check(g, "bp16_q", ref32.bandpass_filter(Xf, FS, FMIN, FMAX, FWID, quantization_unit=0.5, num_threads=16))
    _check(g, "bp16_sub", ref32.bandpass_filter(Xf, FS, FMIN, FMAX, FWID, subsample_factor=3, num_threads=19))
    _check(g, "wh", ref32.whiten(bp)[0])
    _check(g, "wh_q", ref32.whiten(bp, quantization_unit=0.01)[0])
    _check(g, "mask", ref32.mask_out_artifacts(bp, threshold=3.0, interval_size=500)[0])
    W, _, _ = ref32.whitening_matrix(g["C16"])
    np.testing.assert_array_equal(W, g["W16"])


@needs_ref
@pytest.mark.parametrize("M,N,kw", [
    (32, 250000, dict(num_threads=16)),                        # L = 240000, last chunk partial
    (7, 1000, dict(num_threads=27)),                           # shorter than one chunk, odd M
    (3, 130000, dict(num_threads=63)),                         # odd M
    (16, 200000, dict(num_threads=16, freq_min=0.0)),          # no low cut
    (10, 120000, dict(num_threads=19, subsample_factor=7)),    # subsampled
    (12, 150000, dict(num_threads=16, quantization_unit=2.0)), # int16 output
    (6, 40000, dict(num_threads=16)),                          # L = 466033 (prime: Bluestein)
])
def test_bandpass_matches_reference_code(ref32, M, N, kw):
    kw = dict(kw)
    fmin = kw.pop("freq_min", FMIN)
    X = synth.generate_numpy(M, N, K=max(1, M // 3), seed=M * 7 + N % 13)
    a = refpin.bandpass_filter(X, FS, fmin, FMAX, FWID, **kw)
    b = ref32.bandpass_filter(X, FS, fmin, FMAX, FWID, **kw)
    assert a.dtype == b.dtype and a.shape == b.shape
    np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("M,N,q", [(24, 150000, 0.0), (9, 90000, 0.01), (64, 40000, 0.0)])
def test_whiten_matches_reference_code(ref32, M, N, q):
    X = synth.generate_numpy(M, N, K=max(1, M // 3), seed=M + N)
    F = ref32.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=max(16, 187 // M + 1))
    a = refpin.whiten(F, quantization_unit=q)
    b = ref32.whiten(F, quantization_unit=q)[0]
    np.testing.assert_array_equal(a, b)


@needs_ref
@pytest.mark.parametrize("M", [1, 4, 33, 128])
def test_whitening_matrix_matches_reference_code(ref32, M):
    rng = np.random.default_rng(M)
    A = rng.standard_normal((M, 3 * M + 5))
    C = A @ A.T / A.shape[1]
    np.testing.assert_array_equal(refpin.whitening_matrix(C), ref32.whitening_matrix(C)[0])
    # the reference's unit-test construction: separated diagonal -> diag(1/sqrt(d))
    d = np.linspace(1.0, 9.0, M) ** 2
    np.testing.assert_array_equal(refpin.whitening_matrix(np.diag(d)), ref32.whitening_matrix(np.diag(d))[0])


@needs_ref
def test_whitening_processors_match_reference_code(ref32):
    M = 12
    X1 = synth.generate_numpy(M, 60000, K=4, seed=1)
    X2 = synth.generate_numpy(M, 45000, K=4, seed=2)
    ch = [2, 5, 6, 11]
    Wr = refpin.compute_whitening_matrix([X1, X2], channels=ch)
    W3, _ = ref32.compute_whitening_matrix([X1, X2], channels=ch)
    np.testing.assert_array_equal(Wr, W3)
    Xs = np.ascontiguousarray(X1[:, [c - 1 for c in ch]])
    np.testing.assert_array_equal(refpin.apply_whitening_matrix(Xs, Wr, quantization_unit=0.05),
                                  ref32.whiten_apply(Xs, Wr, quantization_unit=0.05))
    # 30 clips of 50 timepoints on the 4 channels: (L, T, M) rows = the .mda M x T x L array
    clips = (np.random.default_rng(3).standard_normal((30, 50, 4)) * 20).astype(np.float32)
    got = refpin.whiten_clips(clips.transpose(2, 1, 0), Wr).transpose(2, 1, 0)
    np.testing.assert_array_equal(got, ref32.whiten_clips(clips, Wr))


@needs_ref
def test_mask_out_artifacts_matches_reference_code(ref32):
    X = synth.generate_numpy(8, 300000, K=3, seed=4)
    X[123000:123300, 2] += 3000.0
    X[200000:200100, :] -= 2000.0
    a = refpin.mask_out_artifacts(X, threshold=5.0, interval_size=1000)
    b, _ = ref32.mask_out_artifacts(X, threshold=5.0, interval_size=1000)
    np.testing.assert_array_equal(a, b)
