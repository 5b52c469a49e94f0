"""FP64 oracle for the ms3 bandpass_filter + whiten path (test infrastructure).

The same algorithm and geometry as the reference
(packages/ms3/p_bandpass_filter.cpp:115-229, :421-447;
packages/ms3/p_whiten.cpp:45-206; packages/ms3/pca.cpp:172-195, 409-431,
542-558, 635-651), evaluated entirely in double precision with numpy's
complex128 FFT.  It is the yardstick for the mixed-precision forms (gate: 1e-4
relative L2) and shows the FP32 rounding floor of ref32.

Arrays are (N, M) C-contiguous: one row of M channels per timepoint.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

OVERLAP = 60000


def chunk_size(M: int, num_threads: int) -> int:
    # p_bandpass_filter.cpp:147-155
    target = 1.0 * (1024 * 1024 * 1024) / (6 * 4 * M * num_threads) - 2 * OVERLAP
    c = int(target)
    return max(c, 2 * OVERLAP)


def define_kernel(L: int, samplerate: float, freq_min: float, freq_max: float, freq_wid: float) -> np.ndarray:
    # p_bandpass_filter.cpp:421-447
    i = np.arange(L, dtype=np.float64)
    df = 1.0 / (L / samplerate)
    fgrid = np.where(np.arange(L) <= (L + 1) // 2, df * i, df * (i - L))
    absf = np.abs(fgrid)
    val = np.ones(L)
    if freq_min != 0:
        val = val * (1 + erf(3.0 * (absf - freq_min) / freq_min)) / 2
        val[0] = 0.0
    if freq_max != 0:
        val = val * (1 - erf((absf - freq_max) / freq_wid)) / 2
    return np.sqrt(val)


def bandpass_filter(X: np.ndarray, samplerate, freq_min, freq_max, freq_wid=1000.0,
                    subsample_factor=1, num_threads=16) -> np.ndarray:
    """FP64 bandpass with the reference's chunk geometry; returns float64
    (N // subsample_factor, M) before any quantization."""
    X = np.asarray(X, dtype=np.float64)
    N, M = X.shape
    sub = subsample_factor or 1
    if freq_max == 0:
        return X.copy()
    ch = chunk_size(M, num_threads)
    L = ch + 2 * OVERLAP
    K = define_kernel(L, samplerate, freq_min, freq_max, freq_wid) / L
    out = np.zeros((N // sub, M))
    for t in range(0, N, ch):
        w = np.zeros((L, M))
        a = t - OVERLAP
        lo, hi = max(a, 0), min(a + L, N)
        if hi > lo:
            w[lo - a:hi - a] = X[lo:hi]
        y = np.fft.ifft(np.fft.fft(w, axis=0) * K[:, None], axis=0).real * L
        y = y[OVERLAP:OVERLAP + ch:sub]
        o0 = t // sub
        n = min(len(y), N // sub - o0)
        if n > 0:
            out[o0:o0 + n] = y[:n]
    return out


def xxt(X: np.ndarray) -> np.ndarray:
    """Exact channel covariance sum_t x_t x_t^T / (N-1) (no mean removal)."""
    X = np.asarray(X, dtype=np.float64)
    N = X.shape[0]
    C = X.T @ X
    if N > 1:
        C /= (N - 1)
    return C


def whitening_matrix(C: np.ndarray, num_iterations: int = 10):
    """The reference's power-iteration whitening matrix in FP64 (deflation
    written as the equivalent rank-2 update)."""
    C = np.array(C, dtype=np.float64)
    M = C.shape[0]
    comps = np.zeros((M, M))
    sig = np.zeros(M)
    v0 = np.sin(np.arange(1, M + 1, dtype=np.float64))
    v0 /= np.linalg.norm(v0)
    for k in range(M):
        v = v0.copy()
        s = 0.0
        for _ in range(num_iterations):
            v = C @ v
            s = np.linalg.norm(v)
            if s:
                v = v / s
        comps[:, k] = v
        sig[k] = s
        u = C @ v
        a = v @ u
        C = C - np.outer(v, u) - np.outer(u, v) + a * np.outer(v, v)
    d = np.zeros(M)
    nz = sig != 0
    d[nz] = 1.0 / np.sqrt(sig[nz])
    return (comps * d) @ comps.T, comps, sig


def quantize(y: np.ndarray) -> np.ndarray:
    # p_whiten.cpp:31-41
    return np.floor(y / 0.0001 + 0.5) * 0.0001


def whiten(X: np.ndarray):
    """Returns (pre_unrounded_fp64, pre_quantized_fp64, XXt, W)."""
    X = np.asarray(X, dtype=np.float64)
    C = xxt(X)
    W, _, _ = whitening_matrix(C)
    # out[t, m1] = sum_m2 x[t, m2] W(m2, m1): the reference reads W[m1*M + m2]
    # of a column-major matrix, i.e. applies W^T (p_whiten.cpp:174-183).
    y = X @ W
    return y, quantize(y), C, W


def rel_l2(a, b) -> float:
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    if not (np.iscomplexobj(a) or np.iscomplexobj(b)):
        a = a.astype(np.float64)
        b = b.astype(np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb else float(np.linalg.norm(a - b))
