"""ctypes loader for oracle/build/libref32.so, the C++ restatement ("ref32")
of the reference's ms3.bandpass_filter / ms3.whiten (test infrastructure).

Arrays follow the C ABI layout used throughout: a timeseries of M channels
and N timepoints is an (N, M) C-contiguous float32 array, i.e. the .mda
column-major M x N layout with the channel index fastest.  M x M matrices
(XXt, W) are numpy arrays in matrix notation, W[i, j] = W(i, j); at the ctypes
boundary they are passed column-major like the reference's Mda.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "build", "libref32.so")
_lib = None

c_i64 = ctypes.c_int64
c_dbl = ctypes.c_double
c_int = ctypes.c_int
_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_i16p = ctypes.POINTER(ctypes.c_int16)


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.ref32_define_kernel.argtypes = [c_i64, _dp, c_dbl, c_dbl, c_dbl, c_dbl]
        L.ref32_bandpass_chunk_size.argtypes = [c_i64, c_i64]
        L.ref32_bandpass_chunk_size.restype = c_i64
        L.ref32_bandpass_peak_ram_mb.argtypes = [c_i64, c_i64]
        L.ref32_bandpass_peak_ram_mb.restype = c_dbl
        L.ref32_whiten_peak_ram_mb.argtypes = [c_i64]
        L.ref32_whiten_peak_ram_mb.restype = c_dbl
        L.ref32_fft.argtypes = [_fp, c_i64, c_i64, c_int]
        L.ref32_bandpass_filter.argtypes = [_fp, c_i64, c_i64, c_dbl, c_dbl, c_dbl, c_dbl, c_dbl,
                                            c_int, c_i64, c_int, _fp, _i16p]
        L.ref32_whiten_xxt.argtypes = [_fp, c_i64, c_i64, c_int, _dp]
        L.ref32_whitening_matrix.argtypes = [_dp, c_i64, _dp, _dp, _dp]
        L.ref32_whiten_apply.argtypes = [_fp, c_i64, c_i64, _dp, c_dbl, c_int, _fp]
        L.ref32_whiten.argtypes = [_fp, c_i64, c_i64, c_dbl, c_int, _fp, _dp, _dp]
        L.ref32_compute_whitening_matrix.argtypes = [ctypes.POINTER(_fp), ctypes.POINTER(c_i64), c_int, c_i64,
                                                     ctypes.POINTER(ctypes.c_int32), c_int, _dp, _dp]
        L.ref32_compute_whitening_matrix.restype = c_int
        L.ref32_whiten_clips.argtypes = [_fp, c_i64, c_i64, c_i64, _dp, c_dbl, _fp]
        L.ref32_mask_out_artifacts.argtypes = [_fp, c_i64, c_i64, c_dbl, c_i64, _fp]
        L.ref32_mask_out_artifacts.restype = c_i64
        L.ref32_detect_events.argtypes = [_fp, c_i64, c_i64, c_dbl, c_dbl, c_int, c_i64, c_i64,
                                          ctypes.POINTER(c_i64), ctypes.POINTER(c_i64), c_i64]
        L.ref32_detect_events.restype = c_i64
        L.ref32_float_to_int16.argtypes = [ctypes.c_float]
        L.ref32_float_to_int16.restype = ctypes.c_int16
        _lib = L
    return _lib


def _f(a):
    return a.ctypes.data_as(_fp)


def _d(a):
    return a.ctypes.data_as(_dp)


def define_kernel(L, samplerate, freq_min, freq_max, freq_wid):
    k = np.zeros(L, np.float64)
    lib().ref32_define_kernel(L, _d(k), samplerate, freq_min, freq_max, freq_wid)
    return k


def chunk_size(M, num_threads):
    return lib().ref32_bandpass_chunk_size(M, num_threads)


def fft(z: np.ndarray, sign: int) -> np.ndarray:
    """z: (L, howmany) complex64; returns the unnormalised DFT along axis 0."""
    a = np.ascontiguousarray(z, dtype=np.complex64).copy()
    L, B = a.shape
    rc = lib().ref32_fft(a.view(np.float32).ctypes.data_as(_fp), L, B, sign)
    if rc != 0:
        raise RuntimeError("ref32_fft failed")
    return a


def bandpass_filter(X_rows: np.ndarray, samplerate, freq_min, freq_max, freq_wid=1000.0,
                    quantization_unit=0.0, subsample_factor=1, num_threads=16, exec_threads=0):
    """X_rows: (N, M) float32.  Returns (N//sub, M) float32, or int16 when
    quantization_unit != 0 (the content of the reference's output file)."""
    X = np.ascontiguousarray(X_rows, dtype=np.float32)
    N, M = X.shape
    sub = subsample_factor or 1
    out = np.zeros((N // sub, M), np.float32)
    o16 = np.zeros((N // sub, M), np.int16) if quantization_unit else None
    lib().ref32_bandpass_filter(_f(X), M, N, samplerate, freq_min, freq_max, freq_wid,
                                quantization_unit, sub, num_threads, exec_threads, _f(out),
                                o16.ctypes.data_as(_i16p) if o16 is not None else None)
    return o16 if o16 is not None else out


def whiten_xxt(X_rows, exec_threads=0):
    X = np.ascontiguousarray(X_rows, dtype=np.float32)
    N, M = X.shape
    C = np.zeros((M, M), np.float64)
    lib().ref32_whiten_xxt(_f(X), M, N, exec_threads, _d(C))
    return C.T.copy()


def whitening_matrix(XXt):
    C = np.ascontiguousarray(np.asarray(XXt, dtype=np.float64).T)
    M = C.shape[0]
    W = np.zeros((M, M), np.float64)
    comps = np.zeros((M, M), np.float64)
    sig = np.zeros(M, np.float64)
    lib().ref32_whitening_matrix(_d(C), M, _d(W), _d(comps), _d(sig))
    return W.T.copy(), comps.T.copy(), sig


def whiten_apply(X_rows, W, quantization_unit=0.0, exec_threads=0):
    X = np.ascontiguousarray(X_rows, dtype=np.float32)
    N, M = X.shape
    out = np.zeros((N, M), np.float32)
    Wc = np.ascontiguousarray(np.asarray(W, dtype=np.float64).T)
    lib().ref32_whiten_apply(_f(X), M, N, _d(Wc), quantization_unit, exec_threads, _f(out))
    return out


def float_to_int16(a: np.ndarray) -> np.ndarray:
    f = lib().ref32_float_to_int16
    flat = np.asarray(a, np.float32).ravel()
    return np.array([f(float(v)) for v in flat], np.int16).reshape(np.shape(a))


def whiten(X_rows, quantization_unit=0.0, exec_threads=0):
    """Returns (out, XXt, W); out is float32 (N, M), or int16 when
    quantization_unit > 0 (values already integral, converted as the
    reference's writer does)."""
    X = np.ascontiguousarray(X_rows, dtype=np.float32)
    N, M = X.shape
    out = np.zeros((N, M), np.float32)
    C = np.zeros((M, M), np.float64)
    W = np.zeros((M, M), np.float64)
    lib().ref32_whiten(_f(X), M, N, quantization_unit, exec_threads, _f(out), _d(C), _d(W))
    C, W = C.T.copy(), W.T.copy()
    if quantization_unit > 0:
        return float_to_int16(out), C, W
    return out, C, W


def compute_whitening_matrix(X_list, channels=None):
    """ms3.compute_whitening_matrix on in-memory recordings: (N_i, M) float32
    row arrays concatenated in time, optional 1-based channel numbers.
    Returns (W, XXt) in matrix notation."""
    arrs = [np.ascontiguousarray(X, dtype=np.float32) for X in X_list]
    M = arrs[0].shape[1]
    ptrs = (ctypes.POINTER(ctypes.c_float) * len(arrs))(*[_f(a) for a in arrs])
    Ns = (ctypes.c_int64 * len(arrs))(*[a.shape[0] for a in arrs])
    ch = np.ascontiguousarray(channels if channels is not None else [], dtype=np.int32)
    M2 = len(ch) if len(ch) else M
    W = np.zeros((M2, M2), np.float64)
    C = np.zeros((M2, M2), np.float64)
    rc = lib().ref32_compute_whitening_matrix(ptrs, Ns, len(arrs), M,
                                              ch.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(ch),
                                              _d(W), _d(C))
    if rc != 0:
        raise ValueError("channel number outside 1..M")
    return W.T.copy(), C.T.copy()


def whiten_clips(clips, W, quantization_unit=0.0):
    """ms3.whiten_clips: clips as an (L, T, M) float32 array (the .mda
    M x T x L layout); float32 out, or int16 when quantization_unit > 0."""
    c = np.ascontiguousarray(clips, dtype=np.float32)
    L, T, M = c.shape
    out = np.zeros_like(c)
    Wc = np.ascontiguousarray(np.asarray(W, dtype=np.float64).T)
    lib().ref32_whiten_clips(_f(c), M, T, L, _d(Wc), float(quantization_unit), _f(out))
    if quantization_unit > 0:
        return float_to_int16(out)
    return out


def mask_out_artifacts(X_rows, threshold=6.0, interval_size=2000):
    """ms3.mask_out_artifacts on an (N, M) float32 array; returns (out, kept)."""
    X = np.ascontiguousarray(X_rows, dtype=np.float32)
    N, M = X.shape
    out = np.zeros_like(X)
    kept = lib().ref32_mask_out_artifacts(_f(X), M, N, float(threshold), int(interval_size), _f(out))
    if kept < 0:
        raise ValueError("Problem with input parameters. Either threshold or interval_size is zero.")
    return out, kept


def detect_events(X_rows, detect_threshold=3.0, detect_interval=10.0, detect_sign=0, chunk_size=None, pad=1000):
    """mountainsortalg's event detection on every channel over mountainsort3's
    time chunks; returns a list of per-channel int64 time arrays."""
    X = np.ascontiguousarray(X_rows, dtype=np.float32)
    N, M = X.shape
    if not chunk_size:
        chunk_size = max(20000, min(N, int(1e9) // (M * 4)))
    counts = np.zeros(M, np.int64)
    cap = N * M // 2 + 1
    times = np.zeros(cap, np.int64)
    p64 = ctypes.POINTER(c_i64)
    total = lib().ref32_detect_events(_f(X), M, N, float(detect_threshold), float(detect_interval), int(detect_sign),
                                      int(chunk_size), int(pad), counts.ctypes.data_as(p64),
                                      times.ctypes.data_as(p64), cap)
    return np.split(times[:total], np.cumsum(counts)[:-1])
