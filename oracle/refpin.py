"""ctypes loader for oracle/_ref/libmsref.so: the reference's own ms3
processor functions (packages/ms3/p_bandpass_filter.cpp, p_whiten.cpp,
pca.cpp, p_mask_out_artifacts.cpp with the mda/ I/O classes), compiled from
the reference checkout by `make -C oracle ref` against a Qt subset and an
FFTW interface over the oracle's FFT (test infrastructure only).

The processors read and write .mda files as the reference does; these
wrappers write the input with mountainsort_b200.mdaio (whose format is pinned
by the reference's own writer) into a temporary directory and read the
outputs back.  Arrays follow the layout used throughout: an (N, M) float32
timeseries, M x M matrices in matrix notation.

available() is False when the library was not built (a checkout without the
reference); tests that need it skip then, and rely on the committed golden
vectors in tests/golden/ that it produced.
"""
from __future__ import annotations

import ctypes
import os
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libmsref.so")
_lib = None

_c = ctypes.c_char_p
_d = ctypes.c_double
_i = ctypes.c_int
_i64 = ctypes.c_int64
_dp = ctypes.POINTER(ctypes.c_double)


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = ctypes.CDLL(LIB_PATH)
        L.msref_bandpass_filter.argtypes = [_c, _c, _d, _d, _d, _d, _d, _i, _i]
        L.msref_whiten.argtypes = [_c, _c, _d, _i]
        L.msref_whitening_matrix.argtypes = [_dp, _i64, _dp]
        L.msref_compute_whitening_matrix.argtypes = [ctypes.POINTER(_c), _i, ctypes.POINTER(_i), _i, _c]
        L.msref_apply_whitening_matrix.argtypes = [_c, _c, _c, _d]
        L.msref_whiten_clips.argtypes = [_c, _c, _c, _d]
        L.msref_mask_out_artifacts.argtypes = [_c, _c, _d, _i]
        for f in ("msref_bandpass_filter", "msref_whiten", "msref_whitening_matrix", "msref_compute_whitening_matrix",
                  "msref_apply_whitening_matrix", "msref_whiten_clips", "msref_mask_out_artifacts"):
            getattr(L, f).restype = _i
        _lib = L
    return _lib


def _mdaio():
    from mountainsort_b200 import mdaio

    return mdaio


def _run(fn, *args):
    rc = fn(*args)
    if rc != 0:
        raise RuntimeError(f"reference processor failed ({rc})")


def bandpass_filter(X_rows, samplerate, freq_min, freq_max, freq_wid=1000.0, quantization_unit=0.0,
                    subsample_factor=1, num_threads=16):
    """ms3.bandpass_filter with the chunk geometry of num_threads threads.
    Returns the output file's content as (N', M) rows (float32, or int16 when
    quantization_unit != 0)."""
    io = _mdaio()
    with tempfile.TemporaryDirectory() as d:
        pin, pout = os.path.join(d, "in.mda"), os.path.join(d, "out.mda")
        io.writemda(np.ascontiguousarray(X_rows).T, pin)
        _run(lib().msref_bandpass_filter, pin.encode(), pout.encode(), samplerate, freq_min, freq_max, freq_wid,
             quantization_unit, int(subsample_factor), int(num_threads))
        return np.ascontiguousarray(io.readmda(pout).T)


def whiten(X_rows, quantization_unit=0.0, exec_threads=0):
    """ms3.whiten; returns the output file's content as (N, M) rows."""
    io = _mdaio()
    with tempfile.TemporaryDirectory() as d:
        pin, pout = os.path.join(d, "in.mda"), os.path.join(d, "out.mda")
        io.writemda(np.ascontiguousarray(X_rows, dtype=np.float32).T, pin)
        _run(lib().msref_whiten, pin.encode(), pout.encode(), quantization_unit, int(exec_threads))
        return np.ascontiguousarray(io.readmda(pout).T)


def whitening_matrix(XXt):
    """whitening_matrix_from_XXt on an M x M matrix (matrix notation)."""
    C = np.asfortranarray(np.asarray(XXt, dtype=np.float64))
    M = C.shape[0]
    W = np.zeros(M * M, np.float64)
    flat = np.ascontiguousarray(C.ravel(order="F"))
    _run(lib().msref_whitening_matrix, flat.ctypes.data_as(_dp), M, W.ctypes.data_as(_dp))
    return W.reshape((M, M), order="F")


def compute_whitening_matrix(X_list, channels=None):
    """ms3.compute_whitening_matrix over recordings given as (N_i, M) rows;
    channels: 1-based channel numbers (None: all)."""
    io = _mdaio()
    with tempfile.TemporaryDirectory() as d:
        paths = []
        for k, X in enumerate(X_list):
            p = os.path.join(d, f"in{k}.mda")
            io.writemda(np.ascontiguousarray(X, dtype=np.float32).T, p)
            paths.append(p.encode())
        pout = os.path.join(d, "W.mda")
        arr = (_c * len(paths))(*paths)
        ch = list(channels or [])
        carr = (_i * max(1, len(ch)))(*ch)
        _run(lib().msref_compute_whitening_matrix, arr, len(paths), carr, len(ch), pout.encode())
        return np.asarray(io.readmda(pout), dtype=np.float64)


def apply_whitening_matrix(X_rows, W, quantization_unit=0.0):
    io = _mdaio()
    with tempfile.TemporaryDirectory() as d:
        pin, pw, pout = (os.path.join(d, n) for n in ("in.mda", "W.mda", "out.mda"))
        io.writemda(np.ascontiguousarray(X_rows, dtype=np.float32).T, pin)
        io.writemda(np.asarray(W, dtype=np.float64), pw)
        _run(lib().msref_apply_whitening_matrix, pin.encode(), pw.encode(), pout.encode(), quantization_unit)
        return np.ascontiguousarray(io.readmda(pout).T)


def whiten_clips(clips, W, quantization_unit=0.0):
    """clips: the .mda M x T x L array (numpy shape (M, T, L)); returns the
    output file's array in the same shape."""
    io = _mdaio()
    with tempfile.TemporaryDirectory() as d:
        pin, pw, pout = (os.path.join(d, n) for n in ("clips.mda", "W.mda", "out.mda"))
        io.writemda(np.asarray(clips, dtype=np.float32), pin)
        io.writemda(np.asarray(W, dtype=np.float64), pw)
        _run(lib().msref_whiten_clips, pin.encode(), pw.encode(), pout.encode(), quantization_unit)
        return io.readmda(pout)


def mask_out_artifacts(X_rows, threshold=6.0, interval_size=2000):
    io = _mdaio()
    with tempfile.TemporaryDirectory() as d:
        pin, pout = os.path.join(d, "in.mda"), os.path.join(d, "out.mda")
        io.writemda(np.ascontiguousarray(X_rows, dtype=np.float32).T, pin)
        _run(lib().msref_mask_out_artifacts, pin.encode(), pout.encode(), float(threshold), int(interval_size))
        return np.ascontiguousarray(io.readmda(pout).T)
