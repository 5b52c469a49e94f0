"""File-level mirror of the reference's whitening and filter processors, for
Python callers.

The same names, parameters, defaults and output dtypes as the reference's
ms3.mp (packages/ms3/mountainsort3_main.cpp:146-189, 547-615): each function
reads the input .mda, runs the GPU path and writes the output .mda (via
path.tmp and a rename).  Returns True on success like the reference's
processor functions; errors raise Ms3GpuError / MdaError.  The C++
executable ms3gpu.mp next to this file is the drop-in for MountainLab.
"""
from __future__ import annotations

import os
import shutil

import numpy as np

from . import api, mdaio

SPEC = {
    "ms3.bandpass_filter": {
        "version": "0.20",
        "inputs": ["timeseries"],
        "outputs": ["timeseries_out"],
        "parameters": [("samplerate", False, None), ("freq_min", False, None), ("freq_max", False, None),
                       ("freq_wid", True, 1000), ("quantization_unit", True, 0), ("subsample_factor", True, 1)],
    },
    "ms3.whiten": {
        "version": "0.1",
        "inputs": ["timeseries"],
        "outputs": ["timeseries_out"],
        "parameters": [("quantization_unit", True, 0)],
    },
    "ms3.compute_whitening_matrix": {
        "version": "0.11",
        "inputs": ["timeseries_list"],
        "outputs": ["whitening_matrix_out"],
        "parameters": [("channels", True, None)],
    },
    "ms3.whiten_clips": {
        "version": "0.1",
        "inputs": ["clips", "whitening_matrix"],
        "outputs": ["clips_out"],
        "parameters": [("quantization_unit", True, 0)],
    },
    "ms3.apply_whitening_matrix": {
        "version": "0.1",
        "inputs": ["timeseries", "whitening_matrix"],
        "outputs": ["timeseries_out"],
        "parameters": [("quantization_unit", True, 0)],
    },
    "ms3.mask_out_artifacts": {
        "version": "0.1",
        "inputs": ["timeseries"],
        "outputs": ["timeseries_out"],
        "parameters": [("threshold", True, 6), ("interval_size", True, 2000)],
    },
}


def _read_rows(path):
    X = mdaio.readmda(path)
    if X.ndim == 1:
        X = X[:, None]
    M, N = X.shape[0], X.shape[1]
    return np.ascontiguousarray(np.asarray(X, dtype=np.float32).reshape(M, N, order="F").T)


def bandpass_filter(timeseries, timeseries_out, samplerate, freq_min, freq_max, freq_wid=1000,
                    quantization_unit=0, subsample_factor=1, _request_num_threads=None) -> bool:
    """ms3.bandpass_filter (p_bandpass_filter.cpp:115-229)."""
    if float(freq_max) == 0:
        if os.path.exists(timeseries_out):  # QFile::copy does not overwrite
            return False
        shutil.copyfile(timeseries, timeseries_out)
        return True
    # the recording streams through the GPU block by block, as the
    # processor's chunk loop reads it (p_bandpass_filter.cpp:160-220)
    M, N, rows = mdaio.timeseries_rows_view(timeseries)
    in_dt = np.int16 if rows.dtype == np.int16 else np.float32
    sub = int(subsample_factor or 1)
    out_dt = np.int16 if float(quantization_unit) != 0 else np.float32
    out = mdaio.TimeseriesWriter(timeseries_out, out_dt, M, N // sub)
    try:
        api.bandpass_filter_stream(lambda t0, nt: rows[t0:t0 + nt], out.write, M, N, samplerate, freq_min,
                                   freq_max, freq_wid, quantization_unit, sub, num_threads=_request_num_threads,
                                   in_dtype=in_dt)
    except BaseException:
        out.abort()
        raise
    out.close()
    return True


def whiten(timeseries, timeseries_out, quantization_unit=0) -> bool:
    """ms3.whiten (p_whiten.cpp:45-206), reading the input twice like the
    reference (the covariance pass, then the apply pass)."""
    M, N, rows = mdaio.timeseries_rows_view(timeseries)
    q = float(quantization_unit)
    out = mdaio.TimeseriesWriter(timeseries_out, np.int16 if q > 0 else np.float32, M, N)
    try:
        api.whiten_stream(lambda t0, nt: rows[t0:t0 + nt], out.write, M, N, quantization_unit=q)
    except BaseException:
        out.abort()
        raise
    out.close()
    return True


def _parse_channels(channels):
    # split(",", SkipEmptyParts) + toInt, mountainsort3_main.cpp:597-598
    if channels is None or channels == "":
        return None
    if isinstance(channels, str):
        out = []
        for part in channels.split(","):
            if part:
                try:
                    out.append(int(part))
                except ValueError:
                    out.append(0)
        return out or None
    return [int(c) for c in channels]


def _read_matrix(path, M):
    W = np.asarray(mdaio.readmda(path), dtype=np.float64)
    if W.shape[:2] != (M, M):
        raise ValueError(f"whitening matrix {path} is not {M} x {M}")
    return W


def compute_whitening_matrix(timeseries_list, whitening_matrix_out, channels=None) -> bool:
    """ms3.compute_whitening_matrix (p_whiten.cpp:208-298); writes float64."""
    if isinstance(timeseries_list, str):
        timeseries_list = [timeseries_list]
    Xs = [_read_rows(p) for p in timeseries_list]
    W = api.compute_whitening_matrix(Xs, channels=_parse_channels(channels))
    mdaio.writemda(np.asarray(W, dtype=np.float64), whitening_matrix_out, dtype="float64")
    return True


def apply_whitening_matrix(timeseries, whitening_matrix, timeseries_out, quantization_unit=0) -> bool:
    """ms3.apply_whitening_matrix (p_whiten.cpp:347-417)."""
    X = _read_rows(timeseries)
    W = _read_matrix(whitening_matrix, X.shape[1])
    Y = api.apply_whitening_matrix(X, W, quantization_unit=float(quantization_unit))
    mdaio.writemda(Y.T, timeseries_out)
    return True


def whiten_clips(clips, whitening_matrix, clips_out, quantization_unit=0) -> bool:
    """ms3.whiten_clips (p_whiten.cpp:300-345): clips M x T x L."""
    C = np.asarray(mdaio.readmda(clips), dtype=np.float32)
    while C.ndim < 3:
        C = C[..., None]
    M, T, L = C.shape[0], C.shape[1], int(np.prod(C.shape[2:]))
    rows = np.ascontiguousarray(C.reshape(M, T, L, order="F").transpose(2, 1, 0))  # (L, T, M)
    W = _read_matrix(whitening_matrix, M)
    Y = api.whiten_clips(rows, W, quantization_unit=float(quantization_unit))
    mdaio.writemda(np.asarray(Y).transpose(2, 1, 0), clips_out)
    return True


PROCESSORS = {"ms3.bandpass_filter": bandpass_filter, "ms3.whiten": whiten,
              "ms3.compute_whitening_matrix": compute_whitening_matrix,
              "ms3.apply_whitening_matrix": apply_whitening_matrix, "ms3.whiten_clips": whiten_clips}


def mask_out_artifacts(timeseries, timeseries_out, threshold=6, interval_size=2000) -> bool:
    """ms3.mask_out_artifacts (p_mask_out_artifacts.cpp:24-104), streaming the
    memory-mapped input twice (interval norms, then the masked copy).
    Returns False, like the reference, when threshold or interval_size is 0."""
    threshold, interval_size = float(threshold), int(interval_size)
    if threshold == 0 or interval_size <= 0:
        return False
    M, N, rows = mdaio.timeseries_rows_view(timeseries)
    out = mdaio.TimeseriesWriter(timeseries_out, np.float32, M, N)
    try:
        api.mask_out_artifacts_stream(lambda t0, nt: rows[t0:t0 + nt], out.write, M, N, threshold, interval_size)
    except BaseException:
        out.abort()
        raise
    out.close()
    return True


PROCESSORS["ms3.mask_out_artifacts"] = mask_out_artifacts


def run(name: str, **kwargs) -> bool:
    if name not in PROCESSORS:
        raise KeyError(f"Unexpected processor name: {name}")
    return PROCESSORS[name](**kwargs)
