"""File-level mirror of the reference's two processors, for Python callers.

The same names, parameters, defaults and output dtypes as the reference's
ms3.mp (packages/ms3/mountainsort3_main.cpp:146-165, 547-591): each function
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
    X = _read_rows(timeseries)
    Y = api.bandpass_filter(X, samplerate, freq_min, freq_max, freq_wid, quantization_unit,
                            subsample_factor, num_threads=_request_num_threads)
    mdaio.writemda(Y.T, timeseries_out)
    return True


def whiten(timeseries, timeseries_out, quantization_unit=0) -> bool:
    """ms3.whiten (p_whiten.cpp:45-206)."""
    X = _read_rows(timeseries)
    Y = api.whiten(X, quantization_unit=float(quantization_unit))
    mdaio.writemda(Y.T, timeseries_out)
    return True


PROCESSORS = {"ms3.bandpass_filter": bandpass_filter, "ms3.whiten": whiten}


def run(name: str, **kwargs) -> bool:
    if name not in PROCESSORS:
        raise KeyError(f"Unexpected processor name: {name}")
    return PROCESSORS[name](**kwargs)
