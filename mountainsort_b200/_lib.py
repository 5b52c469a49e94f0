"""ctypes binding of libms3gpu.so (the C ABI declared in include/ms3gpu.h).

There is no fallback: if the shared library is missing or fails to load,
importing this module raises.  Buffers may be numpy arrays (host memory) or
torch tensors (host or CUDA); the library classifies each pointer itself.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libms3gpu.so")
# the bounds-checked build (python -m mountainsort_b200.build --checked);
# MS3GPU_LIBRARY=checked makes load() use it
CHECKED_LIB_PATH = os.path.join(HERE, "libms3gpu_checked.so")

OK = 0
ERR_INVALID = -1
ERR_CUDA = -2
ERR_UNSUPPORTED = -3
ERR_NOMEM = -4
ERR_IO = -5
DTYPE_FLOAT32 = -3
DTYPE_INT16 = -4


class BandpassOpts(ctypes.Structure):
    """ms3gpu_bandpass_opts (Bandpass_filter_opts, p_bandpass_filter.h:21-31)."""
    _fields_ = [
        ("samplerate", ctypes.c_double),
        ("freq_min", ctypes.c_double),
        ("freq_max", ctypes.c_double),
        ("freq_wid", ctypes.c_double),
        ("quantization_unit", ctypes.c_double),
        ("subsample_factor", ctypes.c_int32),
        ("num_threads", ctypes.c_int32),
    ]


PRECISION_PLAIN = 0
PRECISION_MIXED = 1


class WhitenOpts(ctypes.Structure):
    """ms3gpu_whiten_opts (Whiten_opts, p_whiten.h:21-26, plus precision)."""
    _fields_ = [("quantization_unit", ctypes.c_double), ("precision", ctypes.c_int32)]


class Job(ctypes.Structure):
    """ms3gpu_job: one recording of ms3gpu_bandpass_whiten_batch."""
    _fields_ = [
        ("timeseries", ctypes.c_void_p),
        ("M", ctypes.c_int64),
        ("N", ctypes.c_int64),
        ("filt_out", ctypes.c_void_p),
        ("pre_out", ctypes.c_void_p),
        ("bp", BandpassOpts),
        ("wh", WhitenOpts),
        ("status", ctypes.c_int32),
    ]


READ_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p)
WRITE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64, ctypes.c_void_p)


class StreamIO(ctypes.Structure):
    """ms3gpu_stream_io: read / write callbacks of the streaming entry points."""
    _fields_ = [
        ("read", READ_FN),
        ("read_ctx", ctypes.c_void_p),
        ("write", WRITE_FN),
        ("write_ctx", ctypes.c_void_p),
        ("slab_bytes", ctypes.c_int64),
    ]


class Ms3GpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ms3gpu error {code}: {msg}")
        self.code = code


_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_dbl = ctypes.c_double

# name -> (restype, argtypes)
SIGNATURES = {
    "ms3gpu_last_error": (ctypes.c_char_p, []),
    "ms3gpu_version": (ctypes.c_char_p, []),
    "ms3gpu_launch_count": (ctypes.c_uint64, []),
    "ms3gpu_release_cached_memory": (ctypes.c_int, []),
    "ms3gpu_bandpass_chunk_size": (_i64, [_i64, ctypes.c_int32]),
    "ms3gpu_bandpass_output_dims": (ctypes.c_int, [_i64, _i64, ctypes.POINTER(BandpassOpts),
                                                   ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                                                   ctypes.POINTER(ctypes.c_int32)]),
    "ms3gpu_bandpass_requirements": (ctypes.c_int, [_i64, _i64, ctypes.POINTER(BandpassOpts),
                                                    ctypes.POINTER(_dbl)]),
    "ms3gpu_whiten_requirements": (ctypes.c_int, [_i64, _i64, ctypes.POINTER(_dbl)]),
    "ms3gpu_bandpass_filter": (ctypes.c_int, [_vp, _i64, _i64, _vp, ctypes.POINTER(BandpassOpts), _vp]),
    "ms3gpu_whiten": (ctypes.c_int, [_vp, _i64, _i64, _vp, ctypes.POINTER(WhitenOpts), _vp]),
    "ms3gpu_bandpass_whiten": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp, ctypes.POINTER(BandpassOpts),
                                              ctypes.POINTER(WhitenOpts), _vp]),
    "ms3gpu_whiten_covariance": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp]),
    "ms3gpu_whiten_covariance_noalloc": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp]),
    "ms3gpu_whitening_matrix": (ctypes.c_int, [_vp, _i64, _vp, _vp, _vp, _vp]),
    "ms3gpu_apply_whitening_matrix": (ctypes.c_int, [_vp, _i64, _i64, _vp, _dbl, ctypes.c_int32, _vp, _vp]),
    "ms3gpu_bandpass_filter_i16": (ctypes.c_int, [_vp, _i64, _i64, _vp, ctypes.POINTER(BandpassOpts), _vp]),
    "ms3gpu_bandpass_whiten_batch": (ctypes.c_int, [ctypes.POINTER(Job), ctypes.c_int32, _vp]),
    "ms3gpu_compute_whitening_matrix": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _i64, _vp, ctypes.c_int32, _vp,
                                                       _vp]),
    "ms3gpu_whiten_blocks": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp, ctypes.c_int32, _vp,
                                            ctypes.POINTER(WhitenOpts), _vp]),
    "ms3gpu_mask_out_artifacts": (ctypes.c_int, [_vp, _i64, _i64, _dbl, _i64, _vp, _vp, _vp]),
    "ms3gpu_detect_events": (ctypes.c_int, [_vp, _i64, _i64, _dbl, _dbl, ctypes.c_int32, _i64, _vp, _vp, _i64, _vp]),
    "ms3gpu_whiten_clips": (ctypes.c_int, [_vp, _i64, _i64, _i64, _vp, _dbl, ctypes.c_int32, _vp, _vp]),
    "ms3gpu_bandpass_filter_stream": (ctypes.c_int, [_i64, _i64, ctypes.c_int32, ctypes.POINTER(StreamIO),
                                                     ctypes.POINTER(BandpassOpts), _vp]),
    "ms3gpu_whiten_stream": (ctypes.c_int, [_i64, _i64, ctypes.POINTER(StreamIO), ctypes.POINTER(WhitenOpts),
                                            _vp]),
    "ms3gpu_bandpass_filter_windows": (ctypes.c_int, [_vp, ctypes.c_int32, _i64, _i64, _i64, _i64, _i64, _i64,
                                                      _vp, _i64, _i64, ctypes.POINTER(BandpassOpts), _vp]),
    "ms3gpu_whiten_covariance_sum": (ctypes.c_int, [_vp, _i64, _i64, _vp, _vp]),
    "ms3gpu_mask_out_artifacts_stream": (ctypes.c_int, [_i64, _i64, _dbl, _i64, ctypes.POINTER(StreamIO), _vp,
                                                        _vp]),
}

_lib = None


def load(path: str = None):
    """Load the library (once): libms3gpu.so, or libms3gpu_checked.so when
    MS3GPU_LIBRARY=checked.  Raises OSError if it is missing."""
    global _lib
    if path is None:
        path = CHECKED_LIB_PATH if os.environ.get("MS3GPU_LIBRARY") == "checked" else LIB_PATH
    if _lib is None:
        if not os.path.exists(path):
            raise OSError(f"libms3gpu.so not built: {path} (run python -m mountainsort_b200.build)")
        L = ctypes.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    return load().ms3gpu_last_error().decode("utf-8", "replace")


def check(rc: int) -> None:
    if rc != OK:
        raise Ms3GpuError(rc, last_error())
