"""The C ABI library: it loads, exports every entry point include/ms3gpu.h
declares, and its host-only functions and argument checks behave (no GPU
needed; nothing here launches a kernel)."""
import ctypes
import os
import re

import pytest

from mountainsort_b200 import _lib, api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ms3gpu.h")


def header_symbols():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"MS3GPU_API\s+[\w\s\*]+?\b(ms3gpu_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    syms = header_symbols()
    for s in ["ms3gpu_bandpass_filter", "ms3gpu_whiten", "ms3gpu_bandpass_whiten", "ms3gpu_whiten_covariance",
              "ms3gpu_whitening_matrix", "ms3gpu_apply_whitening_matrix", "ms3gpu_last_error"]:
        assert s in syms


def test_library_exports_every_declared_symbol():
    L = _lib.load()
    for s in header_symbols():
        assert hasattr(L, s), s
    assert set(header_symbols()) == set(_lib.SIGNATURES)


def test_bounds_checked_library_exports_the_same_symbols():
    # the -DMS3GPU_BOUNDS_CHECK twin is built beside the library and loaded
    # with MS3GPU_LIBRARY=checked; it must offer the same C ABI
    if not os.path.exists(_lib.CHECKED_LIB_PATH):
        pytest.skip("libms3gpu_checked.so not built")
    L = ctypes.CDLL(_lib.CHECKED_LIB_PATH)
    for s in header_symbols():
        assert hasattr(L, s), s
    assert L.ms3gpu_bandpass_chunk_size.restype is not None


def test_version_and_geometry():
    L = _lib.load()
    assert b"sm_100a" in L.ms3gpu_version()
    assert api.chunk_size(384, 16) == 120000
    assert api.chunk_size(16, 8) == 229525
    assert api.chunk_size(4, 16) == 579050
    assert L.ms3gpu_bandpass_chunk_size(0, 16) == -1


def test_chunk_size_matches_the_oracle_on_a_grid(ref32):
    # the window geometry of every (channels, threads) the reference can be run with
    # (p_bandpass_filter.cpp:147-155): the output depends on it beyond any tolerance
    for M in list(range(1, 70)) + [96, 127, 128, 129, 192, 255, 256, 383, 384, 385, 512, 1024, 1536, 4096]:
        for T in (1, 2, 3, 7, 8, 15, 16, 27, 32, 63, 64, 128):
            assert api.chunk_size(M, T) == ref32.chunk_size(M, T), (M, T)


def test_output_dims():
    L = _lib.load()
    M, N, dt = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    o = api.bandpass_opts(30000, 300, 6000, 1000, 0, 3, 16)
    assert L.ms3gpu_bandpass_output_dims(8, 1000, ctypes.byref(o), ctypes.byref(M), ctypes.byref(N), ctypes.byref(dt)) == 0
    assert (M.value, N.value, dt.value) == (8, 333, _lib.DTYPE_FLOAT32)
    o = api.bandpass_opts(30000, 300, 6000, 1000, 0.5, 1, 16)
    L.ms3gpu_bandpass_output_dims(8, 1000, ctypes.byref(o), ctypes.byref(M), ctypes.byref(N), ctypes.byref(dt))
    assert dt.value == _lib.DTYPE_INT16
    o = api.bandpass_opts(30000, 300, 0, 1000, 0.5, 3, 16)  # freq_max 0: a copy
    L.ms3gpu_bandpass_output_dims(8, 1000, ctypes.byref(o), ctypes.byref(M), ctypes.byref(N), ctypes.byref(dt))
    assert (N.value, dt.value) == (1000, _lib.DTYPE_FLOAT32)


def test_requirements_match_reference_model(ref32):
    for M, T in [(32, 16), (384, 16), (4, 8)]:
        mb = api.requirements("ms3.bandpass_filter", M, 1000, samplerate=30000, freq_min=300, freq_max=6000,
                              num_threads=T)
        assert mb == pytest.approx(ref32.lib().ref32_bandpass_peak_ram_mb(M, T), rel=1e-15)
        assert api.requirements("ms3.whiten", M, 1000) == pytest.approx(ref32.lib().ref32_whiten_peak_ram_mb(M), rel=1e-15)


@pytest.mark.parametrize("call", [
    lambda L: L.ms3gpu_bandpass_filter(None, 4, 10, None, None, None),
    lambda L: L.ms3gpu_bandpass_filter(None, -1, 10, None, ctypes.byref(api.bandpass_opts(30000, 300, 6000)), None),
    lambda L: L.ms3gpu_bandpass_filter(None, 4, 10, None, ctypes.byref(api.bandpass_opts(30000, 300, 6000)), None),
    lambda L: L.ms3gpu_bandpass_filter(None, 4, 10, None, ctypes.byref(api.bandpass_opts(0, 300, 6000)), None),
    lambda L: L.ms3gpu_whiten(None, 4, 10, None, None, None),
    lambda L: L.ms3gpu_bandpass_whiten(None, 4, 10, None, None, ctypes.byref(api.bandpass_opts(30000, 300, 6000, 1000, 0, 2)),
                                       ctypes.byref(_lib.WhitenOpts(0)), None),
])
def test_invalid_arguments_rejected_before_device_work(call):
    L = _lib.load()
    assert call(L) == _lib.ERR_INVALID
    assert _lib.last_error()


def _io(read=True, write=True, slab_bytes=0):
    rd = _lib.READ_FN(lambda c, t0, nt, d: 0) if read else _lib.READ_FN()
    wr = _lib.WRITE_FN(lambda c, t0, nt, s: 0) if write else _lib.WRITE_FN()
    return _lib.StreamIO(rd, None, wr, None, slab_bytes)


@pytest.mark.parametrize("make", [
    lambda L, o, w: L.ms3gpu_bandpass_filter_stream(4, 10, _lib.DTYPE_FLOAT32, None, ctypes.byref(o), None),
    lambda L, o, w: L.ms3gpu_bandpass_filter_stream(4, 10, _lib.DTYPE_FLOAT32, ctypes.byref(_io(read=False)),
                                                    ctypes.byref(o), None),
    lambda L, o, w: L.ms3gpu_bandpass_filter_stream(4, 10, _lib.DTYPE_FLOAT32, ctypes.byref(_io(write=False)),
                                                    ctypes.byref(o), None),
    lambda L, o, w: L.ms3gpu_bandpass_filter_stream(4, 10, -7, ctypes.byref(_io()), ctypes.byref(o), None),
    lambda L, o, w: L.ms3gpu_bandpass_filter_stream(4, 10, _lib.DTYPE_FLOAT32, ctypes.byref(_io(slab_bytes=-1)),
                                                    ctypes.byref(o), None),
    lambda L, o, w: L.ms3gpu_bandpass_filter_stream(-4, 10, _lib.DTYPE_FLOAT32, ctypes.byref(_io()),
                                                    ctypes.byref(o), None),
    lambda L, o, w: L.ms3gpu_bandpass_filter_stream(4, 10, _lib.DTYPE_FLOAT32, ctypes.byref(_io()), None, None),
    lambda L, o, w: L.ms3gpu_whiten_stream(4, 10, None, ctypes.byref(w), None),
    lambda L, o, w: L.ms3gpu_whiten_stream(4, 10, ctypes.byref(_io()), None, None),
    lambda L, o, w: L.ms3gpu_whiten_stream(4, 10, ctypes.byref(_io(write=False)), ctypes.byref(w), None),
    lambda L, o, w: L.ms3gpu_whiten_stream(4, 10, ctypes.byref(_io()), ctypes.byref(_lib.WhitenOpts(0, 7)), None),
    lambda L, o, w: L.ms3gpu_mask_out_artifacts_stream(4, 10, 0.0, 2000, ctypes.byref(_io()), None, None),
    lambda L, o, w: L.ms3gpu_mask_out_artifacts_stream(4, 10, 6.0, 0, ctypes.byref(_io()), None, None),
    lambda L, o, w: L.ms3gpu_mask_out_artifacts_stream(4, 10, 6.0, 2000, ctypes.byref(_io(write=False)), None, None),
])
def test_stream_arguments_rejected_before_device_work(make):
    """The streaming entry points check their callbacks, dtype, slab size,
    shape and options before any CUDA call or callback."""
    L = _lib.load()
    o = api.bandpass_opts(30000, 300, 6000, 1000, 0, 1, 16)
    w = _lib.WhitenOpts(0, 0)
    assert make(L, o, w) == _lib.ERR_INVALID
    assert _lib.last_error()


def test_bad_num_threads_rejected():
    L = _lib.load()
    o = api.bandpass_opts(30000, 300, 6000, 1000, 0, 1, 16)
    o.num_threads = 0
    buf = (ctypes.c_float * 40)()
    assert L.ms3gpu_bandpass_filter(buf, 4, 10, buf, ctypes.byref(o), None) == _lib.ERR_INVALID
    assert "num_threads" in _lib.last_error()
