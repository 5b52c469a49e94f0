"""Array-level API over the C ABI.

A timeseries of M channels and N timepoints is passed as an (N, M)
C-contiguous float32 array -- the .mda M x N column-major layout, one row of
M channels per timepoint.  numpy arrays live in host memory; torch tensors
may be on the host or on the current CUDA device.  Outputs are allocated
like the input (numpy -> numpy, torch -> torch on the same device) unless
`out` is given.  M x M matrices use matrix notation, W[i, j] = W(i, j).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib
from ._lib import BandpassOpts, WhitenOpts, check

try:  # torch is optional for host-only use
    import torch
except Exception:  # pragma: no cover
    torch = None


def default_num_threads() -> int:
    """The reference's omp_get_max_threads(): OMP_NUM_THREADS, else the
    number of hardware threads (p_bandpass_filter.cpp:147)."""
    v = os.environ.get("OMP_NUM_THREADS", "").split(",")[0].strip()
    if v.isdigit() and int(v) > 0:
        return int(v)
    return os.cpu_count() or 1


def _is_torch(x) -> bool:
    return torch is not None and isinstance(x, torch.Tensor)


def _ptr(x) -> int:
    if x is None:
        return 0
    if _is_torch(x):
        if not x.is_contiguous():
            raise ValueError("tensor must be contiguous")
        return x.data_ptr()
    if not x.flags["C_CONTIGUOUS"]:
        raise ValueError("array must be C-contiguous")
    return x.ctypes.data


def _stream_ptr(x, stream) -> int:
    if stream is not None:
        return int(getattr(stream, "cuda_stream", stream))
    if _is_torch(x) and x.is_cuda:
        return torch.cuda.current_stream(x.device).cuda_stream
    return 0


def _as_f32_rows(X):
    if _is_torch(X):
        if X.dtype != torch.float32:
            X = X.float()
        return X.contiguous()
    return np.ascontiguousarray(X, dtype=np.float32)


def _empty_like(X, shape, dtype):
    if _is_torch(X):
        tdt = {np.float32: torch.float32, np.int16: torch.int16, np.float64: torch.float64}[dtype]
        return torch.empty(shape, dtype=tdt, device=X.device)
    return np.empty(shape, dtype=dtype)


def _mat_in(W, like):
    """Matrix notation -> the column-major buffer the C ABI expects."""
    if _is_torch(W):
        return W.to(torch.float64).t().contiguous()
    return np.ascontiguousarray(np.asarray(W, dtype=np.float64).T)


def _mat_out(buf):
    return buf.t().contiguous() if _is_torch(buf) else np.ascontiguousarray(buf.T)


def bandpass_opts(samplerate, freq_min, freq_max, freq_wid=1000.0, quantization_unit=0.0,
                  subsample_factor=1, num_threads=None) -> BandpassOpts:
    return BandpassOpts(float(samplerate), float(freq_min), float(freq_max), float(freq_wid),
                        float(quantization_unit), int(subsample_factor or 1),
                        int(num_threads if num_threads else default_num_threads()))


def chunk_size(M: int, num_threads: int) -> int:
    return int(_lib.load().ms3gpu_bandpass_chunk_size(M, num_threads))


def bandpass_filter(X, samplerate, freq_min, freq_max, freq_wid=1000.0, quantization_unit=0.0,
                    subsample_factor=1, num_threads=None, out=None, stream=None):
    """ms3.bandpass_filter (packages/ms3/p_bandpass_filter.cpp:115-229) on an
    (N, M) array; returns (N // subsample_factor, M) float32, or int16 when
    quantization_unit != 0.  An int16 array is filtered as the reference
    reads an int16 file (converted to float), without a float copy of it."""
    L = _lib.load()
    i16 = (_is_torch(X) and X.dtype == torch.int16) or (not _is_torch(X) and np.asarray(X).dtype == np.int16)
    if i16:
        X = X.contiguous() if _is_torch(X) else np.ascontiguousarray(X)
    else:
        X = _as_f32_rows(X)
    N, M = X.shape
    o = bandpass_opts(samplerate, freq_min, freq_max, freq_wid, quantization_unit, subsample_factor,
                      num_threads)
    Mo, No, dt = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int32()
    check(L.ms3gpu_bandpass_output_dims(M, N, ctypes.byref(o), ctypes.byref(Mo), ctypes.byref(No),
                                        ctypes.byref(dt)))
    if out is None:
        out_i16 = dt.value == _lib.DTYPE_INT16 or (i16 and float(freq_max) == 0)
        out = _empty_like(X, (No.value, Mo.value), np.int16 if out_i16 else np.float32)
    fn = L.ms3gpu_bandpass_filter_i16 if i16 else L.ms3gpu_bandpass_filter
    check(fn(_ptr(X), M, N, _ptr(out), ctypes.byref(o), _stream_ptr(X, stream)))
    return out


_PRECISION = {"plain": _lib.PRECISION_PLAIN, "mixed": _lib.PRECISION_MIXED}


def whiten(X, quantization_unit=0.0, out=None, stream=None, precision="plain"):
    """ms3.whiten (packages/ms3/p_whiten.cpp:45-206) on an (N, M) array.
    precision "plain" (FP32, parity with the reference) or "mixed"
    (tensor-core 3-term TF32 apply)."""
    L = _lib.load()
    X = _as_f32_rows(X)
    N, M = X.shape
    if out is None:
        out = _empty_like(X, (N, M), np.int16 if quantization_unit > 0 else np.float32)
    o = WhitenOpts(float(quantization_unit), _PRECISION[precision])
    check(L.ms3gpu_whiten(_ptr(X), M, N, _ptr(out), ctypes.byref(o), _stream_ptr(X, stream)))
    return out


def _stream_io(M, source, sink, in_dtype, out_dtype, slab_bytes, errors):
    """An ms3gpu_stream_io over Python callables: source(t0, nt) returns the
    input timepoints [t0, t0 + nt) as an (nt, M) array; sink(t0, rows)
    receives output timepoints as an (nt, M) array valid only during the
    call.  An exception in either stops the call; it is kept in `errors`."""
    in_ct = ctypes.c_int16 if np.dtype(in_dtype) == np.int16 else ctypes.c_float
    out_ct = ctypes.c_int16 if np.dtype(out_dtype) == np.int16 else ctypes.c_float

    def rd(_ctx, t0, nt, dst):
        try:
            block = np.ctypeslib.as_array(ctypes.cast(dst, ctypes.POINTER(in_ct)), shape=(nt, M))
            block[...] = source(t0, nt)
            return 0
        except BaseException as e:  # noqa: BLE001 -- raised again after the call
            errors.append(e)
            return 1

    def wr(_ctx, t0, nt, src):
        try:
            sink(t0, np.ctypeslib.as_array(ctypes.cast(src, ctypes.POINTER(out_ct)), shape=(nt, M)))
            return 0
        except BaseException as e:  # noqa: BLE001
            errors.append(e)
            return 1

    return _lib.StreamIO(_lib.READ_FN(rd), None, _lib.WRITE_FN(wr), None, int(slab_bytes))


def _run_stream(call, errors):
    rc = call()
    if errors:
        raise errors[0]
    check(rc)


def bandpass_filter_stream(source, sink, M, N, samplerate, freq_min, freq_max, freq_wid=1000.0,
                           quantization_unit=0.0, subsample_factor=1, num_threads=None, in_dtype=np.float32,
                           slab_bytes=0, stream=None):
    """ms3.bandpass_filter over a recording read and written block by block,
    as the processor's chunk loop does (p_bandpass_filter.cpp:160-220).
    source(t0, nt) returns input timepoints [t0, t0 + nt) as an (nt, M)
    array (converted to in_dtype: float32, or int16 for an int16
    recording); sink(t0, rows) receives output timepoints [t0, t0 + len(rows))
    (float32, or int16 when quantization_unit != 0; the input's dtype when
    freq_max == 0), in increasing t0.  The values equal bandpass_filter's.
    slab_bytes: about how many input bytes one block holds (0 = 1 GiB)."""
    L = _lib.load()
    o = bandpass_opts(samplerate, freq_min, freq_max, freq_wid, quantization_unit, subsample_factor,
                      num_threads)
    i16 = np.dtype(in_dtype) == np.int16
    if float(freq_max) == 0:
        out_dt = np.int16 if i16 else np.float32
    else:
        out_dt = np.int16 if float(quantization_unit) != 0 else np.float32
    errors = []
    io = _stream_io(int(M), source, sink, np.int16 if i16 else np.float32, out_dt, slab_bytes, errors)
    dt = _lib.DTYPE_INT16 if i16 else _lib.DTYPE_FLOAT32
    _run_stream(lambda: L.ms3gpu_bandpass_filter_stream(int(M), int(N), dt, ctypes.byref(io), ctypes.byref(o),
                                                        _stream_ptr(None, stream)), errors)


def whiten_stream(source, sink, M, N, quantization_unit=0.0, slab_bytes=0, stream=None, precision="plain"):
    """ms3.whiten over a float32 recording read block by block, twice (the
    covariance pass, then the apply pass, p_whiten.cpp:64-206), written
    block by block through sink (int16 when quantization_unit > 0).
    Callbacks as in bandpass_filter_stream; the values equal whiten's."""
    L = _lib.load()
    o = WhitenOpts(float(quantization_unit), _PRECISION[precision])
    errors = []
    io = _stream_io(int(M), source, sink, np.float32, np.int16 if quantization_unit > 0 else np.float32,
                    slab_bytes, errors)
    _run_stream(lambda: L.ms3gpu_whiten_stream(int(M), int(N), ctypes.byref(io), ctypes.byref(o),
                                               _stream_ptr(None, stream)), errors)


def mask_out_artifacts_stream(source, sink, M, N, threshold=6.0, interval_size=2000, slab_bytes=0, stream=None):
    """ms3.mask_out_artifacts over a float32 recording read block by block,
    twice (the interval norms, then the masked copy), written through sink.
    Callbacks as in bandpass_filter_stream.  Returns the timepoints kept; the
    values equal mask_out_artifacts'."""
    L = _lib.load()
    errors = []
    io = _stream_io(int(M), source, sink, np.float32, np.float32, slab_bytes, errors)
    kept = ctypes.c_int64()
    _run_stream(lambda: L.ms3gpu_mask_out_artifacts_stream(int(M), int(N), float(threshold), int(interval_size),
                                                           ctypes.byref(io), ctypes.byref(kept),
                                                           _stream_ptr(None, stream)), errors)
    return kept.value


def bandpass_whiten(X, samplerate, freq_min, freq_max, freq_wid=1000.0, num_threads=None,
                    quantization_unit=0.0, filt_out=None, out=None, want_filt=False, stream=None,
                    precision="plain"):
    """ms3.bandpass_filter followed by ms3.whiten, as mountainsort3.mlp runs
    them.  Returns pre, or (filt, pre) when want_filt or filt_out is given."""
    L = _lib.load()
    X = _as_f32_rows(X)
    N, M = X.shape
    bp = bandpass_opts(samplerate, freq_min, freq_max, freq_wid, 0.0, 1, num_threads)
    wh = WhitenOpts(float(quantization_unit), _PRECISION[precision])
    if want_filt and filt_out is None:
        filt_out = _empty_like(X, (N, M), np.float32)
    if out is None:
        out = _empty_like(X, (N, M), np.int16 if quantization_unit > 0 else np.float32)
    check(L.ms3gpu_bandpass_whiten(_ptr(X), M, N, _ptr(filt_out), _ptr(out), ctypes.byref(bp),
                                   ctypes.byref(wh), _stream_ptr(X, stream)))
    return (filt_out, out) if filt_out is not None else out


def bandpass_whiten_batch(recordings, stream=None, precision="plain"):
    """Many recordings through ms3.bandpass_filter + ms3.whiten at once
    (ms3gpu_bandpass_whiten_batch): `recordings` is a list of dicts with keys
    X ((N, M) array) and samplerate, freq_min, freq_max, optional freq_wid,
    num_threads, quantization_unit (of the whiten step).  Returns the list of
    whitened outputs; raises on the first failing job after all have run."""
    L = _lib.load()
    jobs = (_lib.Job * len(recordings))()
    keep = []
    outs = []
    for k, r in enumerate(recordings):
        X = _as_f32_rows(r["X"])
        N, M = X.shape
        q = float(r.get("quantization_unit", 0.0))
        out = _empty_like(X, (N, M), np.int16 if q > 0 else np.float32)
        keep.append(X)
        outs.append(out)
        j = jobs[k]
        j.timeseries = _ptr(X)
        j.M, j.N = M, N
        j.filt_out = None
        j.pre_out = _ptr(out)
        j.bp = bandpass_opts(r["samplerate"], r["freq_min"], r["freq_max"], r.get("freq_wid", 1000.0), 0.0, 1,
                             r.get("num_threads"))
        j.wh = WhitenOpts(q, _PRECISION[precision])
    s = _stream_ptr(keep[0], stream) if keep else 0
    check(L.ms3gpu_bandpass_whiten_batch(jobs, len(recordings), s))
    return outs


def whiten_covariance(X, stream=None):
    """XXt = sum_t x_t x_t^T / (N-1) (p_whiten.cpp:64-118), M x M float64."""
    L = _lib.load()
    X = _as_f32_rows(X)
    N, M = X.shape
    buf = _empty_like(X, (M, M), np.float64)
    check(L.ms3gpu_whiten_covariance(_ptr(X), M, N, _ptr(buf), _stream_ptr(X, stream)))
    return _mat_out(buf)


def whitening_matrix(XXt, stream=None, return_components=False):
    """whitening_matrix_from_XXt (pca.cpp:635-651).  Returns W, or
    (W, components, sigma) when return_components."""
    L = _lib.load()
    C = _mat_in(XXt, XXt)
    M = C.shape[0]
    W = _empty_like(C, (M, M), np.float64)
    comps = _empty_like(C, (M, M), np.float64) if return_components else None
    sig = _empty_like(C, (M,), np.float64) if return_components else None
    check(L.ms3gpu_whitening_matrix(_ptr(C), M, _ptr(W), _ptr(comps), _ptr(sig), _stream_ptr(C, stream)))
    if return_components:
        return _mat_out(W), _mat_out(comps), sig
    return _mat_out(W)


def apply_whitening_matrix(X, W, quantization_unit=0.0, out=None, stream=None, precision="plain"):
    """Whiten pass 2 (p_whiten.cpp:153-206) with a given W."""
    L = _lib.load()
    X = _as_f32_rows(X)
    N, M = X.shape
    Wc = _mat_in(W, X)
    if out is None:
        out = _empty_like(X, (N, M), np.int16 if quantization_unit > 0 else np.float32)
    check(L.ms3gpu_apply_whitening_matrix(_ptr(X), M, N, _ptr(Wc), float(quantization_unit),
                                          _PRECISION[precision], _ptr(out), _stream_ptr(X, stream)))
    return out


def compute_whitening_matrix(X_list, channels=None, stream=None):
    """ms3.compute_whitening_matrix (p_whiten.cpp:208-298): the whitening
    matrix of the recordings in X_list -- (N_i, M) arrays, concatenated in
    time -- restricted to `channels` (1-based channel numbers) when given."""
    L = _lib.load()
    if not X_list:
        raise ValueError("X_list is empty")
    arrs = [_as_f32_rows(X) for X in X_list]
    M = arrs[0].shape[1]
    if any(a.ndim != 2 or a.shape[1] != M for a in arrs):
        raise ValueError("all recordings need the same number of channels")
    ptrs = (ctypes.c_void_p * len(arrs))(*[_ptr(a) for a in arrs])
    Ns = (ctypes.c_int64 * len(arrs))(*[a.shape[0] for a in arrs])
    ch = np.ascontiguousarray(channels if channels is not None else [], dtype=np.int32)
    M2 = len(ch) if len(ch) else M
    W = _empty_like(arrs[0], (M2, M2), np.float64)
    check(L.ms3gpu_compute_whitening_matrix(ctypes.cast(ptrs, ctypes.c_void_p), ctypes.cast(Ns, ctypes.c_void_p),
                                            len(arrs), M, ch.ctypes.data if len(ch) else None, len(ch), _ptr(W),
                                            _stream_ptr(arrs[0], stream)))
    return _mat_out(W)


def whiten_blocks(X, blocks, quantization_unit=0.0, out=None, stream=None, precision="plain"):
    """ms3.whiten per channel block (ms3gpu_whiten_blocks): `blocks` is a list
    of 1-based channel-number lists that together name every channel once
    (e.g. the shanks of a probe); each block is whitened on its own."""
    L = _lib.load()
    X = _as_f32_rows(X)
    N, M = X.shape
    ch = np.ascontiguousarray(np.concatenate([np.asarray(b, dtype=np.int32) for b in blocks]), dtype=np.int32)
    sizes = np.ascontiguousarray([len(b) for b in blocks], dtype=np.int32)
    if out is None:
        out = _empty_like(X, (N, M), np.int16 if quantization_unit > 0 else np.float32)
    o = WhitenOpts(float(quantization_unit), _PRECISION[precision])
    check(L.ms3gpu_whiten_blocks(_ptr(X), M, N, ch.ctypes.data, sizes.ctypes.data, len(blocks), _ptr(out),
                                 ctypes.byref(o), _stream_ptr(X, stream)))
    return out


def mask_out_artifacts(X, threshold=6.0, interval_size=2000, out=None, stream=None, return_kept=False):
    """ms3.mask_out_artifacts (p_mask_out_artifacts.cpp:24-104) on an (N, M)
    array: intervals whose norm is an outlier on any channel are zeroed with
    their neighbours.  Returns the masked array (and the number of
    timepoints kept when return_kept)."""
    L = _lib.load()
    X = _as_f32_rows(X)
    N, M = X.shape
    if out is None:
        out = _empty_like(X, (N, M), np.float32)
    kept = ctypes.c_int64()
    check(L.ms3gpu_mask_out_artifacts(_ptr(X), M, N, float(threshold), int(interval_size), _ptr(out),
                                      ctypes.addressof(kept), _stream_ptr(X, stream)))
    return (out, kept.value) if return_kept else out


def detect_events(X, detect_threshold=3.0, detect_interval=10.0, detect_sign=0, chunk_size=0, stream=None):
    """Event detection of mountainsortalg (detect_events.cpp:69-135 over the
    time chunks of p_mountainsort3.cpp:190-215) for every channel of an
    (N, M) array.  Returns a list of M int64 arrays of event timepoints."""
    L = _lib.load()
    X = _as_f32_rows(X)
    N, M = X.shape
    counts = np.zeros(max(M, 1), np.int64)
    args = (_ptr(X), M, N, float(detect_threshold), float(detect_interval), int(detect_sign), int(chunk_size))
    # room for 1% of the samples as events; a second call only when that is too little
    cap = max(1024, (N * M) // 100)
    times = np.empty(cap, np.int64)
    rc = L.ms3gpu_detect_events(*args, counts.ctypes.data, times.ctypes.data, cap, _stream_ptr(X, stream))
    total = int(counts[:M].sum())
    if rc == _lib.ERR_INVALID and total > cap:
        times = np.empty(total, np.int64)
        rc = L.ms3gpu_detect_events(*args, counts.ctypes.data, times.ctypes.data, total, _stream_ptr(X, stream))
    check(rc)
    return np.split(times[:total], np.cumsum(counts[:M])[:-1]) if M else []


def whiten_clips(clips, W, quantization_unit=0.0, out=None, stream=None, precision="plain"):
    """ms3.whiten_clips (p_whiten.cpp:300-345): clips as an (L, T, M) array
    (the .mda M x T x L layout); W^T x at every timepoint, no 1e-4 rounding;
    int16 when quantization_unit > 0."""
    L_ = _lib.load()
    c = _as_f32_rows(clips)
    if c.ndim != 3:
        raise ValueError("clips must be (L, T, M)")
    L, T, M = c.shape
    Wc = _mat_in(W, c)
    if out is None:
        out = _empty_like(c, (L, T, M), np.int16 if quantization_unit > 0 else np.float32)
    check(L_.ms3gpu_whiten_clips(_ptr(c), M, T, L, _ptr(Wc), float(quantization_unit), _PRECISION[precision],
                                 _ptr(out), _stream_ptr(c, stream)))
    return out


def release_cached_memory():
    """Hands the device memory the library keeps between calls back to the
    driver (ms3gpu_release_cached_memory), e.g. before allocating large
    arrays with another allocator."""
    check(_lib.load().ms3gpu_release_cached_memory())


def requirements(processor: str, M: int, N: int, **params) -> float:
    """The processor's peak-RAM model in MB (its "requirements" answer)."""
    L = _lib.load()
    mb = ctypes.c_double()
    if processor == "ms3.bandpass_filter":
        o = bandpass_opts(params.get("samplerate", 0), params.get("freq_min", 0), params.get("freq_max", 0),
                          params.get("freq_wid", 1000), params.get("quantization_unit", 0),
                          params.get("subsample_factor", 1), params.get("num_threads"))
        check(L.ms3gpu_bandpass_requirements(M, N, ctypes.byref(o), ctypes.byref(mb)))
    elif processor == "ms3.whiten":
        check(L.ms3gpu_whiten_requirements(M, N, ctypes.byref(mb)))
    else:
        raise ValueError(f"unknown processor {processor}")
    return mb.value
