"""ms3.bandpass_filter + ms3.whiten of one recording split along time over
several GPUs (one process per GPU, torch.distributed for the exchange).

The filter's windows (chunks) are independent and the covariance of whiten
pass 1 (p_whiten.cpp:64-118) is a sum over time, so each rank

1. filters its own contiguous range of windows from a slab of the recording
   that includes the windows' 60000-timepoint halos
   (ms3gpu_bandpass_filter_windows: the same kernels on the same windows as
   the one-GPU call, identical filtered values);
2. sums x x^T over its own filtered timepoints (ms3gpu_whiten_covariance_sum);
3. exchanges the M x M FP64 sums -- the one collective of the path, an
   all-gather whose parts every rank adds in rank order, so that every rank
   holds the same total bit for bit whatever order the collective library
   reduces in;
4. forms W from total / (N - 1) (deterministic: identical on every rank) and
   whitens its own timepoints.

The whitened values equal the one-GPU call's up to the grouping of the FP64
covariance additions (W moves by ~1e-8 relative at 384 channels).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib, api
from ._lib import check

OVERLAP = 60000  # halo of a window on each side (p_bandpass_filter.cpp:147)


def window_range(N: int, chunk: int, world: int, rank: int):
    """Windows [c0, c1) of `rank` out of `world`: contiguous ranges in rank
    order whose sizes differ by at most one."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world {world}")
    nchunks = -(-N // chunk) if N > 0 else 0
    base, extra = divmod(nchunks, world)
    c0 = rank * base + min(rank, extra)
    return c0, c0 + base + (1 if rank < extra else 0)


@dataclass(frozen=True)
class Shard:
    """A rank's windows [c0, c1), the input timepoints they read [in_row0,
    in_row1) and the output timepoints they produce [out_row0, out_row1)."""
    c0: int
    c1: int
    in_row0: int
    in_row1: int
    out_row0: int
    out_row1: int


def shard_of(M: int, N: int, num_threads: int, world: int, rank: int) -> Shard:
    chunk = api.chunk_size(M, num_threads)
    c0, c1 = window_range(N, chunk, world, rank)
    if c0 == c1:
        t = min(N, c0 * chunk)
        return Shard(c0, c1, t, t, t, t)
    return Shard(c0, c1, max(0, c0 * chunk - OVERLAP), min(N, c1 * chunk + OVERLAP), min(N, c0 * chunk),
                 min(N, c1 * chunk))


def filter_windows(X_slab, shard: Shard, M: int, N: int, samplerate, freq_min, freq_max, freq_wid=1000.0,
                   num_threads=None, stream=None):
    """The filtered timepoints [shard.out_row0, shard.out_row1) from the input
    timepoints [shard.in_row0, shard.in_row1) in X_slab ((rows, M) float32 or
    int16, host or device), as the one-GPU ms3.bandpass_filter gives them."""
    L = _lib.load()
    i16 = (api._is_torch(X_slab) and str(X_slab.dtype) == "torch.int16") or \
        (not api._is_torch(X_slab) and np.asarray(X_slab).dtype == np.int16)
    X_slab = (X_slab.contiguous() if api._is_torch(X_slab) else np.ascontiguousarray(X_slab)) if i16 \
        else api._as_f32_rows(X_slab)
    rows = shard.in_row1 - shard.in_row0
    if X_slab.shape[0] != rows or (rows and X_slab.shape[1] != M):
        raise ValueError(f"slab of shape {tuple(X_slab.shape)}, expected ({rows}, {M})")
    out_rows = shard.out_row1 - shard.out_row0
    out = api._empty_like(X_slab, (out_rows, M), np.float32)
    o = api.bandpass_opts(samplerate, freq_min, freq_max, freq_wid, 0.0, 1, num_threads)
    check(L.ms3gpu_bandpass_filter_windows(api._ptr(X_slab), _lib.DTYPE_INT16 if i16 else _lib.DTYPE_FLOAT32, M, N,
                                           shard.in_row0, rows, shard.c0, shard.c1, api._ptr(out), shard.out_row0,
                                           out_rows, ctypes.byref(o), api._stream_ptr(X_slab, stream)))
    return out


def covariance_sum(filt_rows, stream=None):
    """sum_t x_t x_t^T over the given (n, M) float32 timepoints, M x M float64
    (no division)."""
    L = _lib.load()
    X = api._as_f32_rows(filt_rows)
    n, M = X.shape
    buf = api._empty_like(X, (M, M), np.float64)
    check(L.ms3gpu_whiten_covariance_sum(api._ptr(X), M, n, api._ptr(buf), api._stream_ptr(X, stream)))
    return api._mat_out(buf)


def sum_in_rank_order(t, group=None):
    """The sum of every rank's tensor `t`, added in rank order after an
    all-gather: the same bits on every rank, whatever order the collective
    library would reduce in."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    parts = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(parts, t.contiguous(), group=group)
    total = parts[0].clone()
    for p in parts[1:]:
        total += p
    return total


def whitening_from_sum(total_sum, N: int, stream=None):
    """W of whitening_matrix_from_XXt (pca.cpp:635-651) for XXt = total /
    (N - 1) (no division for N <= 1), as p_whiten.cpp:112-118 divides."""
    XXt = total_sum / float(N - 1) if N > 1 else total_sum
    return api.whitening_matrix(XXt, stream=stream)


def bandpass_whiten_shard(X_slab, M: int, N: int, samplerate, freq_min, freq_max, freq_wid=1000.0,
                          num_threads=None, quantization_unit=0.0, precision="plain", group=None, stream=None):
    """This rank's part of ms3.bandpass_filter + ms3.whiten of an M x N
    recording split over the ranks of `group` (torch.distributed, one GPU per
    rank; tensors on the rank's current CUDA device).  X_slab holds the input
    timepoints [shard.in_row0, shard.in_row1) of shard_of(M, N, num_threads,
    world, rank).  Returns (shard, filt, pre): the filtered and whitened
    timepoints [shard.out_row0, shard.out_row1).  Every rank calls it (the
    covariance exchange is collective)."""
    import torch
    import torch.distributed as dist

    world, rank = dist.get_world_size(group), dist.get_rank(group)
    T = num_threads if num_threads else api.default_num_threads()
    shard = shard_of(M, N, T, world, rank)
    filt = filter_windows(X_slab, shard, M, N, samplerate, freq_min, freq_max, freq_wid, T, stream)
    part = covariance_sum(filt, stream)
    if not api._is_torch(part):
        part = torch.from_numpy(np.ascontiguousarray(part))
    total = sum_in_rank_order(part, group)
    W = whitening_from_sum(total, N, stream)
    pre = api.apply_whitening_matrix(filt, W, quantization_unit, stream=stream, precision=precision)
    return shard, filt, pre
