"""Host logic of the time-sharded filter + whiten (no GPU): the window
partition over ranks, the rows each rank reads and writes, the rank-order
sum of the covariance exchange over gloo ranks, and the argument checks of
the slab entry points."""
import ctypes
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from mountainsort_b200 import _lib, api, sharded

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.parametrize("N,chunk,world", [(18_000_000, 120000, 8), (1_000_001, 120000, 3), (5, 120000, 4),
                                           (0, 120000, 2), (240000, 120000, 5)])
def test_window_ranges_partition_the_windows(N, chunk, world):
    nchunks = -(-N // chunk)
    ranges = [sharded.window_range(N, chunk, world, r) for r in range(world)]
    assert ranges[0][0] == 0 and ranges[-1][1] == nchunks
    assert all(a[1] == b[0] for a, b in zip(ranges, ranges[1:]))
    sizes = [c1 - c0 for c0, c1 in ranges]
    assert max(sizes) - min(sizes) <= 1


@pytest.mark.parametrize("M,N,world", [(384, 18_000_000, 8), (32, 1_000_001, 3), (7, 250000, 4), (16, 100, 2)])
def test_shards_read_their_halos_and_tile_the_output(M, N, world):
    T = max(16, 187 // M + 1)
    chunk = api.chunk_size(M, T)
    shards = [sharded.shard_of(M, N, T, world, r) for r in range(world)]
    # output rows tile [0, N) in rank order
    assert shards[0].out_row0 == 0 and shards[-1].out_row1 == N
    assert all(a.out_row1 == b.out_row0 for a, b in zip(shards, shards[1:]))
    for s in shards:
        if s.c0 == s.c1:
            continue
        assert s.in_row0 == max(0, s.c0 * chunk - 60000)
        assert s.in_row1 == min(N, s.c1 * chunk + 60000)
        assert s.in_row0 <= s.out_row0 <= s.out_row1 <= s.in_row1


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _sum_rank(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    from mountainsort_b200 import sharded as sh

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank order (1e16 + 1) - 1e16 = 0; other orders give 1
        t = torch.tensor([[1e16, 1.0, -1e16][rank], 2.0 * rank], dtype=torch.float64)
        q.put((rank, sh.sum_in_rank_order(t).tolist()))
    finally:
        dist.destroy_process_group()


def test_rank_order_sum_is_the_same_on_every_rank():
    world, port = 3, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_sum_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert [r[1] for r in res] == [[0.0, 6.0]] * world


@pytest.mark.parametrize("args", [
    dict(c_begin=0, c_end=10),      # beyond the recording's windows
    dict(c_begin=2, c_end=1),
    dict(row0=100000),              # the slab starts after the windows' first read
    dict(rows=10),                  # the slab ends before the windows' last read
    dict(out_row0=1),               # the output slab misses the first output row
    dict(in_dtype=-7),
])
def test_window_arguments_rejected_before_device_work(args):
    L = _lib.load()
    M, N = 4, 300000  # windows of 120000 (T = 47): 3 windows
    a = dict(in_dtype=_lib.DTYPE_FLOAT32, row0=0, rows=N, c_begin=0, c_end=3, out_row0=0, out_rows=N)
    a.update(args)
    o = api.bandpass_opts(30000, 300, 6000, 1000, 0, 1, 47)
    buf = (ctypes.c_float * 4)()
    rc = L.ms3gpu_bandpass_filter_windows(buf, a["in_dtype"], M, N, a["row0"], a["rows"], a["c_begin"], a["c_end"],
                                          buf, a["out_row0"], a["out_rows"], ctypes.byref(o), None)
    assert rc == _lib.ERR_INVALID
    assert _lib.last_error()
