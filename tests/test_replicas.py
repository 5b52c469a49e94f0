"""The multi-GPU form of the benchmark: independent replicas (one recording
per GPU, no data-path collective), timed as the maximum over the ranks.
The rank logic runs here as two gloo processes on the CPU."""
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dist.barrier()
        # each rank's own step time; rank 1 is the slow one
        mine = 100.0 + 50.0 * rank
        slowest = bench.max_over_ranks(dist, mine, torch.device("cpu"))
        value = bench.replica_throughput(world, 384, 18_000_000, 5, slowest)
        out.put((rank, mine, slowest, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_ranks_take_the_slowest_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(world))
    assert [r[0] for r in res] == [0, 1]
    # every rank sees the same slowest time and the same whole-job throughput
    assert all(r[2] == 150.0 for r in res)
    expect = 2 * 384 * 18_000_000 * 5 / 0.150 / 1e9
    assert all(r[3] == pytest.approx(expect, rel=1e-12) for r in res)


def test_single_process_needs_no_group():
    assert bench.max_over_ranks(None, 12.5, None) == 12.5
    assert bench.replica_throughput(1, 384, 18_000_000, 5, 1000.0) == pytest.approx(34.56)


def test_reference_arm_prints_on_rank_zero_only():
    # the other ranks of a torchrun launch exit 0 without work or output
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], capture_output=True, text=True, timeout=120, env=env)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
