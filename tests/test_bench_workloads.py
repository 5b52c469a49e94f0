"""The benchmark's workloads are the configurations they are named for
(CPU only: nothing here launches a kernel)."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_headline_and_cpu_size_workloads():
    assert bench.SIZES["c2"][:2] == (384, 18_000_000)  # 10 min at 30 kHz
    assert bench.SIZES["c1"][:2] == (32, 1_800_000)    # 60 s at 30 kHz
    assert (bench.FS, bench.FMIN, bench.FMAX, bench.FWID) == (30000.0, 300.0, 6000.0, 1000.0)
    assert bench.GEOM_T == 16


def test_batched_uneven_workload():
    jobs = bench.c4_jobs()
    assert len(jobs) == 48
    assert bench.c4_jobs() == jobs  # seeded
    for M, N, fs, fmax in jobs:
        assert M in (16, 32, 64, 128, 384)
        assert fs in (20000.0, 30000.0)
        assert 30.0 <= N / fs <= 1200.0
        assert fmax == min(6000.0, 0.4 * fs)
    assert len({j[0] for j in jobs}) == 5 and len({j[2] for j in jobs}) == 2


def test_c5_record_is_four_shanks_of_384_for_five_minutes():
    import inspect

    src = inspect.getsource(bench.c5_record)
    assert "M1, N, S = 384, 9_000_000, 4" in src  # 5 min at 30 kHz, 4 shanks
    assert "0.195" in src                          # int16 gain
