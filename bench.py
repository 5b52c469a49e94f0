#!/usr/bin/env python3
"""Benchmark: ms3.bandpass_filter + ms3.whiten on one B200 (or N, weak scaling).

Workload (default): 384 channels x 18,000,000 timepoints (10 min at 30 kHz,
27.6 GB float32), seeded synthetic recording (correlated noise + 1/f LFP +
300 biphasic units), filter 300-6000 Hz, freq_wid 1000, chunk geometry of
T = 16 threads (chunk 120000, FFT window 240000).  One step = the fused
bandpass -> covariance -> whitening matrix -> apply pass over the whole
recording, inputs resident in HBM (27.6 GB > 126 MB L2, so no L2 flush is
needed between steps).

Metric: Gch-samples/s (one ch-sample = one channel at one timepoint of
output).  `e2e` is the same metric through the C ABI with pinned host
buffers: the host->device copy of the raw recording and the device->host copy
of the whitened output happen inside every timed step.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FS, FMIN, FMAX, FWID = 30000.0, 300.0, 6000.0, 1000.0
GEOM_T = 16
METRIC = "Gch-samples/s bandpass+whiten"
UNIT = "Gch-samples/s"

SIZES = {
    # name: (M, N, units, description)
    "c2": (384, 18_000_000, 300, "384ch x 18M timepoints (10 min @ 30 kHz), plain FP32 form"),
    "c1": (32, 1_800_000, 20, "32ch x 1.8M timepoints (60 s @ 30 kHz), CPU-runnable size"),
    "small": (384, 600_000, 20, "384ch x 600k timepoints (20 s @ 30 kHz), profiling case"),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception as e:  # pragma: no cover
            log("clock sampler unavailable:", e)
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sms, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 8:
                continue
            try:
                sms.append(float(p[0]))
                mx = float(p[1])
            except ValueError:
                continue
            for n, v in zip(names, p[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sms) if sms else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sms)}


# ----------------------------------------------------------------- CPU baseline

class CpuReference:
    """The reference's CPU path timed on this host's cores.

    Where oracle/_ref/libmsref.so exists (the reference's own
    packages/ms3/p_bandpass_filter.cpp, p_whiten.cpp and pca.cpp compiled from
    its sources; its FFT interface runs the oracle's FFT), the bandpass
    processor and the whitening matrix run that code; otherwise ref32, the
    restatement that reproduces it bit for bit.  The whitening loops (pass 1
    XX^T and pass 2 apply, p_whiten.cpp:75-113,153-206) run ref32's copy of
    them, one slice per thread on every thread at once, as the reference's
    OpenMP loop gives each thread its own chunk.

    A full 384 x 18M recording takes the reference about 15 minutes on 16
    cores (the apply alone is ~0.7 ms per timepoint per thread), so one
    measured sample is:
      * bandpass: one parallel round of the reference geometry (T chunks of
        `chunk` timepoints, one per thread), file to file through the
        processor (page-cache I/O included, as the reference runs);
      * whiten loops: T threads x `wh_rows` timepoints each, pass 1 and pass 2;
      * the whitening matrix at the real M, once per process (O(M^4), serial).
    The recording's time is then rounds x each part + the matrix; the value is
    M*N / that time.  ms_per_step is the wall time of one measured sample."""

    def __init__(self, M, N, threads, wh_rows=6250):
        import numpy as np

        from oracle import ref32, refpin

        self.np, self.ref32, self.refpin = np, ref32, refpin
        self.M, self.N, self.T = M, N, max(1, threads)
        self.kind = "reference" if refpin.available() else "port"
        self.chunk = ref32.chunk_size(M, GEOM_T)
        self.wh_rows = wh_rows
        rng = np.random.default_rng(1)
        # one parallel round of the bandpass geometry, written once as the processor's input file
        self.tmp = tempfile.mkdtemp(prefix="ms3ref_")
        rows = self.T * self.chunk
        X = (10 * rng.standard_normal((rows, M))).astype(np.float32)
        self.bp_in = os.path.join(self.tmp, "raw.mda")
        from mountainsort_b200 import mdaio

        mdaio.writemda(X.T, self.bp_in)
        self.wh = [np.ascontiguousarray(X[k * wh_rows:(k + 1) * wh_rows]) for k in range(self.T)]
        del X
        # the whitening matrix at the real channel count (serial O(M^4) power iteration)
        C = np.cov(rng.standard_normal((M, 4 * M))) + np.eye(M)
        t0 = time.perf_counter()
        if self.kind == "reference":
            refpin.whitening_matrix(C)
        else:
            ref32.whitening_matrix(C)
        self.t_W = time.perf_counter() - t0
        self.samples = []

    def sample(self):
        from concurrent.futures import ThreadPoolExecutor

        np, ref32, refpin = self.np, self.ref32, self.refpin
        t0 = time.perf_counter()
        out = os.path.join(self.tmp, "filt.mda")
        if os.path.exists(out):
            os.remove(out)
        if self.kind == "reference":
            if refpin.lib().msref_bandpass_filter(self.bp_in.encode(), out.encode(), FS, FMIN, FMAX, FWID, 0.0, 1,
                                                  GEOM_T) != 0:
                raise RuntimeError("reference bandpass processor failed")
        else:
            from mountainsort_b200 import mdaio

            X = np.ascontiguousarray(mdaio.readmda(self.bp_in).T)
            mdaio.writemda(ref32.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=GEOM_T,
                                                 exec_threads=self.T).T, out)
        t_bp = time.perf_counter() - t0
        W = np.eye(self.M)
        t1 = time.perf_counter()
        with ThreadPoolExecutor(self.T) as ex:  # the ctypes calls release the GIL
            list(ex.map(lambda Y: ref32.whiten_xxt(Y, exec_threads=1), self.wh))
        t_xxt = time.perf_counter() - t1
        t2 = time.perf_counter()
        with ThreadPoolExecutor(self.T) as ex:
            list(ex.map(lambda Y: ref32.whiten_apply(Y, W, exec_threads=1), self.wh))
        t_apply = time.perf_counter() - t2
        rec = {"bp": t_bp, "xxt": t_xxt, "apply": t_apply, "wall": time.perf_counter() - t0}
        self.samples.append(rec)
        return rec

    def total_seconds(self, rec):
        rounds = -(-self.N // (self.T * self.chunk))
        # the whitening loops run on 100000-timepoint chunks, one per thread per round
        wrounds = -(-self.N // (self.T * 100000)) * (100000 / self.wh_rows)
        return rounds * rec["bp"] + wrounds * (rec["xxt"] + rec["apply"]) + self.t_W

    def describe(self, rec):
        src = ("the reference's own processor code (oracle/_ref) for the bandpass and the whitening matrix"
               if self.kind == "reference" else "ref32 (the bit-identical restatement)")
        return (f"{src}; {self.T} threads on this host: bandpass processor file to file on one parallel round "
                f"({self.T} chunks of {self.chunk} x {self.M}ch, {rec['bp']:.2f} s); whiten pass 1 / pass 2 loops "
                f"on {self.T} x {self.wh_rows} timepoints at once ({rec['xxt']:.2f} s / {rec['apply']:.2f} s; "
                f"{len(self.samples) * self.T * self.wh_rows} timepoints measured in all); whitening matrix at "
                f"M={self.M}: {self.t_W:.1f} s once; recording time {self.total_seconds(rec):.1f} s for "
                f"{self.M}x{self.N} = rounds x measured parts + matrix")

    def close(self):
        import shutil

        shutil.rmtree(self.tmp, ignore_errors=True)


def cpu_threads():
    return max(1, int(os.environ.get("MS3_BENCH_CPU_THREADS", str(os.cpu_count() or 1))))


def cpu_baseline(M: int, N: int, threads: int):
    """One measured sample of the CPU reference (see CpuReference)."""
    ref = CpuReference(M, N, threads)
    try:
        rec = ref.sample()
        total = ref.total_seconds(rec)
        return {"value": M * N / total / 1e9, "unit": UNIT, "cores": ref.T, "kind": ref.kind,
                "sample": ref.describe(rec)}
    finally:
        ref.close()


def reference_c1_full(threads):
    """The CPU-runnable size (32 x 1.8M, 60 s at 30 kHz) run in full through
    the reference's own processors, file to file: bandpass then whiten."""
    import numpy as np

    from mountainsort_b200 import mdaio, synth
    from oracle import refpin

    if not refpin.available():
        return None
    M, N = 32, 1_800_000
    X = synth.generate_numpy(M, N, K=20, seed=0, sites=(3, 6))
    tmp = tempfile.mkdtemp(prefix="ms3ref_c1_")
    try:
        pin, pf, pp = (os.path.join(tmp, n) for n in ("raw.mda", "filt.mda", "pre.mda"))
        mdaio.writemda(X.T, pin)
        L = refpin.lib()
        t0 = time.perf_counter()
        if L.msref_bandpass_filter(pin.encode(), pf.encode(), FS, FMIN, FMAX, FWID, 0.0, 1, GEOM_T) != 0:
            return None
        t1 = time.perf_counter()
        if L.msref_whiten(pf.encode(), pp.encode(), 0.0, threads) != 0:
            return None
        t2 = time.perf_counter()
        return {"workload": "32ch x 1.8M timepoints (60 s @ 30 kHz), timed in full",
                "value": M * N / (t2 - t0) / 1e9, "unit": UNIT, "seconds": t2 - t0,
                "bandpass_s": t1 - t0, "whiten_s": t2 - t1, "kind": "reference", "cores": threads,
                "geometry_threads": GEOM_T}
    finally:
        import shutil

        shutil.rmtree(tmp, ignore_errors=True)


def run_reference_arm(args, size):
    M, N, _, desc = SIZES[size]
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = cpu_threads()
    t_start = time.perf_counter()
    c1 = reference_c1_full(threads)
    ref = CpuReference(M, N, threads)
    try:
        vals, walls = [], []
        for i in range(args.warmup + args.steps):
            rec = ref.sample()
            if i >= args.warmup:
                vals.append(M * N / ref.total_seconds(rec) / 1e9)
                walls.append(rec["wall"])
        v = statistics.median(vals)
        cb = {"value": v, "unit": UNIT, "cores": ref.T, "kind": ref.kind, "sample": ref.describe(rec)}
    finally:
        ref.close()
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": statistics.mean(walls) * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": desc, "M": M, "N": N, "geometry_threads": GEOM_T, "freq": [FMIN, FMAX, FWID]},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timing": ("ms_per_step is the wall time of one measured sample (see cpu_baseline.sample); value is "
                   "the recording's throughput from those measurements"),
        "cpu_size_full": c1,
        "wall_s": time.perf_counter() - t_start,
    }
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------- replicas

def max_over_ranks(dist, x, device):
    """The slowest rank's figure: every timing of a multi-GPU run is the
    maximum over the ranks (all ranks take part, rank order does not matter)."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, M, N, steps, ms_total):
    """Whole-job Gch-samples/s of `world` replicas, each filtering and
    whitening its own M x N recording `steps` times in ms_total (the max over
    ranks)."""
    return world * M * N * steps / (ms_total / 1e3) / 1e9


# ----------------------------------------------------------------- GPU arm

def _event_ms(fn, stream, reps):
    import torch

    fn()
    torch.cuda.synchronize()
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        fn()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) / reps


def mixed_record(ms, synth, dev, stream):
    """Plain and mixed forms of bandpass+whiten on the 32 x 1.8M recording
    (device-resident, CUDA events), with the mixed form's error against the
    FP64 oracle."""
    import numpy as np
    import torch

    from oracle import oracle64

    M, N = 32, 1_800_000
    Xh = synth.generate_numpy(M, N, K=20, seed=0, sites=(3, 6))
    X = torch.from_numpy(Xh).to(dev)
    out = torch.empty_like(X)
    t_plain = _event_ms(lambda: ms.bandpass_whiten(X, FS, FMIN, FMAX, FWID, num_threads=GEOM_T, out=out), stream, 5)
    t_mixed = _event_ms(lambda: ms.bandpass_whiten(X, FS, FMIN, FMAX, FWID, num_threads=GEOM_T, out=out,
                                                   precision="mixed"), stream, 5)
    pre_mixed = out.cpu().numpy()
    _, q64, _, _ = oracle64.whiten(oracle64.bandpass_filter(Xh, FS, FMIN, FMAX, FWID, num_threads=GEOM_T))
    return {"workload": "32ch x 1.8M timepoints (60 s @ 30 kHz) data",
            "plain_ms": t_plain, "mixed_ms": t_mixed, "plain_gchs": M * N / t_plain / 1e6,
            "mixed_gchs": M * N / t_mixed / 1e6, "mixed_over_plain": t_plain / t_mixed,
            "mixed_rel_l2_vs_fp64": oracle64.rel_l2(pre_mixed, q64),
            "mixed_max_abs_vs_fp64": float(np.max(np.abs(pre_mixed - q64))),
            "gate_rel_l2": 1e-4}


def c5_record(ms, synth, dev, stream):
    """4 shanks x 384 channels, 5 min at 30 kHz, int16 input (gain 0.195):
    bandpass on the int16 recording, then each shank whitened on its own
    (device-resident, CUDA events), plain and mixed forms.  Algorithmic
    bytes: 2 (int16 read) + 2 (int16 read again for the output pass, were the
    two fused) + 4 (float write) = 8 per ch-sample."""
    import numpy as np
    import torch

    M1, N, S = 384, 9_000_000, 4
    X16 = torch.empty((N, M1 * S), dtype=torch.int16, device=dev)
    for k in range(S):
        Xk = synth.generate_torch(M1, N, K=300, seed=500 + k, sites=(6, 12), device=dev)
        X16[:, k * M1:(k + 1) * M1] = torch.clamp(torch.round(Xk / 0.195), -32768, 32767).to(torch.int16)
        del Xk
    torch.cuda.empty_cache()
    shanks = [list(range(1 + M1 * k, 1 + M1 * (k + 1))) for k in range(S)]
    filt = torch.empty((N, M1 * S), dtype=torch.float32, device=dev)
    pre = torch.empty_like(filt)
    rec = {"workload": "4 shanks x 384ch x 9M timepoints (5 min @ 30 kHz), int16 input, per-shank whitening"}
    for prec in ("plain", "mixed"):
        def run():
            ms.bandpass_filter(X16, FS, FMIN, FMAX, FWID, num_threads=GEOM_T, out=filt)
            ms.whiten_blocks(filt, shanks, out=pre, precision=prec)
        t = _event_ms(run, stream, 2)
        rec[prec + "_ms"] = t
        rec[prec + "_gchs"] = M1 * S * N / t / 1e6
    rec["mixed_over_plain"] = rec["plain_ms"] / rec["mixed_ms"]
    rec["plain_gbs_at_8B_per_ch_sample"] = 8 * M1 * S * N / (rec["plain_ms"] / 1e3) / 1e9
    del X16, filt, pre
    torch.cuda.empty_cache()
    return rec


def c4_jobs(seed=1):
    """The batched uneven workload: 48 recordings, channel counts from
    {16, 32, 64, 128, 384}, durations uniform 30 s - 20 min, sample rates from
    {20, 30} kHz, freq_max = min(6000, 0.4 fs)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    jobs = []
    for _ in range(48):
        M = int(rng.choice([16, 32, 64, 128, 384]))
        fs = float(rng.choice([20000.0, 30000.0]))
        N = int(round(rng.uniform(30.0, 1200.0) * fs))
        jobs.append((M, N, fs, min(6000.0, 0.4 * fs)))
    return jobs


def c4_record(ms, synth, dev, stream, budget_bytes=40 << 30):
    """Times the 48-recording workload in groups whose inputs and outputs fit
    `budget_bytes` of device memory: per group, one batched call against the
    same recordings one call at a time (both device-resident, CUDA events).
    Recordings are generated on the device per group (not timed)."""
    import torch

    jobs = c4_jobs()
    groups, cur, used = [], [], 0
    for j in sorted(jobs, key=lambda j: j[0] * j[1]):
        b = 8 * j[0] * j[1]
        if cur and used + b > budget_bytes:
            groups.append(cur)
            cur, used = [], 0
        cur.append(j)
        used += b
    if cur:
        groups.append(cur)
    t_batch = t_batch_mixed = t_single = 0.0
    total = 0
    skipped = []
    for gi, grp in enumerate(groups):
        recs = []
        try:
            for k, (M, N, fs, fmax) in enumerate(grp):
                X = synth.generate_torch(M, N, fs=fs, K=max(4, M // 2), seed=100 + gi * 64 + k,
                                         sites=(6, 12) if M >= 64 else (3, 6), device=dev)
                recs.append({"X": X, "samplerate": fs, "freq_min": FMIN, "freq_max": fmax, "freq_wid": FWID,
                             "num_threads": GEOM_T})
            del X
            tb = _event_ms(lambda: ms.bandpass_whiten_batch(recs), stream, 1)
            tbm = _event_ms(lambda: ms.bandpass_whiten_batch(recs, precision="mixed"), stream, 1)
            torch.cuda.empty_cache()
            ms.release_cached_memory()
            outs = [torch.empty_like(r["X"]) for r in recs]

            def singles():
                for r, o in zip(recs, outs):
                    ms.bandpass_whiten(r["X"], r["samplerate"], r["freq_min"], r["freq_max"], r["freq_wid"],
                                       num_threads=GEOM_T, out=o)

            ts = _event_ms(singles, stream, 1)
            t_batch += tb
            t_batch_mixed += tbm
            t_single += ts
            total += sum(j[0] * j[1] for j in grp)
            del outs
        except Exception as e:  # a group that does not fit the device is reported, not timed
            skipped.append({"recordings": [list(j[:3]) for j in grp], "error": f"{type(e).__name__}: {e}"[:200]})
        del recs
        torch.cuda.empty_cache()
        ms.release_cached_memory()
    if total == 0:
        return {"error": "no group fit the device", "skipped": skipped}
    return {"workload": "48 recordings, M in {16,32,64,128,384}, 30 s - 20 min, 20/30 kHz, seed 1",
            "ch_samples": total, "groups": len(groups), "batch_ms": t_batch, "single_ms": t_single,
            "batch_gchs": total / t_batch / 1e6, "single_gchs": total / t_single / 1e6,
            "batch_over_single": t_single / t_batch, "batch_mixed_ms": t_batch_mixed,
            "batch_mixed_gchs": total / t_batch_mixed / 1e6,
            "batch_mixed_over_single_plain": t_single / t_batch_mixed,
            "skipped_groups": skipped}



def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", default="c2", choices=sorted(SIZES))
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-stages", action="store_true")
    ap.add_argument("--no-mixed", action="store_true")
    ap.add_argument("--c5", action="store_true",
                    help="also time the 4 x 384-channel int16 shank configuration (5 min, per-shank whitening)")
    ap.add_argument("--c4", action="store_true",
                    help="also time the batched uneven workload (48 recordings, 30 s - 20 min) in memory-bounded "
                         "groups: several minutes")
    args = ap.parse_args()

    if args.impl == "reference":
        run_reference_arm(args, args.size)
        return

    import numpy as np
    import torch

    import mountainsort_b200 as ms
    from mountainsort_b200 import _lib, synth

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    lib = _lib.load()
    M, N, K_units, desc = SIZES[args.size]
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)

    # ---- batched uneven workload (C4) and the 4-shank int16 run (C5) first,
    # while the device holds nothing else (their largest recordings need most
    # of its memory)
    c4 = c5 = None
    if (args.c4 or args.c5) and rank == 0:
        for flag, name, fn in ((args.c5, "c5", c5_record), (args.c4, "c4", c4_record)):
            if not flag:
                continue
            free0, total = torch.cuda.mem_get_info(dev)
            try:
                rec = fn(ms, synth, dev, stream)
            except Exception as e:  # reported in the line; the headline fields stand
                rec = {"error": f"{type(e).__name__}: {e}"}
            rec["device_free_gb_at_start"] = free0 / 1e9
            rec["device_total_gb"] = total / 1e9
            torch.cuda.empty_cache()
            ms.release_cached_memory()
            if name == "c4":
                c4 = rec
            else:
                c5 = rec

    t0 = time.time()
    X = synth.generate_torch(M, N, fs=FS, K=K_units, seed=1000 + rank, sites=(6, 12) if M >= 64 else (3, 6),
                             device=dev)
    torch.cuda.synchronize()
    log(f"[rank {rank}] generated {M}x{N} in {time.time() - t0:.1f} s")
    pre = torch.empty((N, M), dtype=torch.float32, device=dev)

    def step():
        ms.bandpass_whiten(X, FS, FMIN, FMAX, FWID, num_threads=GEOM_T, out=pre)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    l0 = lib.ms3gpu_launch_count()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        step()
    ev1.record(stream)
    torch.cuda.synchronize()
    launches = (lib.ms3gpu_launch_count() - l0) // max(1, args.steps)
    if dist:
        dist.barrier()
    clocks = sampler.stop()
    ms_total = max_over_ranks(dist, ev0.elapsed_time(ev1), dev)
    ms_step = ms_total / args.steps
    value = replica_throughput(world, M, N, args.steps, ms_total)

    # ---- stage breakdown (same data, device pointers, CUDA events on the launching stream)
    stages = {}
    if not args.no_stages:
        filt = torch.empty((N, M), dtype=torch.float32, device=dev)

        def timed(fn, reps=2):
            fn()
            torch.cuda.synchronize()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            for _ in range(reps):
                fn()
            b.record(stream)
            torch.cuda.synchronize()
            return a.elapsed_time(b) / reps

        stages["bandpass_filter"] = timed(lambda: ms.bandpass_filter(X, FS, FMIN, FMAX, FWID, num_threads=GEOM_T,
                                                                      out=filt))
        C = ms.whiten_covariance(filt)
        stages["whiten_covariance"] = timed(lambda: ms.whiten_covariance(filt))
        stages["whitening_matrix"] = timed(lambda: ms.whitening_matrix(C), reps=1)
        Wm = ms.whitening_matrix(C)
        stages["apply_whitening"] = timed(lambda: ms.apply_whitening_matrix(filt, Wm, out=pre))
        del filt

    # ---- the mixed-precision form of the same step on the same recording
    mixed_step = None
    if not args.no_mixed:
        t_mixed = _event_ms(lambda: ms.bandpass_whiten(X, FS, FMIN, FMAX, FWID, num_threads=GEOM_T, out=pre,
                                                       precision="mixed"), stream, max(1, min(args.steps, 3)))
        mixed_step = {"workload": desc, "plain_ms": ms_step, "mixed_ms": t_mixed,
                      "mixed_gchs": M * N / t_mixed / 1e6, "mixed_over_plain": ms_step / t_mixed,
                      "error": ("gated at <= 1e-4 rel-L2 vs the FP64 oracle at 384 channels by the test suite "
                                "(4 x 384-channel shanks); not recomputed at this size")}

    # ---- roofline of the dominant stage (HBM bound: algorithmic bytes per ch-sample)
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peaks = json.load(open(peaks_path))
        hbm_peak, peak_src = float(peaks["hbm_gbs"]), "measured"
    else:
        hbm_peak, peak_src = 6650.0, "fallback"
    algo_bytes = {"bandpass_filter": 8, "whiten_covariance": 4, "apply_whitening": 8}
    roofline = None
    if stages:
        dom = max((k for k in stages if k in algo_bytes), key=lambda k: stages[k])
        achieved = algo_bytes[dom] * M * N / (stages[dom] / 1e3) / 1e9
        traffic = None
        tpath = os.path.join(ROOT, "profiles", "ncu_traffic.json")
        if os.path.exists(tpath):
            tr = json.load(open(tpath)).get(dom)
            if tr:
                traffic = tr.get("dram_bytes_per_launch_full")
        roofline = {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                    "frac": achieved / hbm_peak, "traffic": traffic, "peak_source": peak_src,
                    "algorithmic_bytes_per_ch_sample": algo_bytes[dom], "stage_ms": stages}

    # ---- the whole step against the fused path's compulsory traffic (12 B per ch-sample)
    step_roofline = {"bytes_per_ch_sample": 12, "achieved": 12 * M * N / (ms_step / 1e3) / 1e9, "peak": hbm_peak,
                     "unit": "GB/s", "peak_source": peak_src}
    step_roofline["frac"] = step_roofline["achieved"] / hbm_peak

    # ---- mixed-precision form on the 32ch x 1.8M data, next to the plain form (FP64 oracle for its error)
    mixed = None
    if rank == 0 and not args.no_mixed:
        mixed = mixed_record(ms, synth, dev, stream)

    # ---- end to end through the C ABI with pinned host buffers
    e2e = None
    if not args.no_e2e:
        del pre
        torch.cuda.empty_cache()
        Xh = torch.empty((N, M), dtype=torch.float32, pin_memory=True)
        Xh.copy_(X)
        del X
        torch.cuda.empty_cache()
        Ph = torch.empty((N, M), dtype=torch.float32, pin_memory=True)
        raw_np = Xh.numpy()
        pre_np = Ph.numpy()
        ms.bandpass_whiten(raw_np, FS, FMIN, FMAX, FWID, num_threads=GEOM_T, out=pre_np)  # warm-up
        if dist:
            dist.barrier()
        t1 = time.perf_counter()
        for _ in range(args.e2e_steps):
            ms.bandpass_whiten(raw_np, FS, FMIN, FMAX, FWID, num_threads=GEOM_T, out=pre_np)
        el = max_over_ranks(dist, time.perf_counter() - t1, dev)
        e2e = {"value": world * M * N * args.e2e_steps / el / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": 4 * M * N, "d2h_bytes_per_step": 4 * M * N,
               "ms_per_step": el / args.e2e_steps * 1e3, "steps": args.e2e_steps,
               "timing": "host wall clock around synchronous C-ABI calls (pinned host buffers)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(M, N, cpu_threads())

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": desc, "M": M, "N": N, "geometry_threads": GEOM_T,
                       "freq": [FMIN, FMAX, FWID], "l2_flush": "inputs (27.6 GB) larger than L2" if N * M * 4 > 2**30
                       else "none", "parallelism": f"replicas x{world} (one recording per GPU)"},
            "gpu_launches": int(launches),
            "clocks": clocks,
            "roofline": roofline,
            "step_roofline": step_roofline,
            "mixed": mixed,
            "mixed_step": mixed_step,
            "batched_c4": c4,
            "shanks_c5": c5,
            "cpu_baseline": cpu,
            "e2e": e2e,
        }
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
