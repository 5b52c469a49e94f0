"""Builds libms3gpu.so (CUDA, sm_100a) and the ms3gpu.mp processor executable
in-tree, next to this file.

    python -m mountainsort_b200.build        # or build() from Python
    python -m mountainsort_b200.build --no-checked   # without libms3gpu_checked.so
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
LIB = os.path.join(HERE, "libms3gpu.so")
LIB_CHECKED = os.path.join(HERE, "libms3gpu_checked.so")  # -DMS3GPU_BOUNDS_CHECK
EXE = os.path.join(HERE, "ms3gpu.mp")

CU_SOURCES = ["capi.cu", "bandpass.cu", "whiten.cu", "apply_tc.cu", "pipeline.cu", "stream.cu", "artifacts.cu", "detect.cu", "cov_i8.cu"]
EXE_SOURCES = ["ms3gpu_main.cpp", "mdaio.cpp"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _cxx() -> str:
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else (os.environ.get("CXX") or "g++")


def _newer(target: str, deps) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(d) <= t for d in deps)


def _deps():
    out = [os.path.join(INCLUDE, "ms3gpu.h"), __file__]
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".h", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _lib_cmd(out: str, checked: bool, ptxas_info: bool):
    cmd = [_nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
           "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC, "-DMS3GPU_BUILDING", "-o", out + ".tmp"]
    if checked:
        cmd += ["-DMS3GPU_BOUNDS_CHECK"]
    if ptxas_info:
        cmd += ["-Xptxas", "-v"]
    return cmd + [os.path.join(CSRC, s) for s in CU_SOURCES]


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False, checked: bool = True) -> str:
    """Builds libms3gpu.so and, with `checked`, the bounds-checked
    libms3gpu_checked.so (the two compile at the same time)."""
    deps = _deps()
    jobs = []
    if force or not _newer(LIB, deps):
        jobs.append((LIB, _lib_cmd(LIB, False, ptxas_info)))
    if checked and (force or not _newer(LIB_CHECKED, deps)):
        jobs.append((LIB_CHECKED, _lib_cmd(LIB_CHECKED, True, False)))
    procs = []
    for out, cmd in jobs:
        if verbose:
            print(" ".join(cmd), flush=True)
        procs.append((out, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
    for out, pr in procs:
        text, _ = pr.communicate()
        if pr.returncode != 0:
            raise RuntimeError("nvcc failed for " + os.path.basename(out) + ":\n" + text)
        if ptxas_info or verbose:
            print(text)
        os.replace(out + ".tmp", out)
    if force or not _newer(EXE, deps + [LIB]):
        cmd = [_cxx(), "-O2", "-std=c++17", "-pthread", "-I", INCLUDE, "-I", CSRC, "-o", EXE + ".tmp",
               *[os.path.join(CSRC, s) for s in EXE_SOURCES], "-L", HERE, "-l:libms3gpu.so",
               "-Wl,-rpath,$ORIGIN"]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("g++ failed:\n" + r.stdout + r.stderr)
        os.replace(EXE + ".tmp", EXE)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv,
          checked="--no-checked" not in sys.argv)
