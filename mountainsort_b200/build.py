"""Builds libms3gpu.so (CUDA, sm_100a) and the ms3gpu.mp processor executable
in-tree, next to this file.

    python -m mountainsort_b200.build        # or build() from Python
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


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    deps = _deps()
    if force or not _newer(LIB, deps):
        cmd = [_nvcc(), *ARCH, "-lineinfo", "-O3", "-std=c++17", "-shared", "-Xcompiler", "-fPIC",
               "-Xcompiler", "-fvisibility=hidden", "-I", INCLUDE, "-I", CSRC,
               "-DMS3GPU_BUILDING", "-o", LIB + ".tmp"]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        cmd += [os.path.join(CSRC, s) for s in CU_SOURCES]
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed:\n" + r.stdout + r.stderr)
        if ptxas_info or verbose:
            print(r.stdout + r.stderr)
        os.replace(LIB + ".tmp", LIB)
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
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
