"""How the C ABI classifies a caller's buffer (mountainsort_b200/csrc/ptrkind.h),
checked on the CPU: host memory is staged, device memory of the current GPU
and managed memory are used in place, and device memory of another GPU is
rejected instead of being handed to a kernel that would fault on it.  The
type codes are cudaMemoryType's (0 unregistered, 1 host, 2 device, 3
managed)."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mountainsort_b200", "csrc")

DRIVER = r"""
#include <cstdio>
#include "ptrkind.h"
int main() {
    using namespace ms3gpu;
    const char* names[] = {"host", "here", "managed", "elsewhere"};
    for (int type = 0; type < 4; type++)
        for (int dev = 0; dev < 2; dev++)
            std::printf("%d %d %s\n", type, dev, names[(int)classify_pointer(type, dev, 0)]);
    return 0;
}
"""


def test_pointer_classification(tmp_path):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    src = tmp_path / "drv.cpp"
    src.write_text(DRIVER)
    exe = str(tmp_path / "drv")
    r = subprocess.run([gxx, "-std=c++17", "-I", CSRC, str(src), "-o", exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {(int(a), int(b)): c for a, b, c in (line.split() for line in out if line)}
    assert got == {
        (0, 0): "host", (0, 1): "host",            # unregistered host memory: staged
        (1, 0): "host", (1, 1): "host",            # pinned host memory: staged
        (2, 0): "here", (2, 1): "elsewhere",       # device memory: in place only on the current GPU
        (3, 0): "managed", (3, 1): "managed",      # managed memory: in place
    }
