"""Input forms of the bandpass and whiten processors on the GPU: int16
recordings (converted to float inside the filter's loads, as the reference's
reader converts them, mda/mdaio.cpp:205-230) and directory inputs (the
directory's .mda files concatenated in time, mda/diskreadmda32.cpp:283-288).

Gates: the int16 path equals the float path on the converted recording
bit-for-bit (the conversion is exact and the arithmetic after it is the
same); outputs vs ref32 relative L2 <= 1e-5 (plain FP32 form)."""
import os
import subprocess

import numpy as np
import pytest

from mountainsort_b200 import api, mdaio, synth
from oracle import oracle64 as o64

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "mountainsort_b200", "ms3gpu.mp")
FS, FMIN, FMAX, FWID = 30000.0, 300.0, 6000.0, 1000.0


def _int16_recording(M, N, seed):
    X = synth.generate_numpy(M, N, K=max(1, M // 2), seed=seed)
    return np.clip(np.round(X / 0.195), -32768, 32767).astype(np.int16)  # gain 0.195 like an amplifier


@pytest.mark.parametrize("M,N", [(32, 360000), (7, 250000), (64, 130001)])
def test_int16_input_equals_float_path(gpu_lib, ref32, M, N):
    X16 = _int16_recording(M, N, seed=M)
    Xf = X16.astype(np.float32)
    T = max(16, 187 // M + 1)  # M * T >= 187: the L = 240000 window
    a = api.bandpass_filter(X16, FS, FMIN, FMAX, FWID, num_threads=T)
    b = api.bandpass_filter(Xf, FS, FMIN, FMAX, FWID, num_threads=T)
    np.testing.assert_array_equal(a, b)
    ref = ref32.bandpass_filter(Xf, FS, FMIN, FMAX, FWID, num_threads=T)
    assert o64.rel_l2(a, ref) <= 1e-5


def test_int16_input_from_device_and_quantized_output(gpu_lib, ref32):
    import torch

    X16 = _int16_recording(16, 300000, seed=3)
    a = api.bandpass_filter(torch.from_numpy(X16).cuda(), FS, FMIN, FMAX, FWID, quantization_unit=0.5,
                            num_threads=16)
    b = api.bandpass_filter(X16.astype(np.float32), FS, FMIN, FMAX, FWID, quantization_unit=0.5, num_threads=16)
    assert a.dtype == torch.int16
    np.testing.assert_array_equal(a.cpu().numpy(), b)
    # freq_max = 0 copies the int16 input unchanged
    c = api.bandpass_filter(X16, FS, FMIN, 0.0)
    assert c.dtype == np.int16
    np.testing.assert_array_equal(c, X16)


def _run(*args):
    return subprocess.run([EXE, *args], capture_output=True, text=True, timeout=600)


def test_executable_int16_file_and_directory_inputs(gpu_lib, ref32, tmp_path):
    X16 = _int16_recording(32, 400000, seed=7)
    p16 = str(tmp_path / "raw16.mda")
    mdaio.writemda(X16.T, p16)
    o16, of = str(tmp_path / "f16.mda"), str(tmp_path / "ff.mda")
    pf = str(tmp_path / "rawf.mda")
    mdaio.writemda(X16.astype(np.float32).T, pf)
    args = ["--samplerate=30000", "--freq_min=300", "--freq_max=6000", "--_request_num_threads=16"]
    r = _run("ms3.bandpass_filter", f"--timeseries={p16}", f"--timeseries_out={o16}", *args)
    assert r.returncode == 0, r.stderr
    r = _run("ms3.bandpass_filter", f"--timeseries={pf}", f"--timeseries_out={of}", *args)
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(mdaio.readmda(o16), mdaio.readmda(of))

    # a directory of three files is the concatenation of the files, in name order
    d = tmp_path / "parts"
    d.mkdir()
    Xf = X16.astype(np.float32)
    cuts = [0, 150000, 170000, 400000]
    for k, name in enumerate(["p0.mda", "p1.mda", "p2.mda"]):
        mdaio.writemda(Xf[cuts[k]:cuts[k + 1]].T, str(d / name))
    od = str(tmp_path / "fdir.mda")
    r = _run("ms3.bandpass_filter", f"--timeseries={d}", f"--timeseries_out={od}", *args)
    assert r.returncode == 0, r.stderr
    np.testing.assert_array_equal(mdaio.readmda(od), mdaio.readmda(of))
    ow = str(tmp_path / "wdir.mda")
    r = _run("ms3.whiten", f"--timeseries={d}", f"--timeseries_out={ow}")
    assert r.returncode == 0, r.stderr
    pre_ref, _, _ = ref32.whiten(Xf)
    assert o64.rel_l2(mdaio.readmda(ow).T, pre_ref) <= 1e-5
