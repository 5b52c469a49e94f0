"""The bounds-checked build (libms3gpu_checked.so, -DMS3GPU_BOUNDS_CHECK):
every index check in its kernels must pass on ordinary inputs, and its
outputs must be those of the ordinary library bit for bit (the checks guard
the accesses, they change no arithmetic).  Each library runs in its own
process (MS3GPU_LIBRARY selects it)."""
import os
import subprocess
import sys

import numpy as np
import pytest

from mountainsort_b200 import _lib

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
import numpy as np
import torch
sys.path.insert(0, sys.argv[1])
from mountainsort_b200 import api, synth
out = sys.argv[2]
res = {}
X = torch.from_numpy(synth.generate_numpy(384, 260_017, K=40, seed=3)).cuda()
filt, pre = api.bandpass_whiten(X, 30000.0, 300.0, 6000.0, num_threads=16, want_filt=True)
res["filt384"], res["pre384"] = filt.cpu().numpy(), pre.cpu().numpy()
res["mixed384"] = api.bandpass_whiten(X, 30000.0, 300.0, 6000.0, num_threads=16, precision="mixed").cpu().numpy()
del X, filt, pre
recs = [dict(X=synth.generate_numpy(M, N, K=4, seed=M), samplerate=fs, freq_min=300.0, freq_max=6000.0,
             num_threads=16) for M, N, fs in [(16, 200_000, 30000.0), (64, 150_000, 20000.0), (130, 140_000, 30000.0)]]
for k, o in enumerate(api.bandpass_whiten_batch(recs)):
    res[f"batch{k}"] = o
Y = synth.generate_numpy(256, 120_000, K=20, seed=9)
res["blocks"] = api.whiten_blocks(api.bandpass_filter(Y, 30000.0, 300.0, 6000.0, num_threads=16),
                                  [list(range(1, 129)), list(range(129, 257))])
res["int16"] = api.bandpass_filter(Y.astype(np.int16), 30000.0, 300.0, 6000.0, quantization_unit=0.5,
                                   num_threads=16)
np.savez(out, **res)
"""


def _run(tmp_path, which):
    out = str(tmp_path / f"{which}.npz")
    env = dict(os.environ)
    env.pop("MS3GPU_LIBRARY", None)
    if which == "checked":
        env["MS3GPU_LIBRARY"] = "checked"
    r = subprocess.run([sys.executable, "-c", SCRIPT, ROOT, out], env=env, capture_output=True, text=True,
                       timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    return np.load(out)


def test_checked_build_passes_and_matches(tmp_path):
    if not os.path.exists(_lib.CHECKED_LIB_PATH):
        pytest.skip("libms3gpu_checked.so not built")
    plain = _run(tmp_path, "plain")
    checked = _run(tmp_path, "checked")
    assert set(plain.files) == set(checked.files)
    for k in plain.files:
        np.testing.assert_array_equal(checked[k], plain[k], err_msg=k)
