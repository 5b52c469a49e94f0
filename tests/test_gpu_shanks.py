"""Per-shank whitening of a multi-shank int16 recording (the large combined
benchmark configuration at test size: 4 shanks x 32 channels, int16 input
with amplifier gain 0.195 folded into the integers, 30 kHz): bandpass on the
int16 input, then ms3gpu_whiten_blocks with one block per shank.

Gates: plain form vs ref32 whitening each shank's filtered channels on their
own, relative L2 <= 1e-5; mixed form vs the FP64 oracle (filter and per-shank
whitening in FP64), relative L2 <= 1e-4; the result equals whitening each
shank with compute_whitening_matrix(channels) + apply_whitening_matrix."""
import numpy as np
import pytest

from mountainsort_b200 import _lib, api, synth
from oracle import oracle64 as o64

pytestmark = pytest.mark.gpu

FS, FMIN, FMAX, FWID = 30000.0, 300.0, 6000.0, 1000.0


@pytest.fixture(scope="module")
def probe():
    X = synth.generate_numpy(128, 300000, K=60, seed=5, sites=(6, 12))
    X16 = np.clip(np.round(X / 0.195), -32768, 32767).astype(np.int16)
    shanks = [list(range(1 + 32 * k, 33 + 32 * k)) for k in range(4)]
    return X16, shanks


def test_per_shank_whitening_plain_and_mixed(gpu_lib, ref32, probe):
    X16, shanks = probe
    filt = api.bandpass_filter(X16, FS, FMIN, FMAX, FWID, num_threads=16)
    pre = api.whiten_blocks(filt, shanks)
    for sh in shanks:
        cols = [c - 1 for c in sh]
        pre_ref, _, _ = ref32.whiten(np.ascontiguousarray(filt[:, cols]))
        assert o64.rel_l2(pre[:, cols], pre_ref) <= 1e-5
        # the same as the two whitening-matrix processors on the shank
        W = api.compute_whitening_matrix([filt], channels=sh)
        np.testing.assert_array_equal(pre[:, cols], api.apply_whitening_matrix(np.ascontiguousarray(filt[:, cols]), W))
    mixed = api.whiten_blocks(filt, shanks, precision="mixed")
    f64 = o64.bandpass_filter(X16.astype(np.float32), FS, FMIN, FMAX, FWID, num_threads=16)
    q64 = np.empty_like(mixed, dtype=np.float64)
    for sh in shanks:
        cols = [c - 1 for c in sh]
        _, q, _, _ = o64.whiten(np.ascontiguousarray(f64[:, cols]))
        q64[:, cols] = q
    err = o64.rel_l2(mixed, q64)
    print(f"per-shank mixed form vs FP64 oracle: rel L2 {err:.3e}, max-abs {np.max(np.abs(mixed - q64)):.3e}")
    assert err <= 1e-4


def test_blocks_must_partition_the_channels(gpu_lib, probe):
    X16, shanks = probe
    X = X16[:1000].astype(np.float32)
    with pytest.raises(_lib.Ms3GpuError):
        api.whiten_blocks(X, shanks[:3])  # channel 97..128 missing
    with pytest.raises(_lib.Ms3GpuError):
        api.whiten_blocks(X, [shanks[0], shanks[0], shanks[2], shanks[3]])  # a channel twice
