"""Regenerates tests/golden/ref_golden.npz from the reference's own code.

Run where the reference checkout is present, after `make -C oracle ref`
(which compiles packages/ms3/p_bandpass_filter.cpp, p_whiten.cpp, pca.cpp,
p_mask_out_artifacts.cpp and the mda/ classes into oracle/_ref/libmsref.so):

    make -C oracle ref REF_ROOT=<root of the reference checkout>
    python tests/golden/make_ref_golden.py

The fixture pins the oracle (ref32) to the reference without the reference
being present: inputs are stored exactly (int16 recordings, which the
reference converts to float on read, and a float64 matrix), outputs as the
SHA-256 of their bytes plus a few values, because ref32 must reproduce them
bit for bit.  Cases:
  bp16     ms3.bandpass_filter, 4 channels x 20000 (int16 input), T = 16
           geometry (chunk 579050, window L = 699050), float32 output
  bp16_q   the same with quantization_unit 0.5 (int16 output)
  bp16_sub the same with subsample_factor 3 and T = 19
  wh       ms3.whiten of bp16's output (1e-4 rounding), and with
           quantization_unit 0.01 (int16 output)
  W16      whitening_matrix_from_XXt of a 16 x 16 covariance (stored whole)
  mask     ms3.mask_out_artifacts of bp16's output (threshold 3, interval 500)
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

FS, FMIN, FMAX, FWID = 30000.0, 300.0, 6000.0, 1000.0


def digest(a: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def inputs():
    rng = np.random.default_rng(20250)
    N, M = 20000, 4
    t = np.arange(N) / FS
    X = 40 * rng.standard_normal((N, M)) + 300 * np.sin(2 * np.pi * 7 * t)[:, None]
    X[5000:5045, 1] -= 900 * np.hanning(45)
    X16 = np.clip(np.round(X), -32768, 32767).astype(np.int16)
    A = rng.standard_normal((16, 64))
    C = A @ A.T / 64 + np.diag(np.linspace(0.5, 3.0, 16))
    return X16, C


def main():
    from oracle import refpin

    if not refpin.available():
        sys.exit("oracle/_ref/libmsref.so is missing: run `make -C oracle ref` first")
    X16, C = inputs()
    Xf = X16.astype(np.float32)
    out = {"X16": X16, "C16": C}
    bp = refpin.bandpass_filter(Xf, FS, FMIN, FMAX, FWID, num_threads=16)
    bq = refpin.bandpass_filter(Xf, FS, FMIN, FMAX, FWID, quantization_unit=0.5, num_threads=16)
    bs = refpin.bandpass_filter(Xf, FS, FMIN, FMAX, FWID, subsample_factor=3, num_threads=19)
    wh = refpin.whiten(bp)
    wq = refpin.whiten(bp, quantization_unit=0.01)
    W = refpin.whitening_matrix(C)
    mk = refpin.mask_out_artifacts(bp, threshold=3.0, interval_size=500)
    for name, a in (("bp16", bp), ("bp16_q", bq), ("bp16_sub", bs), ("wh", wh), ("wh_q", wq), ("mask", mk)):
        out[name + "_sha256"] = np.array(digest(a))
        out[name + "_shape"] = np.array(a.shape)
        out[name + "_dtype"] = np.array(str(a.dtype))
        out[name + "_head"] = np.ascontiguousarray(a.ravel()[:64])
    out["W16"] = W
    np.savez_compressed(os.path.join(HERE, "ref_golden.npz"), **out)
    print("wrote", os.path.join(HERE, "ref_golden.npz"))


if __name__ == "__main__":
    main()
