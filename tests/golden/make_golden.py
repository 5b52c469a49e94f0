"""Regenerates the committed fixtures in tests/golden/.

Run in a checkout where the reference project is available:

    python tests/golden/make_golden.py <root of the reference checkout>

1. .mda files written by the reference's own Python writer
   (packages/pyms/mlpy/mdaio.py: writemda8/16i/16ui/32/32i/32ui/64 and
   DiskWriteMda) for the array of its mdaio_test (M=4, N=12,
   X[m, n] = 10 n + m, mdaio.py:312-318), plus one file whose header uses
   64-bit dims, produced by the same writer with its 64-bit-dims branch.
   These pin the .mda format of the boundary.
2. Oracle vectors (computed by oracle/, the CPU restatement): band kernel
   samples, a whitening matrix and its components, a small bandpass+whiten
   case.  These are regression fixtures for the oracle itself -- the
   reference publishes no numeric golden vectors for this path.
"""
from __future__ import annotations

import importlib.util
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def _load_ref_mdaio(ref_root):
    path = os.path.join(ref_root, "packages", "pyms", "mlpy", "mdaio.py")
    spec = importlib.util.spec_from_file_location("ref_mdaio", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def make_mda_fixtures(ref_root):
    ref = _load_ref_mdaio(ref_root)
    M, N = 4, 12
    X = np.ndarray((M, N))
    for n in range(N):
        for m in range(M):
            X[m, n] = n * 10 + m
    writers = {"uint8": ref.writemda8, "int16": ref.writemda16i, "uint16": ref.writemda16ui,
               "float32": ref.writemda32, "int32": ref.writemda32i, "uint32": ref.writemda32ui,
               "float64": ref.writemda64}
    for name, fn in writers.items():
        fn(X, os.path.join(HERE, f"mda_{name}.mda"))
    # DiskWriteMda + writeChunk (the chunked writer), float32
    p = os.path.join(HERE, "mda_chunked_float32.mda")
    if os.path.exists(p):
        os.remove(p)
    W = ref.DiskWriteMda(p, (M, N), dt="float32")
    W.writeChunk(X[:, :5].astype(np.float32), i1=0, i2=0)
    W.writeChunk(X[:, 5:].astype(np.float32), i1=0, i2=5)
    # the writer's 64-bit-dims header branch (taken for dims > 2e9) on a small array
    p = os.path.join(HERE, "mda_dims64_float32.mda")
    H = ref.MdaHeader("float32", [M, N])
    H.uses64bitdims = True
    H.header_size = 3 * 4 + H.num_dims * 8
    ref._write_header(p, H)
    with open(p, "ab") as f:
        np.reshape(X, X.size, order="F").astype("float32").tofile(f)
    # and read back through the reference reader to record what it sees
    seen = {name: ref.readmda(os.path.join(HERE, f"mda_{name}.mda")).tolist() for name in writers}
    with open(os.path.join(HERE, "mda_expected.json"), "w") as f:
        json.dump({"M": M, "N": N, "values": X.tolist(), "reference_readmda": seen}, f)


def make_oracle_fixtures():
    sys.path.insert(0, ROOT)
    from oracle import ref32, oracle64
    from mountainsort_b200 import synth

    out = {}
    # band kernel at the canonical window (L = 240000, fs 30 kHz, 300-6000 Hz, wid 1000)
    K = ref32.define_kernel(240000, 30000.0, 300.0, 6000.0, 1000.0)
    idx = [0, 1, 2, 80, 800, 2400, 2401, 48000, 48001, 56000, 119999, 120000, 120001, 239999]
    out["kernel_240000"] = {"index": idx, "value": [float(K[i]) for i in idx]}
    # chunk geometry samples (M, T) -> chunk
    out["chunk_size"] = [[M, T, int(ref32.chunk_size(M, T))] for (M, T) in
                         [(1, 1), (4, 16), (8, 16), (16, 8), (16, 16), (32, 16), (384, 1), (384, 64)]]
    # whitening matrix of a seeded 6x6 covariance
    rng = np.random.default_rng(7)
    B = rng.standard_normal((6, 200))
    C = (B @ B.T) / 199
    W, comps, sig = ref32.whitening_matrix(C)
    out["whitening_6"] = {"XXt": C.tolist(), "W": W.tolist(), "components": comps.tolist(), "sigma": sig.tolist()}
    np.savez_compressed(os.path.join(HERE, "oracle_vectors.npz"),
                        kernel_index=np.array(idx), kernel_value=K[idx])
    # small end-to-end case: M=4 channels, N=3000, T=16 (chunk 579050, L=699050)
    X = synth.generate_numpy(4, 3000, K=2, seed=3, sites=(1, 3))
    filt = ref32.bandpass_filter(X, 30000, 300, 6000, 1000, num_threads=16)
    pre, xxt, Wp = ref32.whiten(filt)
    np.savez_compressed(os.path.join(HERE, "small_case.npz"), raw=X, filt=filt, pre=pre, xxt=xxt, W=Wp)
    with open(os.path.join(HERE, "oracle_vectors.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: make_golden.py <root of the reference checkout>")
    ref_root = sys.argv[1]
    make_mda_fixtures(ref_root)
    make_oracle_fixtures()
    print("fixtures written to", HERE)
