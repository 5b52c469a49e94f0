"""The whitening apply's three-TF32-product arithmetic
(mountainsort_b200/csrc/apply_tc.cu), restated in numpy on the CPU.

y_t = W^T x_t (p_whiten.cpp:174-183).  The kernel reads x truncated to TF32
(x_hi: the top 19 bits of the FP32 pattern), forms x_lo = rna_tf32(x - x_hi)
from the bit pattern ((bits + 0x1000) & 0xFFFFE000: nearest, ties away from
zero), splits w into w_hi = rna_tf32(w), w_lo = rna_tf32(w - w_hi), and sums
x_hi w_hi + x_hi w_lo + x_lo w_hi.  Every product of two TF32 values is exact
in FP32; the tensor core's sums over a K-block of 32 (which round toward
zero) are modelled here as round-to-nearest FP32 sums, drained into
round-to-nearest FP32 running sums as the plain form does.  The tests pin the bit formulas and show the representation error the
kernel's precision claim rests on (~2^-22 of each term, against ~2^-11 for a
single TF32 product); the GPU kernel itself is checked against the oracle in
tests/test_gpu_parity.py and tests/test_gpu_chain.py."""
import numpy as np

from oracle import oracle64 as o64


def bits(x):
    return np.asarray(x, np.float32).view(np.uint32)


def from_bits(b):
    return np.asarray(b, np.uint32).view(np.float32)


def trunc_tf32(x):
    return from_bits(bits(x) & np.uint32(0xFFFFE000))


def rna_tf32(x):
    """Round FP32 to TF32 (10 explicit mantissa bits), nearest, ties away
    from zero: the integer round-half-up of the magnitude bits at bit 13."""
    return from_bits((bits(x) + np.uint32(0x1000)) & np.uint32(0xFFFFE000))


def rna_tf32_reference(x):
    """The same rounding from the value (frexp), for checking the bit form."""
    x = np.asarray(x, np.float64)
    m, e = np.frexp(np.abs(x))                 # |x| = m 2^e, m in [0.5, 1)
    q = np.floor(m * 2.0**11 + 0.5)            # 11 significant bits, half away from zero
    return (np.sign(x) * np.ldexp(q, e - 11)).astype(np.float32)


def split_w(w):
    w = np.asarray(w, np.float64)
    hi = rna_tf32(w.astype(np.float32))
    lo = rna_tf32((w - hi.astype(np.float64)).astype(np.float32))
    return hi, lo


def apply_three_tf32(X, Wt):
    """OUT[t][m1] = sum_m2 X[t][m2] Wt[m1][m2] by the kernel's split, K-blocks
    of 32 summed in FP32 and drained into FP32 running sums."""
    xh = trunc_tf32(X)
    xl = rna_tf32(X - xh)
    wh, wl = split_w(Wt)
    K = X.shape[1]
    out = np.zeros((X.shape[0], Wt.shape[0]), np.float32)
    for k0 in range(0, K, 32):
        s = slice(k0, k0 + 32)
        blk = (xh[:, s] @ wh[:, s].T) + (xh[:, s] @ wl[:, s].T) + (xl[:, s] @ wh[:, s].T)
        out = (out + blk.astype(np.float32)).astype(np.float32)
    return out


def test_rna_bit_formula_matches_the_value_rounding():
    rng = np.random.default_rng(0)
    x = (rng.standard_normal(200000) * np.exp(rng.uniform(-20, 20, 200000))).astype(np.float32)
    # exact ties: 12 significant bits ending in 1 round away from zero
    x[:6] = np.array([1 + 2.0**-11, -(1 + 2.0**-11), 3 * 2.0**-12 + 1, 1.5 + 2.0**-11, 2.0**-11 + 2.0**-22, 0.0],
                     np.float32)
    assert np.array_equal(rna_tf32(x), rna_tf32_reference(x))
    assert rna_tf32(np.float32(1 + 2.0**-11)) == np.float32(1 + 2.0**-10)
    assert rna_tf32(np.float32(-(1 + 2.0**-11))) == np.float32(-(1 + 2.0**-10))


def test_x_split_is_exact_to_two_to_minus_21():
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(100000) * 30.0).astype(np.float32)
    xh = trunc_tf32(x)
    d = x.astype(np.float64) - xh.astype(np.float64)
    assert np.array_equal(d.astype(np.float32).astype(np.float64), d)  # x - x_hi is exact in FP32
    xl = rna_tf32(x - xh)
    err = np.abs(x.astype(np.float64) - xh - xl.astype(np.float64))
    assert np.all(err <= 2.0**-21 * np.abs(x.astype(np.float64)))
    # one TF32 value alone is ~2^-11 off
    assert np.abs(x.astype(np.float64) - xh).max() > 2.0**-13 * np.abs(x).max()


def test_w_split_is_exact_to_two_to_minus_21():
    rng = np.random.default_rng(2)
    w = rng.standard_normal(50000) * 0.01
    wh, wl = split_w(w)
    err = np.abs(w - wh.astype(np.float64) - wl.astype(np.float64))
    assert np.all(err <= 2.0**-21 * np.abs(w) + 2.0**-24 * np.abs(w))  # + the FP32 cast of w - w_hi


def test_three_products_meet_the_float_reference_level():
    # a whitening matrix from the oracle (power iteration, p_whiten.cpp:120-163)
    # at 64 channels.  The whitened values cancel heavily (float arithmetic as
    # the reference does it is ~2e-5 off in relative L2 here), so the errors are
    # measured against the magnitude of the summed terms, |x| . |w|.
    rng = np.random.default_rng(3)
    M, N = 64, 4000
    mix = rng.standard_normal((M, M)) * 0.3 + np.eye(M)
    X = (rng.standard_normal((N, M)) @ mix * 40.0).astype(np.float32)
    W = o64.whitening_matrix(o64.xxt(X))[0]
    Wt = np.ascontiguousarray(W.T)  # Wt[m1][m2] = W[m1 M + m2] read as the GEMM's K-major operand
    X64 = X.astype(np.float64)
    exact = X64 @ Wt.T
    norm = np.abs(X64) @ np.abs(Wt).T
    xh = trunc_tf32(X)
    xl = rna_tf32(X - xh)
    wh, wl = split_w(Wt)
    f64 = [a.astype(np.float64) for a in (xh, xl, wh, wl)]
    rep = f64[0] @ f64[2].T + f64[0] @ f64[3].T + f64[1] @ f64[2].T  # the three products, summed exactly
    three = apply_three_tf32(X, Wt)
    one = f64[0] @ rna_tf32(Wt.astype(np.float32)).astype(np.float64).T
    f32 = (X @ Wt.astype(np.float32).T).astype(np.float64)  # float products and sums

    def err(v):
        return (np.abs(v - exact) / norm).max()

    assert err(rep) <= 2.0**-22, err(rep)     # measured 1.2e-7
    assert err(three) <= 2.0**-21, err(three)  # measured 1.7e-7 (FP32 sums of K-blocks)
    assert err(one) >= 2.0**-14, err(one)      # measured 3.0e-4: one TF32 product
    assert o64.rel_l2(three, exact) <= 2.5 * o64.rel_l2(f32, exact)
