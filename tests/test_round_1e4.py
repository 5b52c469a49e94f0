"""The whitened output's rounding to multiples of 1e-4 (p_whiten.cpp:31-41,
185-189: x = (float)(floor(x / 0.0001 + 0.5) * 0.0001) in double), as the
GPU epilogues compute it (quantize_1e4 in mountainsort_b200/csrc/whiten.cu,
quantize_1e4_x32 in apply_tc.cu): x * 10000 instead of the division, and
the division only where x * 10000 + 0.5 lies within 1e-6 of an integer.
Restated here with numpy's IEEE double operations (the same round-to-nearest
multiply, add and divide as __dmul_rn, __dadd_rn and __ddiv_rn) and checked
to give the reference's bits on random values and on every float near a
rounding boundary of several ranges.

For a float32 x the multiply alone already gives the reference's bits: x *
10000 is exact in double (a 24-bit significand times 625 * 2^4 needs at most
34 bits), and the double nearest 0.0001 is 1e-4 (1 + 4.8e-17), so the exact
quotient x / 0.0001 lies within 0.43 ulp of that representable product and
rounds to it.  (Checked once for all 2^32 bit patterns: x * 10000 + 0.5 ==
x / 0.0001 + 0.5 for every finite float32.)  The kernels' division branch is
therefore a guard that never changes a result for float32 input."""
from fractions import Fraction

import numpy as np


def reference_round(x):
    xd = np.asarray(x, np.float32).astype(np.float64)
    return (np.floor(xd / 0.0001 + 0.5) * 0.0001).astype(np.float32)


def gpu_round(x, redo=True):
    xd = np.asarray(x, np.float32).astype(np.float64)
    t = xd * 10000.0 + 0.5
    f = np.floor(t)
    if redo:
        with np.errstate(invalid="ignore"):
            near = (t - f < 1e-6) | (f + 1.0 - t < 1e-6)
        f = np.where(near, np.floor(xd / 0.0001 + 0.5), f)
    return (f * 0.0001).astype(np.float32)


def same_bits(a, b):
    return np.array_equal(np.asarray(a).view(np.uint32), np.asarray(b).view(np.uint32))


def near_boundaries(k, ulps=6):
    """The float32 values within `ulps` units of each rounding boundary
    (k - 0.5) * 1e-4, both signs."""
    b = ((k.astype(np.float64) - 0.5) * 1e-4).astype(np.float32)
    steps = np.arange(-ulps, ulps + 1, dtype=np.int64)
    v = (b.view(np.int32)[:, None].astype(np.int64) + steps[None, :]).astype(np.int32).view(np.float32).ravel()
    v = v[np.isfinite(v)]
    return np.concatenate([v, -v])


def test_random_values_round_like_the_reference():
    rng = np.random.default_rng(0)
    for _ in range(4):
        x = (np.exp(rng.uniform(np.log(1e-7), np.log(1e5), 4_000_000)) * rng.choice([-1.0, 1.0], 4_000_000))
        x = x.astype(np.float32)
        assert same_bits(gpu_round(x), reference_round(x))


def test_values_at_rounding_boundaries_round_like_the_reference():
    rng = np.random.default_rng(1)
    ks = [np.arange(0, 200_000),                                # |x| < 20
          rng.integers(200_000, 100_000_000, 400_000),         # up to 1e4
          rng.integers(10**8, 10**11, 100_000)]                # up to 1e7 (float spacing above 1e-4 near 1e4)
    for k in ks:
        x = near_boundaries(k)
        ref = reference_round(x)
        assert same_bits(gpu_round(x), ref)
        assert same_bits(gpu_round(x, redo=False), ref)  # the multiply alone, too


def test_the_multiply_is_the_division_for_float_inputs():
    # the argument of the module docstring, on values where x * 10000 + 0.5 is
    # (or is next to) a half-integer: x = m / 32, m odd, gives x * 10000 = 312.5 m
    m = np.arange(1, 2_000_001, 2, dtype=np.float64)
    x = (m / 32).astype(np.float32)
    assert np.array_equal(x.astype(np.float64), m / 32)
    xd = x.astype(np.float64)
    assert np.array_equal(xd * 10000.0, xd / 0.0001)
    # the margin: the double 0.0001 is 1e-4 (1 + delta); a quotient is off
    # the exact product by m delta ulp-units of 2^-52, m < 2 the significand
    delta = float(Fraction(0.0001) * 10000 - 1)
    assert 0 < delta and 2 * delta * 2.0**52 < 0.5


def test_special_values():
    x = np.array([0.0, -0.0, 1e-45, -1e-45, 5e-5, -5e-5, 4.9999e-5, 1e12, -3e38, np.inf, -np.inf, np.nan],
                 np.float32)
    g, r = gpu_round(x), reference_round(x)
    assert np.array_equal(g, r, equal_nan=True)
    assert np.array_equal(np.signbit(g), np.signbit(r))
