"""The bandpass's four-step formulation (mountainsort_b200/csrc/bandpass.cu),
restated in FP64 numpy on the CPU and checked against a direct DFT filter,
the operation of p_bandpass_filter.cpp:64-110 (forward DFT, times
kernel[k] / L, inverse DFT).

The kernel splits L = L1 * L2 with the window index n = L2 n1 + n2 and the
frequency k = k1 + L1 k2:
    F1  for each n2: the L1-point DFT over n1             -> A[k1][n2]
    F2  for each k1: twiddle w_L^(n2 k1), the L2-point DFT over n2 -> k2,
        times kernel[k1 + L1 k2] / L, the inverse L2-point DFT, twiddle
        w_L^(-n2 k1)
    F3  for each n2: the inverse L1-point DFT over k1      -> n1
and carries two real channels as one complex signal x_a + i x_b, which is
exact because the band kernel is real and even (kernel[k] = kernel[L - k]):
the real and imaginary parts of the filtered signal are the two filtered
channels.  A window length with a prime factor above 64 is filtered as a
zero-padded circular convolution of a 5-smooth length P >= 2L - 1, which
equals the length-L circular filter because the taps are even.  These tests
check the index algebra, the pairing and the padding, not the GPU:
the GPU passes are checked against the oracle in tests/test_gpu_parity.py."""
import numpy as np
import pytest

from oracle import oracle64 as o64


def four_step_filter(z, kern, L1, L2):
    """Filter the complex signals z (L x S) with kern (length L) by the
    kernel's three passes."""
    L = L1 * L2
    S = z.shape[1]
    x = z.reshape(L1, L2, S)                           # x[n1][n2] = z[L2 n1 + n2]
    A = np.fft.fft(x, axis=0)                          # F1: over n1 -> k1
    k1 = np.arange(L1)[:, None, None]
    n2 = np.arange(L2)[None, :, None]
    tw = np.exp(-2j * np.pi * (k1 * n2) / L)           # w_L^(n2 k1)
    B = np.fft.fft(A * tw, axis=1)                     # F2: over n2 -> k2; B[k1][k2] = Z[k1 + L1 k2]
    k = (np.arange(L1)[:, None] + L1 * np.arange(L2)[None, :])
    B = B * (kern[k] / L)[:, :, None]
    C = np.fft.ifft(B, axis=1) * L2 * np.conj(tw)      # inverse over k2 -> n2, twiddle w_L^(-n2 k1)
    y = np.fft.ifft(C, axis=0) * L1                    # F3: inverse over k1 -> n1
    return y.reshape(L, S)


def direct_filter(x, kern):
    """Forward DFT, times kern / L, unnormalised inverse DFT."""
    L = x.shape[0]
    return np.fft.ifft(np.fft.fft(x, axis=0) * (kern / L)[:, None], axis=0) * L


def _even_kernel(L, rng):
    k = rng.random(L)
    k[1:] = (k[1:] + k[1:][::-1]) / 2  # kernel[k] = kernel[L - k]
    return k


@pytest.mark.parametrize("L1,L2", [(12, 10), (30, 16), (7, 11)])
def test_four_step_equals_direct_filter(L1, L2):
    rng = np.random.default_rng(L1 * L2)
    L = L1 * L2
    kern = _even_kernel(L, rng)
    z = rng.standard_normal((L, 3)) + 1j * rng.standard_normal((L, 3))
    assert o64.rel_l2(four_step_filter(z, kern, L1, L2), direct_filter(z, kern)) < 1e-13


def test_band_kernel_is_real_and_even(ref32):
    # define_kernel (p_bandpass_filter.cpp:421-447) at the window length of
    # 384 channels and 16 threads, L = 240000 = 480 x 500
    L = 240000
    kern = ref32.define_kernel(L, 30000.0, 300.0, 6000.0, 1000.0)
    assert kern[0] == 0.0  # the DC bin when freq_min != 0
    assert np.array_equal(kern[1:], kern[1:][::-1])


def test_four_step_at_the_reference_window_with_paired_channels(ref32):
    L1, L2 = 480, 500
    L = L1 * L2
    kern = ref32.define_kernel(L, 30000.0, 300.0, 6000.0, 1000.0)
    rng = np.random.default_rng(5)
    x = rng.standard_normal((L, 4)) * 50.0  # four real channels
    z = x[:, 0::2] + 1j * x[:, 1::2]        # pairs (0, 1) and (2, 3) as complex signals
    y = four_step_filter(z, kern, L1, L2)
    ref = direct_filter(x, kern).real
    assert o64.rel_l2(y.real, ref[:, 0::2]) < 1e-12
    assert o64.rel_l2(y.imag, ref[:, 1::2]) < 1e-12
    assert np.abs(direct_filter(x, kern).imag).max() < 1e-9 * np.abs(ref).max()


def test_pairing_needs_an_even_kernel():
    # with a kernel that is not even, the two channels of a pair mix
    rng = np.random.default_rng(9)
    L1, L2 = 12, 10
    L = L1 * L2
    kern = rng.random(L)
    x = rng.standard_normal((L, 2))
    y = four_step_filter((x[:, 0] + 1j * x[:, 1])[:, None], kern, L1, L2)[:, 0]
    ref = direct_filter(x, kern)
    assert o64.rel_l2(y.real, ref[:, 0].real) > 1e-3


def _smooth5_at_least(n):
    """The smallest 2^a 3^b 5^c >= n."""
    best = None
    p5 = 1
    while p5 < 2 * n:
        p35 = p5
        while p35 < 2 * n:
            p = p35
            while p < n:
                p *= 2
            best = p if best is None else min(best, p)
            p35 *= 3
        p5 *= 5
    return best


def padded_filter(x, kern):
    """A window whose length L has a large prime factor: the length-L
    circular filter as a length-P circular convolution, P >= 2L - 1 and
    5-smooth, with the taps h = IDFT(kernel) / L laid out as g[j] = g[P - j]
    = h[j] (the layout of bandpass.cu's padded plans).  g is real and even,
    so its P-point spectrum is real and even and pairs of channels still
    travel as one complex signal."""
    L = x.shape[0]
    P = _smooth5_at_least(2 * L - 1)
    h = np.fft.ifft(kern).real
    g = np.zeros(P)
    g[:L] = h
    g[P - L + 1:] = h[1:][::-1]
    G = np.fft.fft(g)
    assert np.abs(G.imag).max() <= 1e-12 * np.abs(G.real).max()
    xp = np.zeros((P,) + x.shape[1:], dtype=np.result_type(x, np.complex128))
    xp[:L] = x
    return np.fft.ifft(np.fft.fft(xp, axis=0) * G.real[:, None], axis=0)[:L]


def test_smooth5_lengths():
    assert [_smooth5_at_least(n) for n in (1, 7, 11, 97, 932065)] == [1, 8, 12, 100, 933120]


@pytest.mark.parametrize("L", [1009, 466033])
def test_padded_window_equals_the_circular_filter(ref32, L):
    # 466033 (prime) is the window of 6 channels at 16 threads
    kern = ref32.define_kernel(L, 30000.0, 300.0, 6000.0, 1000.0)
    rng = np.random.default_rng(L)
    x = rng.standard_normal((L, 2)) * 50.0
    z = x[:, 0] + 1j * x[:, 1]
    y = padded_filter(z[:, None], kern)[:, 0]
    ref = direct_filter(x, kern).real
    assert o64.rel_l2(y.real, ref[:, 0]) < 1e-12
    assert o64.rel_l2(y.imag, ref[:, 1]) < 1e-12
