"""The integer-digit covariance scheme of mountainsort_b200/csrc/cov_i8.cu,
restated in numpy on the CPU and held to the same gate as the GPU kernel
(relative L2 <= 1e-8 against the FP64 covariance of whiten pass 1,
p_whiten.cpp:64-118), and the diagonal to 2e-9 (the dropped d2^2 term alone
would bias it by ~1.3e-8).

The restatement follows the kernel's arithmetic step by step: the per-run
channel exponent from the max-magnitude bits (run_exponent), the digits from
two float roundings (digits4: rint(x 2^(22-e)), then the remainder held at
127), the four weight classes of digit products (exact: every class sum is
an integer far below 2^53, so FP64 matrix products give it exactly), the
seven-product form of a diagonal block pair (classes 1 and 3 one half at a
time, the transposed half added when the tile is reduced), the d2^2 term
kept on the diagonal, the FP64 combination and power-of-two scaling of the
drain, and the run-ordered reduction divided by N - 1.  It checks the
algorithm, not the GPU: the GPU kernel itself is checked against the oracle
in tests/test_gpu_covariance_tc.py."""
import numpy as np
import pytest

from oracle import oracle64 as o64

KB = 128  # channels per block (one 128 x 128 accumulator tile)
SENTINEL = 1000


def run_exponent(col):
    """Smallest e with 2^e > max |x| (at least -96); 0 for an all-zero run;
    SENTINEL when the run holds inf / NaN."""
    m = int((col.view(np.uint32) & np.uint32(0x7FFFFFFF)).max()) if col.size else 0
    if m >= 0x7F800000:
        return SENTINEL
    if m == 0:
        return 0
    return max((m >> 23) - 126, -96)


def digits(x, e):
    """Four signed digits of v = rint-ish(x 2^(30-e)) for one channel's run:
    v = d0 2^24 + d1 2^16 + d2 2^8 + d3, |d0| <= 64, d1..d3 in [-128, 127]."""
    x = x.astype(np.float64)
    vh = np.rint(x * 2.0 ** (22 - e))  # one rounding of x 2^(22-e) to an integer, ties to even
    rem = np.minimum(x * 2.0 ** (30 - e) - 256.0 * vh, 127.0)  # exact; +128 after a tie is held at 127
    d3 = np.rint(rem).astype(np.int64)
    h = vh.astype(np.int64) + 0x8080  # balanced bytes: bias by 0x80 in bytes 0 and 1
    d2 = (h & 0xFF) - 128
    d1 = ((h >> 8) & 0xFF) - 128
    d0 = h >> 16
    return [d0, d1, d2, d3], (256 * vh.astype(np.int64) + d3)


def run_tile(D, bi, bj, cols_i, cols_j, e, seven):
    """One run's FP64 partial tile of block pair (bi, bj), as the drain
    writes it.  D[k] holds digit plane k, shape (R, Mp)."""
    def g(k, cols):
        return D[k][:, cols].astype(np.float64)

    def prod(k, l):  # sum over the run of d_k(i) d_l(j)
        return g(k, cols_i).T @ g(l, cols_j)

    diag = bi == bj
    A0 = prod(0, 0)
    A2 = prod(0, 2) + prod(2, 0) + prod(1, 1)
    if diag and seven:
        A1 = prod(0, 1)
        A3 = prod(0, 3) + prod(1, 2)
    else:
        A1 = prod(0, 1) + prod(1, 0)
        A3 = prod(0, 3) + prod(3, 0) + prod(1, 2) + prod(2, 1)
    for A in (A0, A1, A2, A3):
        assert np.abs(A).max() < 2**31  # the int32 accumulators cannot overflow
    r, c = np.meshgrid(np.arange(len(cols_i)), np.arange(len(cols_j)), indexing="ij")
    if diag:
        dcorr = (g(2, cols_i) ** 2).sum(axis=0)  # per-channel sums of d2^2
    if not diag:
        acc = (A0 * 16777216.0 + A1 * 65536.0) + (A2 * 256.0 + A3)
    elif seven:
        half = A1 * 65536.0 + A3
        sym = A0 * 16777216.0 + A2 * 256.0
        sym = np.where(r == c, sym + dcorr[r] * 0.00390625, sym)
        acc = np.where(c > r, sym + half, np.where(c == r, sym + 2.0 * half, half))
    else:
        acc = (A0 * 16777216.0 + A1 * 65536.0) + (A2 * 256.0 + A3)
        acc = np.where(r == c, acc + dcorr[r] * 0.00390625, acc)
    ei, ej = e[cols_i][:, None], e[cols_j][None, :]
    bad = (ei == SENTINEL) | (ej == SENTINEL)
    scale = np.ldexp(1.0, np.where(bad, 0, ei + ej - 36))
    return np.where(bad, np.nan, acc * scale)


def digit_covariance(X, R, seven=True):
    """XXt / (N - 1) of X (N timepoints x M channels, float32) by the digit
    scheme, runs of R timepoints, 128-channel block pairs bi <= bj."""
    N, M = X.shape
    nb = -(-M // KB)
    blocks = [np.arange(b * KB, min(M, (b + 1) * KB)) for b in range(nb)]
    pairs = [(bi, bj) for bi in range(nb) for bj in range(bi, nb)]
    parts = {p: [] for p in pairs}
    for t0 in range(0, N, R):
        Xr = X[t0:t0 + R]
        e = np.array([run_exponent(Xr[:, m]) for m in range(M)])
        D = [np.zeros(Xr.shape, np.int64) for _ in range(4)]
        for m in range(M):
            if e[m] == SENTINEL:
                # the kernel's digits of such a channel are arbitrary bytes; the
                # drain writes NaN wherever the channel appears, so they stay 0 here
                continue
            dm, _ = digits(Xr[:, m], e[m])
            for k in range(4):
                D[k][:, m] = dm[k]
        for (bi, bj) in pairs:
            parts[(bi, bj)].append(run_tile(D, bi, bj, blocks[bi], blocks[bj], e, seven))
    C = np.empty((M, M))
    for (bi, bj) in pairs:
        s = np.zeros((len(blocks[bi]), len(blocks[bj])))
        for t in parts[(bi, bj)]:  # the runs in order
            if bi != bj:
                s = s + t
            elif seven:  # tile(r, c) + tile(c, r) above the diagonal, tile(r, r) on it
                s = s + (np.triu(t, 1) + np.triu(t.T, 1) + np.diag(np.diag(t)))
            else:
                s = s + np.triu(t)
        if bi == bj:  # the lower half mirrors the upper half
            s = np.triu(s) + np.triu(s, 1).T
        if N > 1:
            s = s / (N - 1)
        C[np.ix_(blocks[bi], blocks[bj])] = s
        C[np.ix_(blocks[bj], blocks[bi])] = s.T
    return C


def _signals(M, N, seed):
    rng = np.random.default_rng(seed)
    X = rng.standard_normal((N, M)).astype(np.float32) * np.float32(20.0)
    X[:, :: max(1, M // 7)] *= np.float32(40.0)  # a few channels at a larger scale
    return X


def test_digits_reconstruct_the_fixed_point_value():
    rng = np.random.default_rng(1)
    x = (rng.standard_normal(20000) * 3.0).astype(np.float32)
    e0 = run_exponent(x)
    # values whose x 2^(22-e) falls on a half: where rounding to even goes down
    # the remainder is +128, which a byte cannot hold, and is held at 127
    n = np.arange(8)
    x[:8] = ((2 * n + 1) * 2.0 ** (e0 - 23)).astype(np.float32)
    assert run_exponent(x) == e0
    for e in (e0, e0 + 3, 40):
        d, v = digits(x, e)
        assert np.abs(d[0]).max() <= 64
        for k in (1, 2, 3):
            assert d[k].min() >= -128 and d[k].max() <= 127
        assert np.array_equal(v, d[0] * 2**24 + d[1] * 2**16 + d[2] * 2**8 + d[3])
        xs = x.astype(np.float64) * 2.0 ** (30 - e)
        assert np.abs(v - xs).max() <= 1.0
        if e == e0:
            assert np.array_equal(xs[:8] - v[:8], np.where(n % 2 == 0, 1.0, 0.0))


@pytest.mark.parametrize("M,N,R", [(130, 40000, 8192), (128, 20001, 8192), (8, 5000, 1024)])
def test_digit_covariance_vs_fp64(M, N, R):
    X = _signals(M, N, seed=M + N)
    C = digit_covariance(X, R)
    ref = o64.xxt(X)
    e = o64.rel_l2(C, ref)
    assert e <= 1e-8, e
    assert np.array_equal(C, C.T)
    # the diagonal: 1.6e-10 .. 6.4e-10 here; 1.3e-8 without the d2^2 term
    d = np.abs(np.diag(C) - np.diag(ref)) / np.diag(ref)
    assert d.max() <= 2e-9, d.max()


def test_seven_products_match_ten_on_diagonal_pairs():
    X = _signals(130, 30000, seed=3)
    C7 = digit_covariance(X, 8192, seven=True)
    C10 = digit_covariance(X, 8192, seven=False)
    assert o64.rel_l2(C7, C10) <= 1e-15


def test_digit_covariance_edge_channels():
    M, N = 130, 20000
    X = _signals(M, N, seed=11)
    X[:, 5] = 0.0  # a channel of zeros
    X[:, 9] = np.float32(1e-3)
    X[7000, 9] = np.float32(5e4)  # tiny values next to a large transient
    C = digit_covariance(X, 8192)
    ref = o64.xxt(X)
    assert o64.rel_l2(C, ref) <= 1e-8
    assert np.all(C[5] == 0.0) and np.all(C[:, 5] == 0.0)
    X[123, 40] = np.float32(np.inf)
    C = digit_covariance(X, 8192)
    assert np.all(np.isnan(C[40])) and np.all(np.isnan(C[:, 40]))
    keep = np.setdiff1d(np.arange(M), [40])
    assert o64.rel_l2(C[np.ix_(keep, keep)], o64.xxt(X[:, keep])) <= 1e-8


def digits_from_bit_patterns(x, e):
    """digits4 and convert_stage as the converter warps compute them, in
    float32 and uint32: y1 = x 2^(22-e) + 1.5 2^23 (one rounding: the product
    is exact, and the FP64 sum is exact for every input, so its cast is the
    fma's rounding), vh = y1 - 1.5 2^23, rem = min(vh (-256) + x 2^(30-e),
    127) (exact), y2 = rem + 1.5 2^23; w = bits(y1) - 0x3F7F80, lo = bits(y2);
    d0 = byte 2 of w, d1 = byte 1 ^ 0x80, d2 = byte 0 ^ 0x80, d3 = byte 0 of
    lo, each read as a signed byte."""
    x = np.asarray(x, np.float32)
    m8 = np.float32(2.0 ** (22 - e))
    m = np.float32(2.0 ** (30 - e))
    c = np.float32(12582912.0)
    y1 = (x.astype(np.float64) * np.float64(m8) + 12582912.0).astype(np.float32)
    vh = y1 - c
    xm = x * m
    rem = np.minimum((vh.astype(np.float64) * -256.0 + xm.astype(np.float64)).astype(np.float32), np.float32(127.0))
    y2 = rem + c
    w = (y1.view(np.uint32).astype(np.int64) - 0x3F7F80) & 0xFFFFFFFF
    lo = y2.view(np.uint32).astype(np.int64)

    def sbyte(b):
        return ((b & 0xFF) ^ 0x80) - 0x80

    return [sbyte(w >> 16), sbyte(((w >> 8) & 0xFF) ^ 0x80), sbyte((w & 0xFF) ^ 0x80), sbyte(lo)]


def test_kernel_bit_patterns_give_the_digits():
    rng = np.random.default_rng(7)
    x = (rng.standard_normal(400000) * np.exp(rng.uniform(-12, 12, 400000))).astype(np.float32)
    x[:4] = [0.0, -0.0, np.float32(1e-40), np.float32(-3e-39)]
    for e in sorted({run_exponent(x), run_exponent(x[: 1000]), -20, 0, 9}):
        xx = x[np.abs(x.astype(np.float64)) < 2.0 ** e]  # the run's values lie below 2^e
        n = np.arange(min(16, xx.size))
        xx[: n.size] = ((2 * n + 1) * 2.0 ** (e - 23) * np.where(n % 2, -1, 1)).astype(np.float32)  # ties
        got = digits_from_bit_patterns(xx, e)
        want, _ = digits(xx, e)
        for k in range(4):
            assert np.array_equal(got[k], want[k]), (e, k)
