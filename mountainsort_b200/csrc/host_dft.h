// FP64 discrete Fourier transforms on the host, for the bandpass plan's
// tables (run once per window length and filter, never on the data path).
//
//   dft(x, s)   X[k] = sum_j x[j] exp(s 2 pi i j k / n), any n >= 1, s = -1 / +1
//
// Lengths whose prime factors are all at most 64 use a recursive mixed-radix
// decimation in time (each level: the sub-transforms of the p interleaved
// subsequences, then p-point DFTs with the twiddles w_n^{r k}); other
// lengths use Bluestein's chirp-z identity
//     j k = (j^2 + k^2 - (k - j)^2) / 2
//     X[k] = c[k] sum_j (x[j] c[j]) conj(c[k - j]),   c[j] = exp(s pi i j^2 / n)
// with the convolution done by transforms of a 5-smooth length >= 2n - 1.
// Roots are taken from one table of the top-level length with exact integer
// reduction of the exponents.
#pragma once

#include <cmath>
#include <complex>
#include <cstdint>
#include <vector>

namespace ms3gpu {
namespace hostdft {

using cd = std::complex<double>;

inline int64_t smallest_factor(int64_t n) {
    for (int64_t p = 2; p * p <= n; p++)
        if (n % p == 0) return p;
    return n;
}

inline int64_t largest_prime_factor(int64_t n) {
    int64_t m = 1;
    for (int64_t p = 2; p * p <= n; p++)
        while (n % p == 0) {
            m = p;
            n /= p;
        }
    return n > 1 ? std::max(n, m) : m;
}

inline bool smooth5(int64_t n) {
    for (int64_t p : {2, 3, 5})
        while (n % p == 0) n /= p;
    return n == 1;
}

inline int64_t next_smooth5(int64_t n) {
    while (!smooth5(n)) n++;
    return n;
}

// n-th roots exp(s 2 pi i e / n), e < n
inline std::vector<cd> roots(int64_t n, int s) {
    std::vector<cd> r((size_t)n);
    for (int64_t e = 0; e < n; e++) {
        const double a = s * 2.0 * M_PI * (double)e / (double)n;
        r[(size_t)e] = cd(std::cos(a), std::sin(a));
    }
    return r;
}

// out[0..n) = DFT of in[0], in[stride], ...; root table rt of length N0 with
// n dividing N0.
inline void mixed_radix(const cd* in, int64_t stride, cd* out, int64_t n, const std::vector<cd>& rt, int64_t N0) {
    if (n == 1) {
        out[0] = in[0];
        return;
    }
    const int64_t p = smallest_factor(n), m = n / p;
    for (int64_t r = 0; r < p; r++) mixed_radix(in + r * stride, stride * p, out + r * m, m, rt, N0);
    const int64_t step = N0 / n;  // w_n^e = w_N0^(e * step)
    std::vector<cd> v((size_t)p), w((size_t)p);
    for (int64_t k = 0; k < m; k++) {
        for (int64_t r = 0; r < p; r++) v[(size_t)r] = out[r * m + k] * rt[(size_t)((r * k % n) * step)];
        for (int64_t q = 0; q < p; q++) {
            cd acc = 0;
            for (int64_t r = 0; r < p; r++) acc += v[(size_t)r] * rt[(size_t)(((r * q) % p) * m * step)];
            w[(size_t)q] = acc;
        }
        for (int64_t q = 0; q < p; q++) out[k + q * m] = w[(size_t)q];
    }
}

inline std::vector<cd> dft(const std::vector<cd>& x, int s) {
    const int64_t n = (int64_t)x.size();
    std::vector<cd> out((size_t)n);
    if (n == 0) return out;
    if (largest_prime_factor(n) <= 64) {
        const std::vector<cd> rt = roots(n, s);
        mixed_radix(x.data(), 1, out.data(), n, rt, n);
        return out;
    }
    // Bluestein
    const int64_t Q = next_smooth5(2 * n - 1);
    std::vector<cd> c((size_t)n);
    for (int64_t j = 0; j < n; j++) {
        const int64_t e = (int64_t)((__int128)j * j % (2 * n));  // exact before the trig call
        const double a = s * M_PI * (double)e / (double)n;
        c[(size_t)j] = cd(std::cos(a), std::sin(a));
    }
    std::vector<cd> a((size_t)Q, cd(0)), b((size_t)Q, cd(0));
    for (int64_t j = 0; j < n; j++) a[(size_t)j] = x[(size_t)j] * c[(size_t)j];
    b[0] = std::conj(c[0]);
    for (int64_t j = 1; j < n; j++) b[(size_t)j] = b[(size_t)(Q - j)] = std::conj(c[(size_t)j]);
    const std::vector<cd> A = dft(a, -1), B = dft(b, -1);
    std::vector<cd> AB((size_t)Q);
    for (int64_t k = 0; k < Q; k++) AB[(size_t)k] = A[(size_t)k] * B[(size_t)k];
    const std::vector<cd> conv = dft(AB, +1);
    for (int64_t k = 0; k < n; k++) out[(size_t)k] = c[(size_t)k] * conv[(size_t)k] / (double)Q;
    return out;
}

}  // namespace hostdft
}  // namespace ms3gpu
