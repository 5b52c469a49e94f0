// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// Batched single-precision complex FFT used by the CPU restatement of
// ms3.bandpass_filter.  The reference calls FFTW 3 (single precision,
// `fftwf_plan_many_dft` with rank 1, n = L, howmany = M, istride = M,
// idist = 1, FFTW_ESTIMATE; packages/ms3/p_bandpass_filter.cpp:64-75).
// FFTW is a third-party dependency that is not vendored in the reference
// (a Debian `libfftw3-dev` build dependency, debian/control:5, no pinned
// version) and is not installed here, so this file restates the published
// algorithm it computes: the unnormalised DFT
//     forward:  Y[k] = sum_j X[j] exp(-2 pi i j k / L)
//     backward: Y[k] = sum_j X[j] exp(+2 pi i j k / L)
// evaluated in FP32 arithmetic with twiddles computed in FP64 and rounded
// once.  Any accurate FP32 FFT reproduces FFTW's output to about 1e-7
// relative; that is the parity floor of the oracle.
//
// Layout: `howmany` transforms interleaved with the transform index fastest,
// exactly FFTW's istride = howmany, idist = 1 layout of an M x L channel-major
// window: element j of transform b sits at (j * howmany + b).
//
// Algorithm: Stockham autosort, decimation in time.  Pass with radix r and
// p = product of the radices already applied:
//     for i in [0, L/r):  k = i mod p
//         u_q = x[i + q L/r] * w_{p r}^{q k}        (q = 0..r-1)
//         u   = DFT_r(u)
//         y[(i - k) r + k + q p] = u_q
// Radices 4, 2, 3, 5 have closed-form butterflies; any other prime up to 64
// uses the O(r^2) direct DFT with precomputed roots.  Lengths with a prime
// factor above 64 use Bluestein's chirp-z algorithm: with
// c[n] = exp(s pi i n^2 / L),  X[k] = c[k] sum_n (x[n] c[n]) conj(c[k - n]),
// a linear convolution evaluated with power-of-two FFTs of size P >= 2L - 1.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <vector>

namespace ms3ref {

struct FftPass {
    int r;
    int64_t p;
    std::vector<float> tw;     // (p * r) complex, interleaved re/im: w_{pr}^{q k} at [(k*r+q)*2]
    std::vector<float> roots;  // r complex roots w_r^{m} for the generic radix
};

inline int64_t max_prime_factor(int64_t n) {
    int64_t m = 1;
    for (int64_t p = 2; p * p <= n; p++)
        while (n % p == 0) { m = p > m ? p : m; n /= p; }
    return n > 1 ? (n > m ? n : m) : m;
}

class BatchedFft {
public:
    BatchedFft(int64_t L, int sign) : L_(L), sign_(sign) {
        if (L < 1) throw std::invalid_argument("FFT length must be >= 1");
        if (L > 64 && max_prime_factor(L) > 64) {
            init_bluestein();
            return;
        }
        std::vector<int> radices;
        int64_t n = L;
        while (n % 4 == 0) { radices.push_back(4); n /= 4; }
        while (n % 2 == 0) { radices.push_back(2); n /= 2; }
        for (int f = 3; (int64_t)f * f <= n; f += 2)
            while (n % f == 0) { radices.push_back(f); n /= f; }
        if (n > 1) radices.push_back((int)n);
        int64_t p = 1;
        for (int r : radices) {
            FftPass ps;
            ps.r = r;
            ps.p = p;
            ps.tw.resize((size_t)(p * r * 2));
            for (int64_t k = 0; k < p; k++)
                for (int q = 0; q < r; q++) {
                    // angle = sign * 2 pi q k / (p r), reduced exactly in integers first
                    int64_t num = (q * k) % (p * r);
                    double a = sign * 2.0 * M_PI * (double)num / (double)(p * r);
                    ps.tw[(k * r + q) * 2 + 0] = (float)std::cos(a);
                    ps.tw[(k * r + q) * 2 + 1] = (float)std::sin(a);
                }
            if (r != 2 && r != 3 && r != 4 && r != 5) {
                ps.roots.resize((size_t)r * 2);
                for (int m = 0; m < r; m++) {
                    double a = sign * 2.0 * M_PI * (double)m / (double)r;
                    ps.roots[m * 2 + 0] = (float)std::cos(a);
                    ps.roots[m * 2 + 1] = (float)std::sin(a);
                }
            }
            passes_.push_back(std::move(ps));
            p *= r;
        }
    }

    int64_t length() const { return L_; }

    // In-place transform of `howmany` interleaved signals in `data`
    // (L * howmany complex values = 2 * L * howmany floats).  `work` must
    // hold the same number of floats.
    void execute(float* data, float* work, int64_t howmany) const {
        if (blue_) {
            execute_bluestein(data, howmany);
            return;
        }
        float* x = data;
        float* y = work;
        for (const FftPass& ps : passes_) {
            run_pass(ps, x, y, howmany);
            std::swap(x, y);
        }
        if (x != data) std::memcpy(data, x, sizeof(float) * 2 * L_ * howmany);
    }

private:
    void init_bluestein() {
        int64_t P = 1;
        while (P < 2 * L_ - 1) P <<= 1;
        P_ = P;
        fwdP_.reset(new BatchedFft(P, -1));
        invP_.reset(new BatchedFft(P, +1));
        chirp_.resize((size_t)(2 * L_));
        for (int64_t n = 0; n < L_; n++) {
            // n^2 mod 2L keeps the angle exact before the FP64 trig call
            const int64_t e = (int64_t)((__int128)n * n % (2 * L_));
            const double a = sign_ * M_PI * (double)e / (double)L_;
            chirp_[(size_t)(2 * n)] = (float)std::cos(a);
            chirp_[(size_t)(2 * n + 1)] = (float)std::sin(a);
        }
        // bhat = FFT_P(b), b[m] = conj(c[m]) for |m| < L (negative m wrapped to P - m)
        std::vector<float> b((size_t)(2 * P), 0.f), w((size_t)(2 * P));
        for (int64_t m = 0; m < L_; m++) {
            const float re = chirp_[(size_t)(2 * m)], im = -chirp_[(size_t)(2 * m + 1)];
            b[(size_t)(2 * m)] = re; b[(size_t)(2 * m + 1)] = im;
            if (m > 0) { b[(size_t)(2 * (P - m))] = re; b[(size_t)(2 * (P - m) + 1)] = im; }
        }
        fwdP_->execute(b.data(), w.data(), 1);
        bhat_ = std::move(b);
        blue_ = true;
    }

    void execute_bluestein(float* data, int64_t B) const {
        const int64_t P = P_;
        std::vector<float> a((size_t)(2 * P * B), 0.f), w((size_t)(2 * P * B));
        for (int64_t n = 0; n < L_; n++) {
            const float cr = chirp_[(size_t)(2 * n)], ci = chirp_[(size_t)(2 * n + 1)];
            for (int64_t b = 0; b < B; b++) {
                const float xr = data[(n * B + b) * 2], xi = data[(n * B + b) * 2 + 1];
                a[(size_t)((n * B + b) * 2)] = xr * cr - xi * ci;
                a[(size_t)((n * B + b) * 2 + 1)] = xr * ci + xi * cr;
            }
        }
        fwdP_->execute(a.data(), w.data(), B);
        for (int64_t k = 0; k < P; k++) {
            const float br = bhat_[(size_t)(2 * k)], bi = bhat_[(size_t)(2 * k + 1)];
            for (int64_t b = 0; b < B; b++) {
                float* v = &a[(size_t)((k * B + b) * 2)];
                const float vr = v[0], vi = v[1];
                v[0] = vr * br - vi * bi;
                v[1] = vr * bi + vi * br;
            }
        }
        invP_->execute(a.data(), w.data(), B);
        const float inv = 1.0f / (float)P;
        for (int64_t k = 0; k < L_; k++) {
            const float cr = chirp_[(size_t)(2 * k)], ci = chirp_[(size_t)(2 * k + 1)];
            for (int64_t b = 0; b < B; b++) {
                const float yr = a[(size_t)((k * B + b) * 2)] * inv, yi = a[(size_t)((k * B + b) * 2 + 1)] * inv;
                data[(k * B + b) * 2] = yr * cr - yi * ci;
                data[(k * B + b) * 2 + 1] = yr * ci + yi * cr;
            }
        }
    }

    void run_pass(const FftPass& ps, const float* x, float* y, int64_t B) const {
        const int r = ps.r;
        const int64_t p = ps.p;
        const int64_t T = L_ / r;
        const float s = (float)sign_;
        float ur[64], ui[64];
        std::vector<float> gr, gi;
        if (r > 64) { gr.resize(r); gi.resize(r); }
        float* vr = (r > 64) ? gr.data() : ur;
        float* vi = (r > 64) ? gi.data() : ui;
        std::vector<float> outr, outi;
        if (r != 2 && r != 3 && r != 4 && r != 5) { outr.resize(r); outi.resize(r); }
        for (int64_t i = 0; i < T; i++) {
            const int64_t k = i % p;
            const int64_t j = (i - k) * r + k;
            const float* tw = &ps.tw[(size_t)(k * r * 2)];
            for (int64_t b = 0; b < B; b++) {
                for (int q = 0; q < r; q++) {
                    const float* src = x + ((i + q * T) * B + b) * 2;
                    float a = src[0], c = src[1];
                    float wr = tw[q * 2], wi = tw[q * 2 + 1];
                    vr[q] = a * wr - c * wi;
                    vi[q] = a * wi + c * wr;
                }
                if (r == 2) {
                    float r0 = vr[0] + vr[1], i0 = vi[0] + vi[1];
                    float r1 = vr[0] - vr[1], i1 = vi[0] - vi[1];
                    vr[0] = r0; vi[0] = i0; vr[1] = r1; vi[1] = i1;
                } else if (r == 4) {
                    float ar = vr[0] + vr[2], ai = vi[0] + vi[2];
                    float br = vr[0] - vr[2], bi = vi[0] - vi[2];
                    float cr = vr[1] + vr[3], ci = vi[1] + vi[3];
                    float dr = vr[1] - vr[3], di = vi[1] - vi[3];
                    // w = s*i ; w*d = (-s*di, s*dr)
                    float wdr = -s * di, wdi = s * dr;
                    vr[0] = ar + cr; vi[0] = ai + ci;
                    vr[2] = ar - cr; vi[2] = ai - ci;
                    vr[1] = br + wdr; vi[1] = bi + wdi;
                    vr[3] = br - wdr; vi[3] = bi - wdi;
                } else if (r == 3) {
                    const float h = 0.866025403784438646763723f;  // sin(2 pi / 3)
                    float tr = vr[1] + vr[2], ti = vi[1] + vi[2];
                    float mr = vr[0] - 0.5f * tr, mi = vi[0] - 0.5f * ti;
                    float dr = s * h * (vr[1] - vr[2]), di = s * h * (vi[1] - vi[2]);
                    vr[0] = vr[0] + tr; vi[0] = vi[0] + ti;
                    // i * (dr + i di) = -di + i dr
                    vr[1] = mr - di; vi[1] = mi + dr;
                    vr[2] = mr + di; vi[2] = mi - dr;
                } else if (r == 5) {
                    const float c1 = 0.309016994374947424102293f;   // cos(2 pi / 5)
                    const float c2 = -0.809016994374947424102293f;  // cos(4 pi / 5)
                    const float s1 = 0.951056516295153572116439f;   // sin(2 pi / 5)
                    const float s2 = 0.587785252292473129168706f;   // sin(4 pi / 5)
                    float a1r = vr[1] + vr[4], a1i = vi[1] + vi[4];
                    float b1r = vr[1] - vr[4], b1i = vi[1] - vi[4];
                    float a2r = vr[2] + vr[3], a2i = vi[2] + vi[3];
                    float b2r = vr[2] - vr[3], b2i = vi[2] - vi[3];
                    float p1r = vr[0] + c1 * a1r + c2 * a2r, p1i = vi[0] + c1 * a1i + c2 * a2i;
                    float p2r = vr[0] + c2 * a1r + c1 * a2r, p2i = vi[0] + c2 * a1i + c1 * a2i;
                    float q1r = s * (s1 * b1r + s2 * b2r), q1i = s * (s1 * b1i + s2 * b2i);
                    float q2r = s * (s2 * b1r - s1 * b2r), q2i = s * (s2 * b1i - s1 * b2i);
                    vr[0] = vr[0] + a1r + a2r; vi[0] = vi[0] + a1i + a2i;
                    // y1 = p1 + i q1, y4 = p1 - i q1, y2 = p2 + i q2, y3 = p2 - i q2
                    vr[1] = p1r - q1i; vi[1] = p1i + q1r;
                    vr[4] = p1r + q1i; vi[4] = p1i - q1r;
                    vr[2] = p2r - q2i; vi[2] = p2i + q2r;
                    vr[3] = p2r + q2i; vi[3] = p2i - q2r;
                } else {
                    const float* ro = ps.roots.data();
                    for (int m = 0; m < r; m++) {
                        float sr = 0.f, si = 0.f;
                        for (int q = 0; q < r; q++) {
                            int e = (int)(((int64_t)q * m) % r);
                            float wr = ro[e * 2], wi = ro[e * 2 + 1];
                            sr += vr[q] * wr - vi[q] * wi;
                            si += vr[q] * wi + vi[q] * wr;
                        }
                        outr[m] = sr; outi[m] = si;
                    }
                    for (int m = 0; m < r; m++) { vr[m] = outr[m]; vi[m] = outi[m]; }
                }
                for (int q = 0; q < r; q++) {
                    float* dst = y + ((j + q * p) * B + b) * 2;
                    dst[0] = vr[q];
                    dst[1] = vi[q];
                }
            }
        }
    }

    int64_t L_;
    int sign_;
    std::vector<FftPass> passes_;
    bool blue_ = false;
    int64_t P_ = 0;
    std::unique_ptr<BatchedFft> fwdP_, invP_;
    std::vector<float> chirp_, bhat_;
};

}  // namespace ms3ref
