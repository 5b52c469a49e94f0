// Register-resident small DFTs with compile-time twiddles.
//
// RegDft<N, INV>::run(v) replaces v[0..N) by its N-point DFT
//     v[k] <- sum_n v[n] exp(s 2 pi i n k / N),   s = -1 forward, +1 inverse,
// fully unrolled: every index is a compile-time constant, so the values live
// in registers and every twiddle is an immediate operand.  N = 2, 3, 4, 5 are
// closed-form butterflies; a composite N = A * B is one Cooley-Tukey step
// (A-point DFTs over the B interleaved subsequences, twiddles w_N^{n2 k1},
// B-point DFTs) done in registers.  Twiddles come from a constexpr table
// evaluated at compile time from the Taylor series of sin and cos in double
// precision, then rounded once to float.
#pragma once

#include <cuda_runtime.h>

namespace ms3gpu {

// ---------------------------------------------------------------- constants

namespace ct {
constexpr double kPi = 3.14159265358979323846264338327950288;

// Taylor series on |x| <= pi/4 (after octant reduction): 14 terms reach
// double precision there.
__host__ __device__ constexpr double sin_series(double x) {
    double x2 = x * x, t = x, s = x;
    for (int k = 1; k < 14; k++) {
        t *= -x2 / ((2.0 * k) * (2.0 * k + 1.0));
        s += t;
    }
    return s;
}
__host__ __device__ constexpr double cos_series(double x) {
    double x2 = x * x, t = 1.0, s = 1.0;
    for (int k = 1; k < 14; k++) {
        t *= -x2 / ((2.0 * k - 1.0) * (2.0 * k));
        s += t;
    }
    return s;
}

// cos and sin of 2 pi e / n for integers, reduced exactly to an octant.
struct CosSin {
    double c, s;
};
__host__ __device__ constexpr CosSin cossin_2pi(long long e, long long n) {
    e %= n;
    if (e < 0) e += n;
    // angle = 2 pi e / n; work with the octant o = floor(8 e / n) and the
    // remainder r = 8 e - o n (so angle = (pi/4) (o + r / n)).
    const long long o = (8 * e) / n;
    const long long r = 8 * e - o * n;
    const double x = (kPi / 4.0) * (double)r / (double)n;  // in [0, pi/4)
    const double sx = sin_series(x), cx = cos_series(x);
    const double sy = sin_series(kPi / 4.0 - x), cy = cos_series(kPi / 4.0 - x);
    // angle = o * pi/4 + x
    switch (o) {
        case 0: return {cx, sx};
        case 1: return {sy, cy};    // pi/4 + x = pi/2 - (pi/4 - x)
        case 2: return {-sx, cx};   // pi/2 + x
        case 3: return {-cy, sy};   // pi - (pi/4 - x)
        case 4: return {-cx, -sx};  // pi + x
        case 5: return {-sy, -cy};
        case 6: return {sx, -cx};
        default: return {cy, -sy};
    }
}

template <int N>
struct RootTable {
    float re[N];
    float im[N];  // forward sign: exp(-2 pi i e / N)
    __host__ __device__ constexpr RootTable() : re(), im() {
        for (int e = 0; e < N; e++) {
            const CosSin cs = cossin_2pi(e, N);
            re[e] = (float)cs.c;
            im[e] = (float)(-cs.s);
        }
    }
};
}  // namespace ct

__host__ __device__ __forceinline__ float2 f2(float x, float y) {
    float2 r;
    r.x = x;
    r.y = y;
    return r;
}
__host__ __device__ __forceinline__ float2 radd(float2 a, float2 b) { return f2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 rsub(float2 a, float2 b) { return f2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 rmul(float2 a, float2 b) {
    return f2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// s*i*a with s = -1 (forward) or +1 (inverse)
template <bool INV>
__host__ __device__ __forceinline__ float2 rmul_si(float2 a) {
    return INV ? f2(-a.y, a.x) : f2(a.y, -a.x);
}

// v * w_N^e (forward) or v * conj(w_N^e) (inverse) with e a compile-time
// constant after unrolling; exact quarter turns become swaps and negations.
template <int N, bool INV>
__host__ __device__ __forceinline__ float2 twiddle_ct(float2 v, int e) {
    e %= N;
    if (e == 0) return v;
    if (4 * e == N) return rmul_si<INV>(v);
    if (2 * e == N) return f2(-v.x, -v.y);
    if (4 * e == 3 * N) return rmul_si<!INV>(v);
    constexpr ct::RootTable<N> t = ct::RootTable<N>();
    const float2 w = f2(t.re[e], INV ? -t.im[e] : t.im[e]);
    return rmul(v, w);
}

// ---------------------------------------------------------------- DFTs

template <int N>
struct SmallestFactor {
    static constexpr int f(int n, int d) { return (d * d > n) ? n : (n % d == 0 ? d : f(n, d + 1)); }
    static constexpr int value = (N % 4 == 0 && N > 4) ? 4 : f(N, 2);
};

template <int N, bool INV, bool PRIME_OR_BASE = (N <= 5 || SmallestFactor<N>::value == N)>
struct RegDft;

template <bool INV>
struct RegDft<1, INV, true> {
    __host__ __device__ __forceinline__ static void run(float2*) {}
};

template <bool INV>
struct RegDft<2, INV, true> {
    __host__ __device__ __forceinline__ static void run(float2* u) {
        const float2 a = u[0], b = u[1];
        u[0] = radd(a, b);
        u[1] = rsub(a, b);
    }
};

template <bool INV>
struct RegDft<3, INV, true> {
    __host__ __device__ __forceinline__ static void run(float2* u) {
        const float h = 0.866025403784438646763723f;  // sin(2 pi / 3)
        const float2 t = radd(u[1], u[2]);
        const float2 m = f2(u[0].x - 0.5f * t.x, u[0].y - 0.5f * t.y);
        const float2 d0 = rsub(u[1], u[2]);
        const float2 sd = rmul_si<INV>(f2(h * d0.x, h * d0.y));
        u[0] = radd(u[0], t);
        u[1] = radd(m, sd);
        u[2] = rsub(m, sd);
    }
};

template <bool INV>
struct RegDft<4, INV, true> {
    __host__ __device__ __forceinline__ static void run(float2* u) {
        const float2 a = radd(u[0], u[2]), b = rsub(u[0], u[2]);
        const float2 c = radd(u[1], u[3]), d = rmul_si<INV>(rsub(u[1], u[3]));
        u[0] = radd(a, c);
        u[2] = rsub(a, c);
        u[1] = radd(b, d);
        u[3] = rsub(b, d);
    }
};

template <bool INV>
struct RegDft<5, INV, true> {
    __host__ __device__ __forceinline__ static void run(float2* u) {
        const float c1 = 0.309016994374947424102293f;   // cos(2 pi / 5)
        const float c2 = -0.809016994374947424102293f;  // cos(4 pi / 5)
        const float s1 = 0.951056516295153572116439f;   // sin(2 pi / 5)
        const float s2 = 0.587785252292473129168706f;   // sin(4 pi / 5)
        const float2 a1 = radd(u[1], u[4]), b1 = rsub(u[1], u[4]);
        const float2 a2 = radd(u[2], u[3]), b2 = rsub(u[2], u[3]);
        const float2 p1 = f2(u[0].x + c1 * a1.x + c2 * a2.x, u[0].y + c1 * a1.y + c2 * a2.y);
        const float2 p2 = f2(u[0].x + c2 * a1.x + c1 * a2.x, u[0].y + c2 * a1.y + c1 * a2.y);
        const float2 q1 = rmul_si<INV>(f2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
        const float2 q2 = rmul_si<INV>(f2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
        u[0] = f2(u[0].x + a1.x + a2.x, u[0].y + a1.y + a2.y);
        u[1] = radd(p1, q1);
        u[4] = rsub(p1, q1);
        u[2] = radd(p2, q2);
        u[3] = rsub(p2, q2);
    }
};

// Prime N > 5: direct DFT with compile-time roots.
template <int N, bool INV>
struct RegDft<N, INV, true> {
    __host__ __device__ __forceinline__ static void run(float2* u) {
        float2 o[N];
#pragma unroll
        for (int k = 0; k < N; k++) {
            float2 acc = u[0];
#pragma unroll
            for (int n = 1; n < N; n++) acc = radd(acc, twiddle_ct<N, INV>(u[n], n * k));
            o[k] = acc;
        }
#pragma unroll
        for (int k = 0; k < N; k++) u[k] = o[k];
    }
};

// Composite N = A * B: input v[B n1 + n2], output v[k1 + A k2].
template <int N, bool INV>
struct RegDft<N, INV, false> {
    static constexpr int A = SmallestFactor<N>::value;
    static constexpr int B = N / A;
    __host__ __device__ __forceinline__ static void run(float2* v) {
        float2 t[N];
#pragma unroll
        for (int n2 = 0; n2 < B; n2++) {
            float2 u[A];
#pragma unroll
            for (int n1 = 0; n1 < A; n1++) u[n1] = v[B * n1 + n2];
            RegDft<A, INV>::run(u);
#pragma unroll
            for (int k1 = 0; k1 < A; k1++) t[n2 * A + k1] = twiddle_ct<N, INV>(u[k1], n2 * k1);
        }
#pragma unroll
        for (int k1 = 0; k1 < A; k1++) {
            float2 u[B];
#pragma unroll
            for (int n2 = 0; n2 < B; n2++) u[n2] = t[n2 * A + k1];
            RegDft<B, INV>::run(u);
#pragma unroll
            for (int k2 = 0; k2 < B; k2++) v[k1 + A * k2] = u[k2];
        }
    }
};

}  // namespace ms3gpu
