// Shared-memory batched FFT building block for the bandpass kernels.
//
// A CTA transforms G complex signals of length n that sit in shared memory
// as float2[n][G] (signal index fastest, so one row of G values is 8*G bytes
// and a half-warp reads a row of 16 signals as one 128-byte wavefront).
// The transform is a chain of Stockham autosort passes (decimation in time):
// pass s with radix r, after radices whose product is p, maps
//     u_q = src[i + q n/r] * w_{pr}^{q k},  k = i mod p,  q = 0..r-1
//     dst[(i - k) r + k + q p] = DFT_r(u)_q
// ping-ponging between two buffers.  Radices 2, 3, 4, 5, 8 have closed-form
// butterflies; any other prime up to kMaxGenericRadix uses an O(r^2) DFT.
// Twiddles are tabulated per pass on the host in FP64 and rounded once.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ms3gpu {

constexpr int kMaxPasses = 24;
constexpr int kMaxGenericRadix = 64;

// Description of one length-n transform as a chain of passes.
struct SubFft {
    int n;
    int npass;
    int twlen;                // total twiddle entries (float2)
    int radix[kMaxPasses];
    int p[kMaxPasses];        // product of the radices before this pass
    int twoff[kMaxPasses];    // offset of this pass's p*r twiddles
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// multiply by s*i  (s = -1 forward, +1 inverse):  s*i*(x + iy) = (-s y, s x)
template <bool INV>
__device__ __forceinline__ float2 mul_si(float2 a) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
}

template <int R, bool INV>
struct Butterfly;

template <bool INV>
struct Butterfly<2, INV> {
    __device__ __forceinline__ static void run(float2* u) {
        float2 a = u[0], b = u[1];
        u[0] = cadd(a, b);
        u[1] = csub(a, b);
    }
};

template <bool INV>
struct Butterfly<4, INV> {
    __device__ __forceinline__ static void run(float2* u) {
        float2 a = cadd(u[0], u[2]), b = csub(u[0], u[2]);
        float2 c = cadd(u[1], u[3]), d = mul_si<INV>(csub(u[1], u[3]));
        u[0] = cadd(a, c);
        u[2] = csub(a, c);
        u[1] = cadd(b, d);
        u[3] = csub(b, d);
    }
};

template <bool INV>
struct Butterfly<8, INV> {
    __device__ __forceinline__ static void run(float2* u) {
        const float h = 0.707106781186547524400844f;  // 1/sqrt(2)
        float2 a[4], b[4];
#pragma unroll
        for (int q = 0; q < 4; q++) {
            a[q] = cadd(u[q], u[q + 4]);
            b[q] = csub(u[q], u[q + 4]);
        }
        // b_q *= w8^q, w8 = exp(s 2 pi i / 8) = h (1 + s i)
        {
            float2 t = b[1];
            b[1] = INV ? make_float2(h * (t.x - t.y), h * (t.x + t.y))
                       : make_float2(h * (t.x + t.y), h * (t.y - t.x));
            b[2] = mul_si<INV>(b[2]);
            t = b[3];  // w8^3 = h (-1 + s i)
            b[3] = INV ? make_float2(-h * (t.x + t.y), h * (t.x - t.y))
                       : make_float2(h * (t.y - t.x), -h * (t.x + t.y));
        }
        Butterfly<4, INV>::run(a);
        Butterfly<4, INV>::run(b);
#pragma unroll
        for (int m = 0; m < 4; m++) {
            u[2 * m] = a[m];
            u[2 * m + 1] = b[m];
        }
    }
};

template <bool INV>
struct Butterfly<3, INV> {
    __device__ __forceinline__ static void run(float2* u) {
        const float h = 0.866025403784438646763723f;  // sin(2 pi / 3)
        float2 t = cadd(u[1], u[2]);
        float2 m = make_float2(u[0].x - 0.5f * t.x, u[0].y - 0.5f * t.y);
        float2 d = csub(u[1], u[2]);
        d = make_float2(h * d.x, h * d.y);
        float2 sd = mul_si<INV>(d);  // s i h (u1 - u2)
        u[0] = cadd(u[0], t);
        u[1] = cadd(m, sd);
        u[2] = csub(m, sd);
    }
};

template <bool INV>
struct Butterfly<5, INV> {
    __device__ __forceinline__ static void run(float2* u) {
        const float c1 = 0.309016994374947424102293f;   // cos(2 pi / 5)
        const float c2 = -0.809016994374947424102293f;  // cos(4 pi / 5)
        const float s1 = 0.951056516295153572116439f;   // sin(2 pi / 5)
        const float s2 = 0.587785252292473129168706f;   // sin(4 pi / 5)
        float2 a1 = cadd(u[1], u[4]), b1 = csub(u[1], u[4]);
        float2 a2 = cadd(u[2], u[3]), b2 = csub(u[2], u[3]);
        float2 p1 = make_float2(u[0].x + c1 * a1.x + c2 * a2.x, u[0].y + c1 * a1.y + c2 * a2.y);
        float2 p2 = make_float2(u[0].x + c2 * a1.x + c1 * a2.x, u[0].y + c2 * a1.y + c1 * a2.y);
        float2 q1 = mul_si<INV>(make_float2(s1 * b1.x + s2 * b2.x, s1 * b1.y + s2 * b2.y));
        float2 q2 = mul_si<INV>(make_float2(s2 * b1.x - s1 * b2.x, s2 * b1.y - s1 * b2.y));
        u[0] = make_float2(u[0].x + a1.x + a2.x, u[0].y + a1.y + a2.y);
        u[1] = cadd(p1, q1);
        u[4] = csub(p1, q1);
        u[2] = cadd(p2, q2);
        u[3] = csub(p2, q2);
    }
};

// One pass with a compile-time radix over G = 1 << log2G signals.
template <int R, bool INV>
__device__ __forceinline__ void stockham_pass(const float2* __restrict__ src, float2* __restrict__ dst,
                                              const float2* __restrict__ tw, int T, int p, int log2G) {
    const int G = 1 << log2G;
    const int items = T << log2G;
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int g = it & (G - 1);
        const int i = it >> log2G;
        const int k = i % p;
        const int j = (i - k) * R + k;
        float2 u[R];
#pragma unroll
        for (int q = 0; q < R; q++) u[q] = src[((i + q * T) << log2G) + g];
        if (k != 0) {
#pragma unroll
            for (int q = 1; q < R; q++) {
                float2 w = tw[k * R + q];
                if (INV) w.y = -w.y;
                u[q] = cmul(u[q], w);
            }
        }
        Butterfly<R, INV>::run(u);
#pragma unroll
        for (int q = 0; q < R; q++) dst[((j + q * p) << log2G) + g] = u[q];
    }
}

// One pass with a runtime prime radix R <= kMaxGenericRadix (direct DFT).
template <bool INV>
__device__ __noinline__ void stockham_pass_generic(const float2* __restrict__ src, float2* __restrict__ dst,
                                                   const float2* __restrict__ tw, int R, int T, int p,
                                                   int log2G) {
    const int G = 1 << log2G;
    const int items = T << log2G;
    float2 u[kMaxGenericRadix];
    for (int it = threadIdx.x; it < items; it += blockDim.x) {
        const int g = it & (G - 1);
        const int i = it >> log2G;
        const int k = i % p;
        const int j = (i - k) * R + k;
        for (int q = 0; q < R; q++) {
            float2 v = src[((i + q * T) << log2G) + g];
            float2 w = tw[k * R + q];
            if (INV) w.y = -w.y;
            u[q] = cmul(v, w);
        }
        for (int m = 0; m < R; m++) {
            float2 acc = make_float2(0.f, 0.f);
            for (int q = 0; q < R; q++) {
                const int e = (q * m) % R;
                float s, c;
                sincospif(2.0f * (float)e / (float)R, &s, &c);
                float2 w = make_float2(c, INV ? s : -s);
                acc = cadd(acc, cmul(u[q], w));
            }
            dst[((j + m * p) << log2G) + g] = acc;
        }
    }
}

// Runs the whole transform.  `a` holds the input; returns the buffer (a or
// b) holding the output.  `tw` is the plan's twiddle table (shared memory or
// global).  Ends with __syncthreads().
template <bool INV>
__device__ float2* fft_smem(float2* a, float2* b, const float2* tw, const SubFft& P, int log2G) {
    for (int s = 0; s < P.npass; s++) {
        const int r = P.radix[s];
        const int T = P.n / r;
        const float2* t = tw + P.twoff[s];
        switch (r) {
            case 2: stockham_pass<2, INV>(a, b, t, T, P.p[s], log2G); break;
            case 3: stockham_pass<3, INV>(a, b, t, T, P.p[s], log2G); break;
            case 4: stockham_pass<4, INV>(a, b, t, T, P.p[s], log2G); break;
            case 5: stockham_pass<5, INV>(a, b, t, T, P.p[s], log2G); break;
            case 8: stockham_pass<8, INV>(a, b, t, T, P.p[s], log2G); break;
            default: stockham_pass_generic<INV>(a, b, t, r, T, P.p[s], log2G); break;
        }
        __syncthreads();
        float2* tmp = a;
        a = b;
        b = tmp;
    }
    return a;
}

}  // namespace ms3gpu
