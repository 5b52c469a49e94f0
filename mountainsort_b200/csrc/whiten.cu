// ms3.whiten on the GPU.
//
// Reference: packages/ms3/p_whiten.cpp:45-206 and packages/ms3/pca.cpp.
//   pass 1   XXt = sum_t x_t x_t^T / (N-1)            (p_whiten.cpp:64-118)
//   matrix   W = whitening_matrix_from_XXt(XXt)        (pca.cpp:635-651)
//   pass 2   y_t = W^T x_t, rounded to multiples of 1e-4, optional int16
//                                                     (p_whiten.cpp:153-206)
//
// Kernels:
//   cov_partial / cov_reduce   channel covariance: 64x64 channel tiles of the
//       upper triangle x time slices.  Products are summed in FP32 over 32
//       timepoints (round-to-nearest FMA, unbiased) and those sums in FP64,
//       so the result agrees with the reference's double sum of float
//       products to ~1e-10 relative.  Partial tiles are reduced in a fixed
//       order: repeat runs are bit-identical.
//   pca_cluster   the reference's power iteration, FP64, one thread-block
//       cluster: the working matrix XXtw is split by rows across the CTAs'
//       shared memory (global memory beyond what fits); each matvec result
//       is broadcast to every CTA through distributed shared memory, one
//       cluster barrier per matvec.  Deflation (I-cc')X(I-cc') is applied as
//       the equivalent symmetric rank-2 update.
//   w_assemble    W = (C D) C^T in the reference's exact summation order.
//   apply_gemm    y = W^T x with W rounded to float, FP32 FMA accumulation,
//       1e-4 rounding in FP64 in the epilogue (bit-exact rounding rule).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>

#include "common.cuh"
#include "ms3gpu.h"
#include "tc_sm100.cuh"
#include "whiten.h"

namespace cg = cooperative_groups;

namespace ms3gpu {

namespace {

// ------------------------------------------------------------ covariance

constexpr int kCT = 64;   // channel tile
constexpr int kTT = 32;  // timepoints summed in FP32 before the FP64 add (slice granularity)
constexpr int kTG = 32;   // timepoints per shared-memory stage of cov_partial

__global__ void __launch_bounds__(256) cov_partial(const float* __restrict__ X, int64_t M, int64_t r0, int64_t N,
                                                   int nb, int64_t tslice, double* __restrict__ partials) {
    __shared__ __align__(16) float As[kTG][kCT];
    __shared__ __align__(16) float Bs[kTG][kCT];
    const int pair = blockIdx.x;
    const int npairs = gridDim.x;
    int bi = 0, rem = pair;
    while (rem >= nb - bi) { rem -= nb - bi; bi++; }
    const int bj = bi + rem;
    const int64_t t_begin = r0 + (int64_t)blockIdx.y * tslice;
    const int64_t t_end = min(N, t_begin + tslice);
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double accd[4][4];
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            accd[i][j] = 0.0;
            acc[i][j] = 0.f;
        }

    for (int64_t t0 = t_begin; t0 < t_end; t0 += kTG) {
        for (int e = threadIdx.x; e < kTG * kCT; e += blockDim.x) {
            const int tt = e / kCT, c = e % kCT;
            const int64_t t = t0 + tt;
            const int64_t ma = (int64_t)bi * kCT + c, mb = (int64_t)bj * kCT + c;
            const bool tv = t < t_end;
            As[tt][c] = (tv && ma < M) ? X[t * M + ma] : 0.f;
            Bs[tt][c] = (tv && mb < M) ? X[t * M + mb] : 0.f;
        }
        __syncthreads();
#pragma unroll 8
        for (int tt = 0; tt < kTG; tt++) {
            const float4 a = *reinterpret_cast<const float4*>(&As[tt][ty * 4]);
            const float4 b = *reinterpret_cast<const float4*>(&Bs[tt][tx * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w};
            const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        // flush the FP32 run every kTT timepoints of the slice
        if (((t0 - t_begin + kTG) % kTT) == 0 || t0 + kTG >= t_end) {
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    accd[i][j] += (double)acc[i][j];
                    acc[i][j] = 0.f;
                }
        }
        __syncthreads();
    }
    double* dst = partials + ((size_t)blockIdx.y * npairs + pair) * (kCT * kCT);
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) dst[(ty * 4 + i) * kCT + tx * 4 + j] = accd[i][j];
}

// cov_partial8: the same partial tiles as cov_partial with 8 x 8 register
// micro-tiles (64 threads per 64 x 64 tile), a 3-deep cp.async ring of
// 16-timepoint stages, and packed FP32 FMAs (fma.rn.f32x2: two independent
// round-to-nearest FMAs per instruction, the same values as two fmaf calls),
// which halve the issue slots of the inner product.  FP32 runs of kTT
// timepoints are flushed to FP64, as in cov_partial, so both kernels produce
// the same FP32 partial sums.  Needs M % 4 == 0 and a 16-byte aligned X.
constexpr int kTS = 16;     // timepoints per stage
constexpr int kStages8 = 3;

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, bool valid) {
    const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(smem_dst));
    const int n = valid ? 16 : 0;  // src-size 0: zero fill
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(gsrc), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// (a, a) as a packed FP32 pair
__device__ __forceinline__ uint64_t dup_f32x2(float a) {
    uint64_t r;
    asm("mov.b64 %0, {%1, %1};" : "=l"(r) : "f"(a));
    return r;
}
// d = a * b + d on both halves of packed FP32 pairs
__device__ __forceinline__ void fma_f32x2(uint64_t& d, uint64_t a, uint64_t b) {
    asm("fma.rn.f32x2 %0, %1, %2, %0;" : "+l"(d) : "l"(a), "l"(b));
}

__global__ void __launch_bounds__(64) cov_partial8(const float* __restrict__ X, int64_t M, int64_t r0, int64_t N,
                                                   int nb, int64_t tslice, double* __restrict__ partials) {
    __shared__ __align__(16) float As[kStages8][kTS][kCT];
    __shared__ __align__(16) float Bs[kStages8][kTS][kCT];
    const int pair = blockIdx.x;
    const int npairs = gridDim.x;
    int bi = 0, rem = pair;
    while (rem >= nb - bi) { rem -= nb - bi; bi++; }
    const int bj = bi + rem;
    const bool diag = (bi == bj);
    const int64_t t_begin = r0 + (int64_t)blockIdx.y * tslice;
    const int64_t t_end = min(N, t_begin + tslice);
    const int nst = (int)((t_end - t_begin + kTS - 1) / kTS);
    const int tid = threadIdx.x;
    const int tx = tid & 7, ty = tid >> 3;

    // each thread copies 4 float4 of A (and of B): stage rows tt = tid/16 + 4k, 16-byte column tid%16
    auto issue = [&](int st, int buf) {
        const int64_t tb = t_begin + (int64_t)st * kTS;
        const int c4 = (tid & 15) * 4;
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int tt = (tid >> 4) + 4 * k;
            const int64_t t = tb + tt;
            const int64_t ca = (int64_t)bi * kCT + c4, cb = (int64_t)bj * kCT + c4;
            const bool tv = t < t_end;
            cp_async16(&As[buf][tt][c4], X + (tv && ca < M ? t * M + ca : 0), tv && ca < M);
            if (!diag) cp_async16(&Bs[buf][tt][c4], X + (tv && cb < M ? t * M + cb : 0), tv && cb < M);
        }
    };

    uint64_t acc[8][4];  // packed pairs: columns (2j, 2j + 1) of row i
    double accd[8][8];
#pragma unroll
    for (int i = 0; i < 8; i++) {
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0ull;
#pragma unroll
        for (int j = 0; j < 8; j++) accd[i][j] = 0.0;
    }
#pragma unroll
    for (int p = 0; p < kStages8 - 1; p++) {
        if (p < nst) issue(p, p);
        cp_async_commit();
    }
    for (int st = 0; st < nst; st++) {
        const int buf = st % kStages8;
        if (st + kStages8 - 1 < nst) issue(st + kStages8 - 1, (st + kStages8 - 1) % kStages8);
        cp_async_commit();
        cp_async_wait<kStages8 - 1>();
        __syncthreads();
        const float(*A)[kCT] = As[buf];
        const float(*B)[kCT] = diag ? As[buf] : Bs[buf];
#pragma unroll
        for (int tt = 0; tt < kTS; tt++) {
            const float4 a0 = *reinterpret_cast<const float4*>(&A[tt][ty * 4]);
            const float4 a1 = *reinterpret_cast<const float4*>(&A[tt][32 + ty * 4]);
            const ulonglong2 b0 = *reinterpret_cast<const ulonglong2*>(&B[tt][tx * 4]);
            const ulonglong2 b1 = *reinterpret_cast<const ulonglong2*>(&B[tt][32 + tx * 4]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const uint64_t bv[4] = {b0.x, b0.y, b1.x, b1.y};
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const uint64_t ai = dup_f32x2(av[i]);
#pragma unroll
                for (int j = 0; j < 4; j++) fma_f32x2(acc[i][j], ai, bv[j]);
            }
        }
        __syncthreads();
        if ((((st + 1) * kTS) % kTT) == 0 || st + 1 == nst) {
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    accd[i][2 * j] += (double)__uint_as_float((uint32_t)acc[i][j]);
                    accd[i][2 * j + 1] += (double)__uint_as_float((uint32_t)(acc[i][j] >> 32));
                    acc[i][j] = 0ull;
                }
        }
    }
    double* dst = partials + ((size_t)blockIdx.y * npairs + pair) * (kCT * kCT);
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const int r = (i < 4) ? ty * 4 + i : 32 + ty * 4 + (i - 4);
#pragma unroll
        for (int j = 0; j < 8; j++) {
            const int c = (j < 4) ? tx * 4 + j : 32 + tx * 4 + (j - 4);
            dst[r * kCT + c] = accd[i][j];
        }
    }
}

__global__ void cov_reduce(const double* __restrict__ partials, int S, int npairs, int nb, int64_t M,
                           int64_t N, double* __restrict__ XXt) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (int64_t)npairs * kCT * kCT) return;
    const int pair = (int)(idx / (kCT * kCT));
    const int e = (int)(idx % (kCT * kCT));
    const int r = e / kCT, c = e % kCT;
    int bi = 0, rem = pair;
    while (rem >= nb - bi) { rem -= nb - bi; bi++; }
    const int bj = bi + rem;
    const int64_t i = (int64_t)bi * kCT + r, j = (int64_t)bj * kCT + c;
    if (i >= M || j >= M) return;
    double s = 0.0;
    for (int k = 0; k < S; k++) s += partials[((size_t)k * npairs + pair) * (kCT * kCT) + e];
    if (N > 1) s /= (double)(N - 1);
    XXt[i + M * j] = s;
    XXt[j + M * i] = s;
}

// ------------------------------------------------------------ power iteration

constexpr int kPcaThreads = 512;

// Sum over the block of per-thread values; every thread returns the total.
// Fixed reduction tree: identical results in every CTA of the cluster.
__device__ double block_sum(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) red[w] = v;
    __syncthreads();
    double t = 0.0;
    const int nw = blockDim.x >> 5;
    for (int i = 0; i < nw; i++) t += red[i];
    return t;
}

// Sum over n < M of f(n), formed by one warp: lane l adds f(l), f(l + 32),
// ... in order, then a 32-lane XOR tree.  Addition is commutative, so every
// lane ends with the same bits; both power-iteration kernels form their norms
// and dot products this way, which keeps their results identical.  The
// dependent chain is M/32 adds plus five shuffles (the previous per-chunk
// trees cost five shuffles per 32 elements).
template <class F>
__device__ __forceinline__ double warp_ordered_sum(int M, F f) {
    const int l = threadIdx.x & 31;
    double t = 0.0;
    for (int n = l; n < M; n += 32) t += f(n);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    return t;
}

// y = X v for this CTA's rows, written into `dst` of every CTA in the cluster,
// followed by a cluster barrier.
__device__ void cluster_matvec(cg::cluster_group& cluster, const double* __restrict__ X, int RS, int r0,
                               int nr, int M, const double* __restrict__ v, double* dst) {
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int nw = blockDim.x >> 5;
    const int CS = (int)cluster.num_blocks();
    for (int r = w; r < nr; r += nw) {
        const double* row = X + (size_t)r * RS;
        double s = 0.0;
        for (int n = l; n < M; n += 32) s += row[n] * v[n];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        for (int d = l; d < CS; d += 32) {
            double* remote = cluster.map_shared_rank(dst, d);
            remote[r0 + r] = s;
        }
    }
    cluster.sync();
}

// pca_from_XXt (pca.cpp:172-195) for all M components.
// Xg: optional global copy of the rows (when they do not fit shared memory).
__global__ void __launch_bounds__(kPcaThreads) pca_cluster(const double* __restrict__ XXt, int M, int R,
                                                            int num_iter, int rows_in_smem, double* Xg,
                                                            double* __restrict__ comps,
                                                            double* __restrict__ sigma) {
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    extern __shared__ double sm[];
    const int RS = M + 1;  // padded row stride
    double* vb[2];
    vb[0] = sm;
    vb[1] = vb[0] + M;
    double* vinit = vb[1] + M;
    double* red = vinit + M;
    double* X = rows_in_smem ? (red + 32) : (Xg + (size_t)rank * R * RS);
    const int r0 = rank * R;
    const int nr = max(0, min(R, M - r0));

    for (int idx = threadIdx.x; idx < nr * M; idx += blockDim.x) {
        const int r = idx % nr, n = idx / nr;
        X[(size_t)r * RS + n] = XXt[(size_t)(r0 + r) + (size_t)M * n];
    }
    // start vector sin(i+1), normalised (pca.cpp:546-549, 457-466)
    for (int n = threadIdx.x; n < M; n += blockDim.x) vinit[n] = sin((double)(n + 1));
    __syncthreads();
    {
        double part = 0.0;
        for (int n = threadIdx.x; n < M; n += blockDim.x) part += vinit[n] * vinit[n];
        const double nrm = sqrt(block_sum(part, red));
        __syncthreads();
        if (nrm != 0.0)
            for (int n = threadIdx.x; n < M; n += blockDim.x) vinit[n] = vinit[n] / nrm;
    }
    cluster.sync();

    for (int k = 0; k < M; k++) {
        int cur = 0;
        for (int n = threadIdx.x; n < M; n += blockDim.x) vb[0][n] = vinit[n];
        __syncthreads();
        double sig = 0.0;
        for (int it = 0; it < num_iter; it++) {
            const int nxt = cur ^ 1;
            cluster_matvec(cluster, X, RS, r0, nr, M, vb[cur], vb[nxt]);
            const double* y = vb[nxt];
            sig = sqrt(warp_ordered_sum(M, [&](int n) { return y[n] * y[n]; }));
            __syncthreads();
            if (sig != 0.0)
                for (int n = threadIdx.x; n < M; n += blockDim.x) vb[nxt][n] = vb[nxt][n] / sig;
            __syncthreads();
            cur = nxt;
        }
        const double* v = vb[cur];
        if (rank == 0) {
            for (int n = threadIdx.x; n < M; n += blockDim.x) comps[(size_t)n + (size_t)M * k] = v[n];
            if (threadIdx.x == 0) sigma[k] = sig;
        }
        // deflation: X <- X - v u' - u v' + (v'u) v v',  u = X v
        double* u = vb[cur ^ 1];
        cluster_matvec(cluster, X, RS, r0, nr, M, v, u);
        const double alpha = warp_ordered_sum(M, [&](int n) { return v[n] * u[n]; });
        for (int idx = threadIdx.x; idx < nr * M; idx += blockDim.x) {
            const int r = idx / M, n = idx % M;
            const int m = r0 + r;
            const double s = __dadd_rn(__dmul_rn(v[m], u[n]), __dmul_rn(u[m], v[n]));
            const double x = __dsub_rn(X[(size_t)r * RS + n], s);
            X[(size_t)r * RS + n] = __dadd_rn(x, __dmul_rn(alpha, __dmul_rn(v[m], v[n])));
        }
        cluster.sync();
    }
}

// The same power iteration with the working matrix in registers, for M up
// to 128 * RPW (8 CTAs x 16 warps x RPW rows) and 32 * CPL columns: lane l
// of a warp holds its RPW rows at columns l + 32 j.  Every sum is formed in
// the order pca_cluster forms it (per-lane column sums then the XOR
// shuffle tree for a matvec row; 32-element warp trees summed in warp order
// for a norm or a dot product), so components, sigma and W are identical.
//
// The matvec results are exchanged point to point instead of through a
// cluster barrier: the warp that owns row m stores y[m] into every CTA's
// receive buffer with st.async, whose bytes complete on the receiving CTA's
// own mbarrier.  Every CTA also sends every CTA (itself included) an 8-byte
// token per step, so a CTA waits for (M + CS) * 8 bytes: the tokens make
// each step depend on every CTA having finished the previous one, also for
// CTAs that own no rows (small M).  Step s uses buffer s & 1 (phase s >> 1
// of its mbarrier); a CTA sends step s + 2 only after it has received all of
// step s + 1, and every CTA sends step s + 1 after its block barrier of step
// s, so no buffer is overwritten while it is read and no CTA's mbarrier gets
// two phases ahead of one of its threads.  Each warp forms the norm itself
// from the received vector, so one iteration is one matvec, one mbarrier
// wait, the division and one block barrier.  Every wait is bounded (error
// flag g_pca_timeout).
constexpr int kPcaWarps = kPcaThreads / 32;
constexpr int kPcaMaxCluster = 16;  // token slots; the register kernel runs in clusters of 8

__device__ int g_pca_timeout;  // set when an exchange wait gave up (checked by the host)

template <int RPW, int CPL>
__global__ void __launch_bounds__(kPcaThreads, 1) pca_cluster_reg(const double* __restrict__ XXt, int M,
                                                                   int num_iter, double* __restrict__ comps,
                                                                   double* __restrict__ sigma) {
    constexpr int kMaxM = 32 * CPL;
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int CS = (int)cluster.num_blocks();
    int* err = &g_pca_timeout;
    __shared__ double ybuf[2][kMaxM];  // matvec results, written by every CTA
    __shared__ double vs[kMaxM];       // the normalised vector
    __shared__ double vinit[kMaxM];
    __shared__ double red[32];
    __shared__ __align__(8) uint64_t ybar[2];  // bytes of ybuf[b] received in the current step
    __shared__ __align__(8) uint64_t tok[2][kPcaMaxCluster];  // one token per sending CTA and step
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    const int row0 = (rank * kPcaWarps + w) * RPW;
    const bool has_rows = row0 < M;
    const uint32_t step_bytes = (uint32_t)(M + CS) * 8u;

    double A[RPW][CPL];
#pragma unroll
    for (int r = 0; r < RPW; r++)
#pragma unroll
        for (int j = 0; j < CPL; j++) {
            const int m = row0 + r, n = l + 32 * j;
            A[r][j] = (m < M && n < M) ? XXt[(size_t)m + (size_t)M * n] : 0.0;
        }
    if (threadIdx.x == 0) {
        tc::mbar_init(&ybar[0], 1);
        tc::mbar_init(&ybar[1], 1);
        tc::fence_mbar_init();
    }
    // start vector sin(i+1), normalised (pca.cpp:546-549, 457-466)
    for (int n = threadIdx.x; n < M; n += blockDim.x) vinit[n] = sin((double)(n + 1));
    __syncthreads();
    {
        double part = 0.0;
        for (int n = threadIdx.x; n < M; n += blockDim.x) part += vinit[n] * vinit[n];
        const double nrm = sqrt(block_sum(part, red));
        __syncthreads();
        if (nrm != 0.0)
            for (int n = threadIdx.x; n < M; n += blockDim.x) vinit[n] = vinit[n] / nrm;
    }
    if (threadIdx.x == 0) {
        tc::mbar_expect_tx(&ybar[0], step_bytes);  // steps 0 and 1
        tc::mbar_expect_tx(&ybar[1], step_bytes);
    }
    // every CTA's barriers are initialised and armed before any store reaches them
    cluster.sync();
    // lane l < CS sends to CTA l: the cluster addresses of its buffers and barriers
    const uint32_t rbuf = l < CS ? tc::mapa_shared(tc::smem_u32(&ybuf[0][0]), (uint32_t)l) : 0u;
    const uint32_t rbar = l < CS ? tc::mapa_shared(tc::smem_u32(&ybar[0]), (uint32_t)l) : 0u;
    const uint32_t rtok = l < CS ? tc::mapa_shared(tc::smem_u32(&tok[0][0]), (uint32_t)l) : 0u;

    // y = A v for this warp's rows, stored into every CTA's ybuf[step & 1];
    // then the wait for the whole vector of the step
    auto matvec = [&](const double* v, int64_t step) -> bool {
        const int b = (int)(step & 1);
        if (w == 0 && l < CS)
            tc::st_async_b64(rtok + (uint32_t)((b * kPcaMaxCluster + rank) * 8), 0ull, rbar + (uint32_t)(b * 8));
        if (has_rows) {
            double s[RPW];
#pragma unroll
            for (int r = 0; r < RPW; r++) s[r] = 0.0;
#pragma unroll
            for (int j = 0; j < CPL; j++) {
                const int n = l + 32 * j;
                if (n < M) {
                    const double vn = v[n];
#pragma unroll
                    for (int r = 0; r < RPW; r++) s[r] += A[r][j] * vn;
                }
            }
#pragma unroll
            for (int r = 0; r < RPW; r++) {
                for (int o = 16; o > 0; o >>= 1) s[r] += __shfl_xor_sync(0xffffffffu, s[r], o);
                const int m = row0 + r;
                if (m < M && l < CS)
                    tc::st_async_b64(rbuf + (uint32_t)((b * kMaxM + m) * 8), (uint64_t)__double_as_longlong(s[r]),
                                     rbar + (uint32_t)(b * 8));
            }
        }
        const bool ok = tc::mbar_wait_cluster(&ybar[b], (uint32_t)((step >> 1) & 1), err);
        // re-arm for step + 2: its stores arrive only after this CTA has sent step + 1
        if (ok && threadIdx.x == 0) tc::mbar_expect_tx(&ybar[b], step_bytes);
        return ok;
    };

    int64_t step = 0;  // matvec count (same sequence in every CTA)
    bool ok = true;
    for (int k = 0; k < M && ok; k++) {
        const double* v = vinit;
        double sig = 0.0;
        for (int it = 0; it < num_iter; it++) {
            const bool got = matvec(v, step);
            const double* y = ybuf[step & 1];
            if (got) {
                sig = sqrt(warp_ordered_sum(M, [&](int n) { return y[n] * y[n]; }));
                for (int n = threadIdx.x; n < M; n += blockDim.x) vs[n] = sig != 0.0 ? y[n] / sig : y[n];
            }
            ok = __syncthreads_and(got) != 0;
            if (!ok) break;
            v = vs;
            step++;
        }
        if (!ok) break;
        if (rank == 0) {
            for (int n = threadIdx.x; n < M; n += blockDim.x) comps[(size_t)n + (size_t)M * k] = v[n];
            if (threadIdx.x == 0) sigma[k] = sig;
        }
        // deflation: X <- X - v u' - u v' + (v'u) v v',  u = X v
        const bool got = matvec(v, step);
        const double* u = ybuf[step & 1];
        step++;
        if (got && has_rows) {
            const double alpha = warp_ordered_sum(M, [&](int n) { return v[n] * u[n]; });
#pragma unroll
            for (int r = 0; r < RPW; r++) {
                const int m = row0 + r;
                if (m >= M) continue;
                const double vm = v[m], um = u[m];
#pragma unroll
                for (int j = 0; j < CPL; j++) {
                    const int n = l + 32 * j;
                    if (n < M) {
                        const double sdef = __dadd_rn(__dmul_rn(vm, u[n]), __dmul_rn(um, v[n]));
                        const double x = __dsub_rn(A[r][j], sdef);
                        A[r][j] = __dadd_rn(x, __dmul_rn(alpha, __dmul_rn(vm, v[n])));
                    }
                }
            }
        }
        // vs and this buffer are read above; the next component rewrites vs
        // after its first wait and the buffer two steps later
        ok = __syncthreads_and(got) != 0;
    }
    // no CTA leaves while a peer may still store into its shared memory
    cluster.sync();
}

// W = (C D) C^T, D = diag(1/sqrt(sigma)) (0 where sigma == 0), in the
// reference's order: tmp(m,l) = C(m,l) d_l (mult_AB with a diagonal,
// pca.cpp:220-243), W(m,n) = sum_l tmp(m,l) C(n,l) (mult_ABtrans, :319-342).
__global__ void w_assemble(const double* __restrict__ C, const double* __restrict__ sigma, int M,
                           double* __restrict__ W) {
    extern __shared__ double dsh[];
    for (int l = threadIdx.x; l < M; l += blockDim.x) {
        const double s = sigma[l];
        dsh[l] = (s != 0.0) ? 1.0 / sqrt(s) : 0.0;
    }
    __syncthreads();
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int n = blockIdx.y;
    if (m >= M) return;
    double acc = 0.0;
    for (int l = 0; l < M; l++) {
        const double tmp = __dmul_rn(C[(size_t)m + (size_t)M * l], dsh[l]);
        acc = __dadd_rn(acc, __dmul_rn(tmp, C[(size_t)n + (size_t)M * l]));
    }
    W[(size_t)m + (size_t)M * n] = acc;
}

// ------------------------------------------------------------ apply

// Wt[m1][m2] = (float) W[m1*M + m2]  (the element the reference multiplies
// x[m2] with when it accumulates out[m1], p_whiten.cpp:174-183)
__global__ void w_to_float(const double* __restrict__ W, int64_t MM, float* __restrict__ Wt) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MM) Wt[i] = (float)W[i];
}

// quantize(x, 1e-4) = floor(x/1e-4 + 0.5) * 1e-4 in double (p_whiten.cpp:31-41).
// For a float x, x * 1e4 is exact in double (at most 34 significant bits)
// and the quotient x / 0.0001 lies within 0.43 ulp of it (the double 0.0001
// is 1e-4 (1 + 4.8e-17)), so the two are the same double; the division is
// kept as a guard for values within 1e-6 of a rounding boundary.
__device__ __forceinline__ float quantize_1e4(float x) {
    const double xd = (double)x;
    double t = __dadd_rn(__dmul_rn(xd, 10000.0), 0.5);
    double f = floor(t);
    if (t - f < 1e-6 || f + 1.0 - t < 1e-6) {
        t = __dadd_rn(__ddiv_rn(xd, 0.0001), 0.5);
        f = floor(t);
    }
    return (float)__dmul_rn(f, 0.0001);
}

constexpr int kBM = 64, kBN = 64, kBK = 16;

__global__ void __launch_bounds__(256) apply_gemm(const float* __restrict__ X, const float* __restrict__ Wt,
                                                  int64_t M, int64_t N, double qunit, int round_1e4,
                                                  void* __restrict__ out) {
    __shared__ __align__(16) float Xs[kBK][kBM + 4];
    __shared__ __align__(16) float Ws[kBK][kBN + 4];
    // column blocks of one time tile are adjacent in launch order, so the
    // time tile of X is read from DRAM once and from L2 by the others
    const int64_t ncb = (M + kBN - 1) / kBN;
    const int64_t t0 = ((int64_t)blockIdx.x / ncb) * kBM;
    const int64_t n0 = ((int64_t)blockIdx.x % ncb) * kBN;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0.f;
    for (int64_t k0 = 0; k0 < M; k0 += kBK) {
        for (int e = threadIdx.x; e < kBM * kBK; e += blockDim.x) {
            const int r = e / kBK, kk = e % kBK;
            const int64_t t = t0 + r, k = k0 + kk;
            Xs[kk][r] = (t < N && k < M) ? X[t * M + k] : 0.f;
            const int64_t n = n0 + r;
            Ws[kk][r] = (n < M && k < M) ? Wt[n * M + k] : 0.f;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; kk++) {
            const float4 a = *reinterpret_cast<const float4*>(&Xs[kk][ty * 4]);
            const float4 b = *reinterpret_cast<const float4*>(&Ws[kk][tx * 4]);
            const float av[4] = {a.x, a.y, a.z, a.w};
            const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int64_t t = t0 + ty * 4 + i;
        if (t >= N) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int64_t n = n0 + tx * 4 + j;
            if (n >= M) continue;
            const float y = round_1e4 ? quantize_1e4(acc[i][j]) : acc[i][j];
            if (qunit > 0) {
                // scale_for_quantization (p_whiten.cpp:445-451): (int)(y/q + 0.5)
                // stored in a float, then written as int16 by the .mda writer.
                const int32_t iv = x86_double_to_int32(__dadd_rn(__ddiv_rn((double)y, qunit), 0.5));
                static_cast<int16_t*>(out)[t * M + n] = x86_float_to_int16((float)iv);
            } else {
                static_cast<float*>(out)[t * M + n] = y;
            }
        }
    }
}

// out[t][j] = X[t][ch[j]] for a channel subset (0-based indices, checked by
// the caller): ms3.compute_whitening_matrix's extract_channels_from_chunk
// (p_whiten.cpp:421-433) applied to a whole device array.
__global__ void gather_channels(const float* __restrict__ X, int64_t M, int64_t N, const int32_t* __restrict__ ch,
                                int64_t M2, float* __restrict__ out) {
    const int64_t total = N * M2;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = i / M2, j = i - t * M2;
        if (MS3_IN_BOUNDS(ch[j], M, 201)) out[i] = X[t * M + ch[j]];
    }
}

// out[t][ch[j]] = Y[t][j]: a whitened channel block back into its columns
// (element size 4 for float32 output, 2 for int16).
template <class T>
__global__ void scatter_channels(const T* __restrict__ Y, int64_t M2, int64_t N, const int32_t* __restrict__ ch,
                                 int64_t M, T* __restrict__ out) {
    const int64_t total = N * M2;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = i / M2, j = i - t * M2;
        if (MS3_IN_BOUNDS(ch[j], M, 202)) out[t * M + ch[j]] = Y[i];
    }
}

int num_sms() {
    int dev = 0, n = 0;
    MS3_CUDA(cudaGetDevice(&dev));
    MS3_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

}  // namespace

// MS3GPU_COV_KERNEL=fma keeps the FP32-FMA kernel for every shape; =tc uses
// the tensor-core kernel whenever M % 4 == 0 (testing).  By default the
// tensor cores take M >= 128 with M % 4 == 0.
static int cov_kernel_choice() {
    static const int v = [] {
        const char* s = std::getenv("MS3GPU_COV_KERNEL");
        if (s && std::string(s) == "fma") return 1;
        if (s && std::string(s) == "tc") return 2;
        return 0;
    }();
    return v;
}

CovPlan cov_plan(const float* X, int64_t M) {
    CovPlan p;
    p.M = M;
    p.nb = (int)ceil_div(M, kCT);
    p.npairs = p.nb * (p.nb + 1) / 2;
    p.vec = (M % 4 == 0) && ((reinterpret_cast<uintptr_t>(X) & 15) == 0);
    const int choice = cov_kernel_choice();
    p.tc = M > 0 && M % 4 == 0 && choice != 1 && (choice == 2 || M >= 128);
    return p;
}

int64_t cov_tslice(const CovPlan& p, int64_t rows) {
    if (p.tc) return cov_i8_run_length(p.M, rows);
    if (rows <= 0) return kTT;
    const int64_t target = std::max<int64_t>(1, (int64_t)(p.vec ? 8 : 4) * num_sms() / p.npairs);
    const int64_t S = std::min<int64_t>(target, ceil_div(rows, kTT));
    return ceil_div(ceil_div(rows, S), kTT) * kTT;
}

int64_t cov_slices(const CovPlan& p, int64_t rows) {
    if (rows <= 0) return 0;
    return ceil_div(rows, cov_tslice(p, rows));
}

size_t cov_partials_bytes(const CovPlan& p, int64_t slices) {
    if (p.tc) return cov_i8_partials_bytes(p.M, slices);
    return (size_t)slices * p.npairs * kCT * kCT * sizeof(double);
}

void cov_partials(const float* X, int64_t M, int64_t r0, int64_t r1, const CovPlan& p, double* partials,
                  int64_t S, cudaStream_t stream) {
    const int64_t rows = r1 - r0;
    if (rows <= 0 || S <= 0) return;
    if (p.tc) {  // runs of the plan's length: the slicing the streamed forms use too
        const int64_t R = cov_tslice(p, rows);
        if (ceil_div(rows, R) != S) throw_invalid("covariance: slice count does not match the plan");
        cov_partials_sliced(X, M, r0, r1, p, partials, R, stream);
        return;
    }
    cov_partials_sliced(X, M, r0, r1, p, partials, ceil_div(ceil_div(rows, S), kTT) * kTT, stream);
}

void cov_partials_sliced(const float* X, int64_t M, int64_t r0, int64_t r1, const CovPlan& p, double* partials,
                         int64_t tslice, cudaStream_t stream) {
    const int64_t rows = r1 - r0;
    if (rows <= 0) return;
    if (tslice <= 0 || tslice % kTT != 0) throw_invalid("covariance slice length must be a multiple of 32");
    if (p.tc) {
        if ((reinterpret_cast<uintptr_t>(X + r0 * M) & 15) == 0) {
            cov_i8_partials(X, M, r0, r1, tslice, partials, stream);
        } else {  // the tensor map needs 16-byte aligned rows: work on an aligned copy
            DevBuf copy(sizeof(float) * (size_t)(rows * M), stream);
            MS3_CUDA(cudaMemcpyAsync(copy.get(), X + r0 * M, sizeof(float) * (size_t)(rows * M),
                                     cudaMemcpyDeviceToDevice, stream));
            cov_i8_partials(copy.as<float>(), M, 0, rows, tslice, partials, stream);
        }
        return;
    }
    const int64_t S = ceil_div(rows, tslice);
    if (p.vec)
        cov_partial8<<<dim3(p.npairs, (unsigned)S), 64, 0, stream>>>(X, M, r0, r1, p.nb, tslice, partials);
    else
        cov_partial<<<dim3(p.npairs, (unsigned)S), 256, 0, stream>>>(X, M, r0, r1, p.nb, tslice, partials);
    MS3_LAUNCH_CHECK();
}

void cov_finish(const double* partials, int64_t S, const CovPlan& p, int64_t M, int64_t N, double* XXt,
                cudaStream_t stream) {
    if (p.tc) {
        cov_i8_finish(partials, S, M, N, XXt, stream);
        return;
    }
    if (S == 0) {
        MS3_CUDA(cudaMemsetAsync(XXt, 0, sizeof(double) * (size_t)(M * M), stream));
        return;
    }
    const int64_t total = (int64_t)p.npairs * kCT * kCT;
    cov_reduce<<<(unsigned)ceil_div(total, 256), 256, 0, stream>>>(partials, (int)S, p.npairs, p.nb, M, N, XXt);
    MS3_LAUNCH_CHECK();
}

void covariance_sum_device(const float* X, int64_t M, int64_t N, double* XXt_sum, cudaStream_t stream) {
    if (M <= 0) return;
    const CovPlan p = cov_plan(X, M);
    const int64_t S = cov_slices(p, N);
    DevBuf partials(cov_partials_bytes(p, S), stream);
    cov_partials(X, M, 0, N, p, partials.as<double>(), S, stream);
    cov_finish(partials.as<double>(), S, p, M, /*N=*/1, XXt_sum, stream);  // N <= 1: no division
}

void covariance_device(const float* X, int64_t M, int64_t N, double* XXt, cudaStream_t stream) {
    if (M <= 0) return;
    const CovPlan p = cov_plan(X, M);
    const int64_t S = cov_slices(p, N);
    DevBuf partials(cov_partials_bytes(p, S), stream);
    cov_partials(X, M, 0, N, p, partials.as<double>(), S, stream);
    cov_finish(partials.as<double>(), S, p, M, N, XXt, stream);
}

// ------------------------------------------------ covariance without allocation
//
// Scratch for the partial covariance tiles of ms3gpu_whiten_covariance_noalloc:
// a fixed array in the library's device image, present on every GPU that
// loads the library until the process exits.  Host code cannot use the
// symbol's name as a device address; its address is looked up once per
// device with cudaGetSymbolAddress and passed to the kernels.
constexpr size_t kNoAllocScratchBytes = size_t(16) << 20;  // 16 MiB
static __device__ __align__(256) unsigned char g_noalloc_cov_scratch[kNoAllocScratchBytes];

namespace {
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[64] = {};

// Device address of the scratch array on the current device (looked up on
// the first call for that device).
double* noalloc_scratch() {
    int dev = 0;
    MS3_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw_unsupported("device index above 63");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        MS3_CUDA(cudaGetSymbolAddress(&p, g_noalloc_cov_scratch));
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    return g_noalloc_ptr[dev];
}
}  // namespace

int64_t covariance_noalloc_max_channels() {
    // the scratch must hold one time slice of 64 x 64 FP64 tiles of the upper triangle
    const size_t tile = (size_t)kCT * kCT * sizeof(double);
    int64_t nb = 1;
    while ((size_t)(nb + 1) * (nb + 2) / 2 * tile <= kNoAllocScratchBytes) nb++;
    return nb * kCT;
}

void covariance_device_noalloc(const float* X, int64_t M, int64_t N, double* XXt, cudaStream_t stream) {
    if (M <= 0) return;
    if (M > covariance_noalloc_max_channels())
        throw_invalid("ms3gpu_whiten_covariance_noalloc handles at most " +
                      std::to_string(covariance_noalloc_max_channels()) + " channels (16 MiB scratch); got " +
                      std::to_string(M));
    double* scratch = noalloc_scratch();
    const int nb = (int)ceil_div(M, kCT);
    const int npairs = nb * (nb + 1) / 2;
    if (N == 0) {
        MS3_CUDA(cudaMemsetAsync(XXt, 0, sizeof(double) * (size_t)(M * M), stream));
        return;
    }
    const int64_t s_max = (int64_t)(kNoAllocScratchBytes / ((size_t)npairs * kCT * kCT * sizeof(double)));
    const int64_t target = std::max<int64_t>(1, (int64_t)4 * num_sms() / npairs);
    int64_t S = std::min<int64_t>(std::min(target, s_max), ceil_div(N, kTT));
    const int64_t tslice = ceil_div(ceil_div(N, S), kTT) * kTT;
    S = ceil_div(N, tslice);
    // Every partial tile the reduction reads is written by cov_partial in this
    // call, so nothing left in the array by an earlier call is ever used.
    cov_partial<<<dim3(npairs, (unsigned)S), 256, 0, stream>>>(X, M, 0, N, nb, tslice, scratch);
    MS3_LAUNCH_CHECK();
    const int64_t total = (int64_t)npairs * kCT * kCT;
    cov_reduce<<<(unsigned)ceil_div(total, 256), 256, 0, stream>>>(scratch, (int)S, npairs, nb, M, N, XXt);
    MS3_LAUNCH_CHECK();
}

// pca_cluster launch: rows in shared memory across 8 or 16 CTAs, else in global memory.
void pca_launch_smem(const double* XXt, int64_t M, double* comps, double* sigma, cudaStream_t stream);

void whitening_matrix_device(const double* XXt, int64_t M, double* W, double* comps, double* sigma,
                             cudaStream_t stream) {
    if (M <= 0) return;
    if (M > 65535) throw_unsupported("whitening matrix for more than 65535 channels");
    DevBuf cbuf, sbuf;
    if (!comps) { cbuf.alloc(sizeof(double) * (size_t)(M * M), stream); comps = cbuf.as<double>(); }
    if (!sigma) { sbuf.alloc(sizeof(double) * (size_t)M, stream); sigma = sbuf.as<double>(); }

    // registers hold the working matrix up to 384 channels (MS3GPU_PCA_KERNEL=smem
    // selects the shared-memory kernel, which gives the same values)
    const char* pk = std::getenv("MS3GPU_PCA_KERNEL");
    const bool force_smem = pk && std::string(pk) == "smem";
    const char* force_global0 = std::getenv("MS3GPU_PCA_ROWS_GLOBAL");
    if (!force_smem && !(force_global0 && force_global0[0] == '1') && M <= 384) {
        auto kern = M <= 128 ? pca_cluster_reg<1, 4> : (M <= 256 ? pca_cluster_reg<2, 8> : pca_cluster_reg<3, 12>);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(8, 1, 1);
        cfg.blockDim = dim3(kPcaThreads, 1, 1);
        cfg.dynamicSmemBytes = 0;
        cfg.stream = stream;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = 8;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        MS3_CUDA(cudaLaunchKernelEx(&cfg, kern, XXt, (int)M, 10, comps, sigma));
        MS3_LAUNCH_CHECK();
    } else {
        pca_launch_smem(XXt, M, comps, sigma, stream);
    }
    const size_t wsm = sizeof(double) * (size_t)M;
    if (wsm > 48 * 1024)
        MS3_CUDA(cudaFuncSetAttribute(w_assemble, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wsm));
    w_assemble<<<dim3((unsigned)ceil_div(M, 128), (unsigned)M), 128, wsm, stream>>>(comps, sigma, (int)M, W);
    MS3_LAUNCH_CHECK();
}

void whitening_check_timeout(cudaStream_t stream) {
    int h = 0;
    MS3_CUDA(cudaMemcpyFromSymbolAsync(&h, g_pca_timeout, sizeof(int), 0, cudaMemcpyDeviceToHost, stream));
    MS3_CUDA(cudaStreamSynchronize(stream));
    if (h) {
        const int zero = 0;
        MS3_CUDA(cudaMemcpyToSymbolAsync(g_pca_timeout, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, stream));
        MS3_CUDA(cudaStreamSynchronize(stream));
        throw Error(MS3GPU_ERR_CUDA, "power iteration: exchange wait timed out");
    }
}

void pca_launch_smem(const double* XXt, int64_t M, double* comps, double* sigma, cudaStream_t stream) {
    int dev = 0, max_optin = 0;
    MS3_CUDA(cudaGetDevice(&dev));
    MS3_CUDA(cudaDeviceGetAttribute(&max_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t vec_bytes = sizeof(double) * (size_t)(3 * M + 32);
    int CS = 0, R = 0, in_smem = 0;
    // MS3GPU_PCA_ROWS_GLOBAL=1 keeps the working matrix in global memory
    // even when it fits shared memory (exercises that path in tests).
    const char* force_global = std::getenv("MS3GPU_PCA_ROWS_GLOBAL");
    const bool allow_smem = !(force_global && force_global[0] == '1');
    for (int cs : {8, 16}) {
        if (!allow_smem) break;
        const int r = (int)ceil_div(M, cs);
        const size_t need = vec_bytes + sizeof(double) * (size_t)r * (size_t)(M + 1);
        if (need <= (size_t)max_optin) { CS = cs; R = r; in_smem = 1; break; }
    }
    DevBuf xg;
    if (!in_smem) {
        CS = 16;
        R = (int)ceil_div(M, CS);
        xg.alloc(sizeof(double) * (size_t)CS * R * (size_t)(M + 1), stream);
    }
    const size_t smem = vec_bytes + (in_smem ? sizeof(double) * (size_t)R * (size_t)(M + 1) : 0);
    MS3_CUDA(cudaFuncSetAttribute(pca_cluster, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (CS > 8) MS3_CUDA(cudaFuncSetAttribute(pca_cluster, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));

    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(CS, 1, 1);
    cfg.blockDim = dim3(kPcaThreads, 1, 1);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = CS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    MS3_CUDA(cudaLaunchKernelEx(&cfg, pca_cluster, XXt, (int)M, R, 10, in_smem, xg.as<double>(), comps, sigma));
    MS3_LAUNCH_CHECK();
}

void gather_channels_device(const float* X, int64_t M, int64_t N, const int32_t* ch, int64_t M2, float* out,
                            cudaStream_t stream) {
    if (N <= 0 || M2 <= 0) return;
    const int64_t blocks = std::min<int64_t>(ceil_div(N * M2, 256), (int64_t)num_sms() * 32);
    gather_channels<<<(unsigned)blocks, 256, 0, stream>>>(X, M, N, ch, M2, out);
    MS3_LAUNCH_CHECK();
}

void scatter_channels_device(const void* Y, int64_t M2, int64_t N, const int32_t* ch, int64_t M, void* out,
                             size_t elem, cudaStream_t stream) {
    if (N <= 0 || M2 <= 0) return;
    const int64_t blocks = std::min<int64_t>(ceil_div(N * M2, 256), (int64_t)num_sms() * 32);
    if (elem == 2)
        scatter_channels<int16_t><<<(unsigned)blocks, 256, 0, stream>>>(static_cast<const int16_t*>(Y), M2, N, ch, M,
                                                                        static_cast<int16_t*>(out));
    else
        scatter_channels<float><<<(unsigned)blocks, 256, 0, stream>>>(static_cast<const float*>(Y), M2, N, ch, M,
                                                                      static_cast<float*>(out));
    MS3_LAUNCH_CHECK();
}

void apply_whitening_device(const float* X, int64_t M, int64_t N, const double* W, double quantization_unit,
                            bool mixed, void* out, cudaStream_t stream, int* err, bool round_1e4) {
    if (M <= 0 || N <= 0) return;
    // MS3GPU_APPLY_FFMA=1 selects the FP32 FMA kernel for the plain form
    const char* ffma = std::getenv("MS3GPU_APPLY_FFMA");
    const bool force_ffma = ffma && ffma[0] == '1';
    if (apply_tc_supported(X, M, N, out) && (mixed || !force_ffma)) {
        apply_whitening_tc(X, M, N, W, quantization_unit, /*drain=*/!mixed, out, stream, err, round_1e4);
        return;
    }
    DevBuf wt(sizeof(float) * (size_t)(M * M), stream);
    w_to_float<<<(unsigned)ceil_div(M * M, 256), 256, 0, stream>>>(W, M * M, wt.as<float>());
    MS3_LAUNCH_CHECK();
    const int64_t blocks = ceil_div(N, kBM) * ceil_div(M, kBN);
    if (blocks > 0x7fffffff) throw_unsupported("too many tiles for the apply kernel");
    apply_gemm<<<(unsigned)blocks, 256, 0, stream>>>(X, wt.as<float>(), M, N, quantization_unit, round_1e4 ? 1 : 0,
                                                     out);
    MS3_LAUNCH_CHECK();
}

int bounds_site_whiten(cudaStream_t s) {
#ifdef MS3GPU_BOUNDS_CHECK
    return take_bounds_site(s);
#else
    (void)s;
    return 0;
#endif
}

}  // namespace ms3gpu
