// ms3.mask_out_artifacts on the GPU (packages/ms3/p_mask_out_artifacts.cpp:24-104),
// the next step on the filtered or whitened timeseries in some pipelines.
//
//   norms(m, i) = sqrt(sum_{a < I} x(m, i*I + a)^2)      i < N / I (floor), double,
//                 summed in timepoint order as the reference's loop does
//   per channel: mean and sample stdev of its norms (MLCompute::mean / stdev,
//                common/mlcompute.cpp:67-85, sums in interval order)
//   an interval whose norm exceeds mean + threshold * stdev on any channel
//   masks itself and its two neighbours (the reference's write to use_it[-1]
//   for interval 0 lands outside the array and is dropped here)
//   out = x on the kept intervals, 0 on masked intervals and on the tail
//         beyond the last whole interval (never written by the reference).
//
// Three kernels: norms (one thread per channel and interval, coalesced over
// channels), per-channel statistics + interval flags, and a masked copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "artifacts.h"
#include "common.cuh"

namespace ms3gpu {

namespace {

// norms[i * M + m]; threads over channels, blocks over intervals (the grid's
// y extent is capped at 65535, so each block row strides over the intervals)
__global__ void artifact_norms(const float* __restrict__ X, int64_t M, int64_t I, int64_t nint,
                               double* __restrict__ norms) {
    for (int64_t i = blockIdx.y; i < nint; i += gridDim.y) {
        for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < M;
             m += (int64_t)gridDim.x * blockDim.x) {
            const float* p = X + i * I * M + m;
            double s = 0.0;
            for (int64_t a = 0; a < I; a++) {
                const double v = (double)p[a * M];
                s = __dadd_rn(s, __dmul_rn(v, v));
            }
            norms[i * M + m] = sqrt(s);
        }
    }
}

// One thread per channel: the reference's per-channel statistics, then the
// intervals it flags.  exceed[i] is set for a flagged interval i.
__global__ void artifact_flags(const double* __restrict__ norms, int64_t M, int64_t nint, double threshold,
                               int* __restrict__ exceed) {
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= M) return;
    double sum = 0.0, sumsqr = 0.0;
    for (int64_t i = 0; i < nint; i++) {
        const double v = norms[i * M + m];
        sum = __dadd_rn(sum, v);
        sumsqr = __dadd_rn(sumsqr, __dmul_rn(v, v));
    }
    const double mean0 = nint ? __ddiv_rn(sum, (double)nint) : 0.0;
    double sigma0 = 0.0;
    if (nint >= 2) {
        const double ct = (double)nint;
        sigma0 = sqrt(__ddiv_rn(__dsub_rn(sumsqr, __ddiv_rn(__dmul_rn(sum, sum), ct)), ct - 1.0));
    }
    const double limit = __dadd_rn(mean0, __dmul_rn(sigma0, threshold));
    for (int64_t i = 0; i < nint; i++)
        if (norms[i * M + m] > limit) exceed[i] = 1;
}

// out(m, t) = x(m, t) where interval t / I is kept, else 0; X and out hold
// the N timepoints from t0
__global__ void artifact_write(const float* __restrict__ X, int64_t M, int64_t N, int64_t I, int64_t nint,
                               const int* __restrict__ exceed, float* __restrict__ out, int64_t t0) {
    const int64_t total = M * N;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = t0 + k / M;
        const int64_t i = t / I;
        bool keep = i < nint;
        if (keep) keep = !exceed[i] && !exceed[i + 1] && !(i >= 1 && exceed[i - 1]);
        out[k] = keep ? X[k] : 0.f;
    }
}

int sm_count() {
    int dev = 0, n = 0;
    MS3_CUDA(cudaGetDevice(&dev));
    MS3_CUDA(cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev));
    return n;
}

}  // namespace

int64_t mask_out_artifacts_device(const float* X, int64_t M, int64_t N, double threshold, int64_t interval_size,
                                  float* out, cudaStream_t stream) {
    if (M <= 0 || N <= 0) return 0;
    const int64_t I = interval_size;
    const int64_t nint = N / I;
    DevBuf norms(sizeof(double) * (size_t)std::max<int64_t>(1, nint * M), stream);
    DevBuf exceed(sizeof(int) * (size_t)(nint + 2), stream);
    MS3_CUDA(cudaMemsetAsync(exceed.get(), 0, sizeof(int) * (size_t)(nint + 2), stream));
    if (nint > 0) {
        artifact_norms_device(X, M, I, nint, norms.as<double>(), stream);
        artifact_flags<<<(unsigned)ceil_div(M, 128), 128, 0, stream>>>(norms.as<double>(), M, nint, threshold,
                                                                      exceed.as<int>());
        MS3_LAUNCH_CHECK();
    }
    const int64_t blocks = std::min<int64_t>(ceil_div(M * N, 256), (int64_t)sm_count() * 32);
    artifact_write<<<(unsigned)blocks, 256, 0, stream>>>(X, M, N, I, nint, exceed.as<int>(), out, 0);
    MS3_LAUNCH_CHECK();
    return artifact_kept(exceed.as<int>(), nint, I, stream);
}

void artifact_norms_device(const float* X, int64_t M, int64_t I, int64_t nint, double* norms, cudaStream_t stream) {
    if (M <= 0 || nint <= 0) return;
    const int threads = 128;
    const unsigned gx = (unsigned)std::max<int64_t>(1, std::min<int64_t>(ceil_div(M, threads), 65535));
    const unsigned gy = (unsigned)std::min<int64_t>(nint, 65535);
    artifact_norms<<<dim3(gx, gy), threads, 0, stream>>>(X, M, I, nint, norms);
    MS3_LAUNCH_CHECK();
}

void artifact_flags_device(const double* norms, int64_t M, int64_t nint, double threshold, int* exceed,
                           cudaStream_t stream) {
    MS3_CUDA(cudaMemsetAsync(exceed, 0, sizeof(int) * (size_t)(nint + 2), stream));
    if (M <= 0 || nint <= 0) return;
    artifact_flags<<<(unsigned)ceil_div(M, 128), 128, 0, stream>>>(norms, M, nint, threshold, exceed);
    MS3_LAUNCH_CHECK();
}

void artifact_write_device(const float* X, int64_t M, int64_t rows, int64_t t0, int64_t I, int64_t nint,
                           const int* exceed, float* out, cudaStream_t stream) {
    if (M <= 0 || rows <= 0) return;
    const int64_t blocks = std::min<int64_t>(ceil_div(M * rows, 256), (int64_t)sm_count() * 32);
    artifact_write<<<(unsigned)blocks, 256, 0, stream>>>(X, M, rows, I, nint, exceed, out, t0);
    MS3_LAUNCH_CHECK();
}

int64_t artifact_kept(const int* exceed, int64_t nint, int64_t I, cudaStream_t stream) {
    // timepoints kept, for the reference's "Using x% of all timepoints" line
    std::vector<int> h((size_t)(nint + 2));
    MS3_CUDA(cudaMemcpyAsync(h.data(), exceed, sizeof(int) * (size_t)(nint + 2), cudaMemcpyDeviceToHost, stream));
    MS3_CUDA(cudaStreamSynchronize(stream));
    int64_t kept = 0;
    for (int64_t i = 0; i < nint; i++)
        if (!h[(size_t)i] && !h[(size_t)i + 1] && !(i >= 1 && h[(size_t)i - 1])) kept += I;
    return kept;
}

}  // namespace ms3gpu
