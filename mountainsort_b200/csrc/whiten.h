// Internal interface of the whitening stages (device pointers only).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ms3gpu {

// XXt (M x M doubles, column-major) = sum_t x_t x_t^T / (N-1 if N > 1).
void covariance_device(const float* X, int64_t M, int64_t N, double* XXt, cudaStream_t stream);
// The same sum over the N rows of X without the division (one shard's part
// of a recording whose rows are spread over several GPUs).
void covariance_sum_device(const float* X, int64_t M, int64_t N, double* XXt_sum, cudaStream_t stream);

// The covariance in pieces, for callers that stream the rows in: partial
// tiles of rows [r0, r1) go to `S` slices of a partials buffer; cov_finish
// sums all slices written so far (fixed order) and divides by N-1.
// tc: the tensor-core kernel (exact int8 digit products, cov_i8.cu), whose
// slices are runs of cov_tslice timepoints with one partial tile per 128 x
// 128 channel block pair; otherwise the FP32-FMA kernel (64 x 64 tiles).
struct CovPlan {
    int nb = 0, npairs = 0;
    bool vec = false;
    bool tc = false;
    int64_t M = 0;
};
CovPlan cov_plan(const float* X, int64_t M);
int64_t cov_slices(const CovPlan& p, int64_t rows);
size_t cov_partials_bytes(const CovPlan& p, int64_t slices);
void cov_partials(const float* X, int64_t M, int64_t r0, int64_t r1, const CovPlan& p, double* partials,
                  int64_t S, cudaStream_t stream);
// The slice length covariance_device uses for `rows` rows (a multiple of 32),
// and cov_partials with that length given: ceil((r1 - r0) / tslice) slices.
// A recording streamed in slabs of whole slices, each slab's slices written
// after the previous slab's, sums to the same XXt bit for bit.
int64_t cov_tslice(const CovPlan& p, int64_t rows);
void cov_partials_sliced(const float* X, int64_t M, int64_t r0, int64_t r1, const CovPlan& p, double* partials,
                         int64_t tslice, cudaStream_t stream);
void cov_finish(const double* partials, int64_t S, const CovPlan& p, int64_t M, int64_t N, double* XXt,
                cudaStream_t stream);

// Tensor-core covariance pieces (cov_i8.cu): runs of R timepoints (a
// multiple of 32, at most 32768) of rows [r0, r1) of X, one FP64 partial tile
// per (run, block pair); finish sums `runs` runs in order.  X + r0 * M must
// be 16-byte aligned with M % 4 == 0.
int cov_i8_pairs(int64_t M);
int64_t cov_i8_run_length(int64_t M, int64_t rows);
size_t cov_i8_partials_bytes(int64_t M, int64_t runs);
void cov_i8_partials(const float* X, int64_t M, int64_t r0, int64_t r1, int64_t R, double* partials,
                     cudaStream_t stream);
void cov_i8_finish(const double* partials, int64_t runs, int64_t M, int64_t N, double* XXt, cudaStream_t stream);
// Raises MS3GPU_ERR_CUDA (after a synchronize) when a tensor-core covariance
// pipeline wait or a power-iteration exchange wait gave up, and clears the
// flag.
void covariance_check_timeout(cudaStream_t stream);

// The power-iteration part of covariance_check_timeout.
void whitening_check_timeout(cudaStream_t stream);

// The same covariance with its partial sums in a fixed 16 MiB device array
// instead of allocated scratch (X and XXt must be device memory).
void covariance_device_noalloc(const float* X, int64_t M, int64_t N, double* XXt, cudaStream_t stream);
int64_t covariance_noalloc_max_channels();

// out (N x M2 rows) = the channels ch[0..M2) (0-based, in range) of X (N x M rows).
void gather_channels_device(const float* X, int64_t M, int64_t N, const int32_t* ch, int64_t M2, float* out,
                            cudaStream_t stream);

// out (N x M rows) columns ch[j] = Y (N x M2 rows) column j; elem 4 (float32) or 2 (int16).
void scatter_channels_device(const void* Y, int64_t M2, int64_t N, const int32_t* ch, int64_t M, void* out,
                             size_t elem, cudaStream_t stream);

// Power-iteration whitening matrix; comps / sigma may be null.
void whitening_matrix_device(const double* XXt, int64_t M, double* W, double* comps, double* sigma,
                             cudaStream_t stream);

// out = quantize(W^T x) per timepoint; out float32, or int16 when
// quantization_unit > 0.  mixed: tensor-core 3-term TF32 (when the shapes
// allow), else FP32 FMA.
// err: optional device flag raised by a timed-out tensor-core pipeline; when
// null the call checks it itself (synchronising the stream).
// round_1e4 = false skips the 1e-4 rounding (ms3.whiten_clips, which does
// not round, p_whiten.cpp:300-345).
void apply_whitening_device(const float* X, int64_t M, int64_t N, const double* W,
                            double quantization_unit, bool mixed, void* out, cudaStream_t stream,
                            int* err = nullptr, bool round_1e4 = true);

// Tensor-core (tcgen05, 3-term TF32) apply; apply_tc_supported tells whether
// the shapes and alignment allow it.
bool apply_tc_supported(const float* X, int64_t M, int64_t N, const void* out);
// drain: per-K-block draining of the large products into round-to-nearest
// FP32 sums (plain form); otherwise one FP32 TMEM accumulator (mixed form).
void apply_whitening_tc(const float* X, int64_t M, int64_t N, const double* W, double quantization_unit,
                        bool drain, void* out, cudaStream_t stream, int* err = nullptr, bool round_1e4 = true);

}  // namespace ms3gpu
