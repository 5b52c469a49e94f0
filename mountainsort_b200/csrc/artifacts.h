// Internal interface of ms3.mask_out_artifacts (device pointers only).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ms3gpu {

// X, out: device (N, M) float32 rows.  interval_size > 0.  Returns the number
// of timepoints kept (synchronizes the stream).
int64_t mask_out_artifacts_device(const float* X, int64_t M, int64_t N, double threshold, int64_t interval_size,
                                  float* out, cudaStream_t stream);

// The three steps on their own, for a recording that arrives in blocks of
// whole intervals: norms[i * M + m] of the nint intervals of X (interval size
// I); the flags exceed[0, nint + 2) from all norms; the masked copy of `rows`
// timepoints of X that start at timepoint t0 (a multiple of I) of the
// recording; the timepoints kept (synchronizes the stream).
void artifact_norms_device(const float* X, int64_t M, int64_t I, int64_t nint, double* norms, cudaStream_t stream);
void artifact_flags_device(const double* norms, int64_t M, int64_t nint, double threshold, int* exceed,
                           cudaStream_t stream);
void artifact_write_device(const float* X, int64_t M, int64_t rows, int64_t t0, int64_t I, int64_t nint,
                           const int* exceed, float* out, cudaStream_t stream);
int64_t artifact_kept(const int* exceed, int64_t nint, int64_t I, cudaStream_t stream);

}  // namespace ms3gpu
