// Internal interface of ms3.mask_out_artifacts (device pointers only).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ms3gpu {

// X, out: device (N, M) float32 rows.  interval_size > 0.  Returns the number
// of timepoints kept (synchronizes the stream).
int64_t mask_out_artifacts_device(const float* X, int64_t M, int64_t N, double threshold, int64_t interval_size,
                                  float* out, cudaStream_t stream);

}  // namespace ms3gpu
