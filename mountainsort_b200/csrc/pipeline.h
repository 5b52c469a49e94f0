// Host-buffer entry points with host<->device copies overlapped with the kernels.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "bandpass.h"

namespace ms3gpu {

// raw_h: host (N, M) float32; filt_h: host float32 or null; pre_h: host
// float32 (q <= 0) or int16 (q > 0).  Requires subsample 1 and no bandpass
// quantization (the pipeline's settings).
void bandpass_whiten_streamed(const float* raw_h, int64_t M, int64_t N, float* filt_h, void* pre_h,
                              const BandpassParams& bp, double q, bool mixed, cudaStream_t s);

}  // namespace ms3gpu
