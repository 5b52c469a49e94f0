// Streaming forms of the bandpass and whitening processors: the recording
// is read and written through caller callbacks, one slab of rows at a time,
// so neither host nor device ever holds the whole recording.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "bandpass.h"
#include "ms3gpu.h"

namespace ms3gpu {

// Rows t of the output written by the same kernels on the same windows as
// bandpass_device over the whole recording: identical values.
void bandpass_stream(int64_t M, int64_t N, bool in_i16, const ms3gpu_stream_io& io, const BandpassParams& bp,
                     cudaStream_t s);

// Two passes over the input like the reference (covariance, then the apply);
// identical to the in-memory whitening whenever one covariance slice of the
// whole recording (about N / 56 rows at M = 384) fits in a slab.
void whiten_stream(int64_t M, int64_t N, const ms3gpu_stream_io& io, double quantization_unit, bool mixed,
                   cudaStream_t s);

// ms3.mask_out_artifacts with two passes over the input (interval norms,
// then the masked copy), slabs of whole intervals; identical values and
// timepoints kept to the in-memory call.  Returns the timepoints kept.
int64_t mask_out_artifacts_stream(int64_t M, int64_t N, double threshold, int64_t interval_size,
                                  const ms3gpu_stream_io& io, cudaStream_t s);

}  // namespace ms3gpu
