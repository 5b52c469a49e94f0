// Internal interface of the bandpass stage (device pointers only).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace ms3gpu {

struct BandpassParams {
    double samplerate = 0, freq_min = 0, freq_max = 0, freq_wid = 1000, quantization_unit = 0;
    int subsample_factor = 1;
    int num_threads = 1;
};

// The reference's chunk size (p_bandpass_filter.cpp:147-155).
int64_t bandpass_chunk_size(int64_t M, int64_t num_threads);

// raw: device (N, M) float32 rows (int16 when in_i16, converted to float on
// load); out: device M x (N/sub), float32 or int16 (freq_max == 0 copies raw).
// Filters the windows (chunks) [c_begin, c_end) of the recording (all by
// default); window c reads raw rows [c*chunk - 60000, (c+1)*chunk + 60000)
// and writes output rows [c*chunk, (c+1)*chunk) / sub.
void bandpass_device(const void* raw, int64_t M, int64_t N, void* out, const BandpassParams& bp,
                     cudaStream_t stream, int64_t c_begin = 0, int64_t c_end = -1, bool in_i16 = false);

// Raises (and clears) the error a bandpass pipeline wait recorded when it gave
// up; synchronizes `stream`.  Call once the bandpass work is ordered before
// `stream`.
void bandpass_check_timeout(cudaStream_t stream);

}  // namespace ms3gpu
