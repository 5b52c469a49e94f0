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
// and writes output rows [c*chunk, (c+1)*chunk) / sub.  The output rows of
// these windows are zeroed first when subsampling leaves gaps between them.
// raw_row0 / out_row0: the first row that `raw` / `out` hold (a slab of the
// recording); they must hold every row the windows read / write.
void bandpass_device(const void* raw, int64_t M, int64_t N, void* out, const BandpassParams& bp,
                     cudaStream_t stream, int64_t c_begin = 0, int64_t c_end = -1, bool in_i16 = false,
                     int64_t raw_row0 = 0, int64_t out_row0 = 0);

// Output rows [o0, o1) written by windows [c_begin, c_end): o0 = c_begin *
// chunk / sub, o1 = min(N / sub, c_end * chunk / sub).
void bandpass_output_rows(int64_t N, int64_t chunk, int sub, int64_t c_begin, int64_t c_end, int64_t& o0,
                          int64_t& o1);

// Raises (and clears) the error a bandpass pipeline wait recorded when it gave
// up; synchronizes `stream`.  Call once the bandpass work is ordered before
// `stream`.
void bandpass_check_timeout(cudaStream_t stream);

}  // namespace ms3gpu
