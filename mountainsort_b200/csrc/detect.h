// Internal interface of the event detection (device input, host output).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace ms3gpu {

// get_time_chunk_infos' chunk length (p_mountainsort3.cpp:507-517).
int64_t detect_chunk_size(int64_t M, int64_t N, int64_t num_simultaneous);

// X: device (N, M) float32 rows.  counts[m] = events of channel m; times =
// the channels' event times one channel after the other, each sorted.
void detect_events_device(const float* X, int64_t M, int64_t N, double detect_threshold, double detect_interval,
                          int sign, int64_t chunk, int64_t pad, std::vector<int64_t>& counts,
                          std::vector<int64_t>& times, cudaStream_t stream);

}  // namespace ms3gpu
