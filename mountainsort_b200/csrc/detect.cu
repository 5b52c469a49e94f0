// Event detection of mountainsortalg on the whitened timeseries, the first
// consumer of the filter + whiten output:
//   detect_events (packages/mountainsortalg/detect_events.cpp:69-135) as
//   NeighborhoodSorter::addTimeChunk applies it (neighborhoodsorter.cpp:74-100)
//   to the central channel of every neighborhood over the time chunks of
//   p_mountainsort3.cpp:190-215 / get_time_chunk_infos (:507-533).
//
// Per (channel, time chunk), with the chunk [t1 - pad, t1 + size + pad) read
// with zeros outside the recording (readChunk's zero fill):
//   1. the chunk's mean and sample stdev in double, summed in index order
//      (MLCompute::mean / stdev, common/mlcompute.cpp:67-85) -- one thread
//      per (channel, chunk), loads batched so that their latencies overlap;
//   2. the candidates -- samples whose signed (or absolute, for sign 0)
//      deviation from the mean exceeds threshold * stdev -- found in parallel
//      over time sub-ranges (a warp = 32 channels x one sub-range; a count
//      pass, then an in-order write at prefix-summed offsets);
//   3. the reference's greedy strongest-within-detect_interval rule over each
//      (channel, chunk)'s candidates in time order (one thread each: the rule
//      is sequential, but it only walks the candidates);
//   4. the kept times inside [t1, t1 + size), channel after channel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "common.cuh"
#include "detect.h"

namespace ms3gpu {

namespace {

constexpr int kSub = 16;  // time sub-ranges per chunk for the candidate passes

struct ChunkStats {
    double mean, threshold2;
};

__device__ __forceinline__ float sample(const float* X, int64_t M, int64_t N, int64_t t, int64_t m) {
    return (t >= 0 && t < N) ? X[t * M + m] : 0.f;
}

// kBatch consecutive samples of channel m from timepoint t, loaded together so
// that their latencies overlap (zeros outside [0, N) and beyond `left`).
constexpr int kBatch = 32;
__device__ __forceinline__ void load_batch(const float* X, int64_t M, int64_t N, int64_t t, int64_t m, int64_t left,
                                           float (&b)[kBatch]) {
    if (t >= 0 && t + kBatch <= N && left >= kBatch) {
        // interior: unconditional loads, all in flight together
        const float* p = X + t * M + m;
#pragma unroll
        for (int k = 0; k < kBatch; k++) b[k] = __ldg(p + (int64_t)k * M);
    } else {
#pragma unroll
        for (int k = 0; k < kBatch; k++) b[k] = (k < left) ? sample(X, M, N, t + k, m) : 0.f;
    }
}

__device__ __forceinline__ int64_t chunk_size_at(int64_t c, int64_t chunk, int64_t N) {
    const int64_t t1 = c * chunk;
    return (chunk < N - t1) ? chunk : N - t1;
}

__global__ void detect_stats(const float* __restrict__ X, int64_t M, int64_t N, int64_t chunk, int64_t pad,
                             double detect_threshold, ChunkStats* __restrict__ stats) {
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    if (m >= M) return;
    const int64_t t1 = c * chunk;
    const int64_t len = chunk_size_at(c, chunk, N) + 2 * pad;
    double sum = 0.0, sumsqr = 0.0;
    for (int64_t n0 = 0; n0 < len; n0 += kBatch) {
        float b[kBatch];
        load_batch(X, M, N, t1 - pad + n0, m, len - n0, b);
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
            if (n0 + k < len) {
                const double v = (double)b[k];
                sum = __dadd_rn(sum, v);
                sumsqr = __dadd_rn(sumsqr, __dmul_rn(v, v));
            }
        }
    }
    const double ct = (double)len;
    const double mean = __ddiv_rn(sum, ct);
    const double stdev =
        len >= 2 ? sqrt(__ddiv_rn(__dsub_rn(sumsqr, __ddiv_rn(__dmul_rn(sum, sum), ct)), ct - 1.0)) : 0.0;
    stats[c * M + m] = {mean, __dmul_rn(detect_threshold, stdev)};
}

__device__ __forceinline__ double deviation(float x, double mean, int sign) {
    double val = (double)x - mean;
    if (sign < 0)
        val = -val;
    else if (sign == 0)
        val = fabs(val);
    return val;
}

// Candidates of (channel m, chunk c, sub-range s): counted (WRITE == false) or
// written in time order from `base` (their index n inside the padded chunk and
// their deviation).
template <bool WRITE>
__global__ void detect_candidates(const float* __restrict__ X, int64_t M, int64_t N, int64_t chunk, int64_t pad,
                                  int64_t nchunks, const ChunkStats* __restrict__ stats, int sign,
                                  int64_t* __restrict__ counts, const int64_t* __restrict__ base,
                                  int64_t* __restrict__ cand_n, double* __restrict__ cand_v) {
    const int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t c = blockIdx.y;
    const int s = blockIdx.z;
    if (m >= M) return;
    const int64_t t1 = c * chunk;
    const int64_t len = chunk_size_at(c, chunk, N) + 2 * pad;
    const int64_t a = len * s / kSub, e = len * (s + 1) / kSub;
    const ChunkStats st = stats[c * M + m];
    const int64_t slot = (m * nchunks + c) * kSub + s;
    int64_t k = WRITE ? base[slot] : 0;
    for (int64_t n0 = a; n0 < e; n0 += kBatch) {
        float b[kBatch];
        load_batch(X, M, N, t1 - pad + n0, m, e - n0, b);
#pragma unroll
        for (int j = 0; j < kBatch; j++) {
            if (n0 + j < e) {
                const double val = deviation(b[j], st.mean, sign);
                if (val > st.threshold2) {
                    if (WRITE) {
                        cand_n[k] = n0 + j;
                        cand_v[k] = val;
                    }
                    k++;
                }
            }
        }
    }
    if (!WRITE) counts[slot] = k;
}

// The greedy rule of detect_events (detect_events.cpp:87-125) over the
// candidates [b, b + n) of one (channel, chunk), in time order; then the
// kept times inside [pad, pad + size) counted (WRITE == false) or written.
template <bool WRITE>
__global__ void detect_greedy(int64_t M, int64_t N, int64_t chunk, int64_t pad, int64_t nchunks, double interval,
                              const int64_t* __restrict__ cand_off, const int64_t* __restrict__ cand_n,
                              const double* __restrict__ cand_v, uint8_t* __restrict__ use,
                              int64_t* __restrict__ kept, const int64_t* __restrict__ kept_off,
                              int64_t* __restrict__ times) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;  // m * nchunks + c
    if (k >= M * nchunks) return;
    const int64_t c = k % nchunks;
    const int64_t b = cand_off[k * kSub], n = cand_off[(k + 1) * kSub] - b;
    const int64_t* tc = cand_n + b;
    const double* vc = cand_v + b;
    uint8_t* to_use = use + b;
    if (!WRITE) {
        int64_t last_best_ind = -1;
        for (int64_t i = 0; i < n; i++) {
            if (last_best_ind >= 0) {
                if ((double)tc[last_best_ind] < (double)tc[i] - interval) {
                    last_best_ind = -1;
                    if ((i > 0) && ((double)tc[i - 1] >= (double)tc[i] - interval)) {
                        last_best_ind = i - 1;
                        int64_t jj = last_best_ind;
                        while ((jj - 1 >= 0) && ((double)tc[jj - 1] >= (double)tc[i] - interval)) {
                            if (vc[jj - 1] > vc[last_best_ind]) last_best_ind = jj - 1;
                            jj--;
                        }
                    }
                }
            }
            if (last_best_ind >= 0) {
                if (vc[i] > vc[last_best_ind]) {
                    to_use[i] = 1;
                    to_use[last_best_ind] = 0;
                    last_best_ind = i;
                } else {
                    to_use[i] = 0;
                }
            } else {
                to_use[i] = 1;
                last_best_ind = i;
            }
        }
    }
    const int64_t size = chunk_size_at(c, chunk, N);
    int64_t count = 0;
    for (int64_t i = 0; i < n; i++) {
        if (!to_use[i]) continue;
        const int64_t t0 = tc[i];
        if (t0 - pad >= 0 && t0 - pad < size) {
            if (WRITE) times[kept_off[k] + count] = t0 - pad + c * chunk;
            count++;
        }
    }
    if (!WRITE) kept[k] = count;
}

}  // namespace

int64_t detect_chunk_size(int64_t M, int64_t N, int64_t num_simultaneous) {
    // get_time_chunk_infos (p_mountainsort3.cpp:507-517) with min_num_chunks 1
    int64_t chunk_size = (int64_t)1e9 / (M * num_simultaneous * 4);
    if (chunk_size > N) chunk_size = N;
    if (chunk_size < 20000) chunk_size = 20000;
    return chunk_size;
}

void detect_events_device(const float* X, int64_t M, int64_t N, double detect_threshold, double detect_interval,
                          int sign, int64_t chunk, int64_t pad, std::vector<int64_t>& counts,
                          std::vector<int64_t>& times, cudaStream_t stream) {
    counts.assign((size_t)std::max<int64_t>(M, 0), 0);
    times.clear();
    if (M <= 0 || N <= 0) return;
    const int64_t nchunks = ceil_div(N, chunk);
    if (nchunks > 65535) throw_unsupported("too many time chunks");
    const int64_t MC = M * nchunks;
    DevBuf stats(sizeof(ChunkStats) * (size_t)MC, stream);
    DevBuf cnt(sizeof(int64_t) * (size_t)(MC * kSub + 1), stream);
    const int threads = 32;  // a warp: 32 consecutive channels
    detect_stats<<<dim3((unsigned)ceil_div(M, threads), (unsigned)nchunks), threads, 0, stream>>>(
        X, M, N, chunk, pad, detect_threshold, stats.as<ChunkStats>());
    MS3_LAUNCH_CHECK();
    const dim3 gc((unsigned)ceil_div(M, threads), (unsigned)nchunks, (unsigned)kSub);
    detect_candidates<false><<<gc, threads, 0, stream>>>(X, M, N, chunk, pad, nchunks, stats.as<ChunkStats>(), sign,
                                                         cnt.as<int64_t>(), nullptr, nullptr, nullptr);
    MS3_LAUNCH_CHECK();
    // candidate offsets, channel-major, then chunk, then sub-range (time order)
    std::vector<int64_t> h((size_t)(MC * kSub)), off((size_t)(MC * kSub + 1));
    MS3_CUDA(cudaMemcpyAsync(h.data(), cnt.get(), sizeof(int64_t) * h.size(), cudaMemcpyDeviceToHost, stream));
    MS3_CUDA(cudaStreamSynchronize(stream));
    off[0] = 0;
    for (size_t k = 0; k < h.size(); k++) off[k + 1] = off[k] + h[k];
    const int64_t ncand = off.back();
    if (ncand > ((int64_t)1 << 31)) throw_unsupported("too many threshold crossings (lower the sensitivity)");
    DevBuf doff(sizeof(int64_t) * off.size(), stream);
    MS3_CUDA(cudaMemcpyAsync(doff.get(), off.data(), sizeof(int64_t) * off.size(), cudaMemcpyHostToDevice, stream));
    DevBuf cn(sizeof(int64_t) * (size_t)std::max<int64_t>(ncand, 1), stream);
    DevBuf cv(sizeof(double) * (size_t)std::max<int64_t>(ncand, 1), stream);
    DevBuf use((size_t)std::max<int64_t>(ncand, 1), stream);
    detect_candidates<true><<<gc, threads, 0, stream>>>(X, M, N, chunk, pad, nchunks, stats.as<ChunkStats>(), sign,
                                                        nullptr, doff.as<int64_t>(), cn.as<int64_t>(), cv.as<double>());
    MS3_LAUNCH_CHECK();
    DevBuf kept(sizeof(int64_t) * (size_t)MC, stream);
    const unsigned gg = (unsigned)ceil_div(MC, 128);
    detect_greedy<false><<<gg, 128, 0, stream>>>(M, N, chunk, pad, nchunks, detect_interval, doff.as<int64_t>(),
                                                 cn.as<int64_t>(), cv.as<double>(), use.as<uint8_t>(),
                                                 kept.as<int64_t>(), nullptr, nullptr);
    MS3_LAUNCH_CHECK();
    std::vector<int64_t> hk((size_t)MC), koff((size_t)MC);
    MS3_CUDA(cudaMemcpyAsync(hk.data(), kept.get(), sizeof(int64_t) * hk.size(), cudaMemcpyDeviceToHost, stream));
    MS3_CUDA(cudaStreamSynchronize(stream));
    int64_t total = 0;
    for (size_t k = 0; k < hk.size(); k++) {
        koff[k] = total;
        total += hk[k];
        counts[k / (size_t)nchunks] += hk[k];
    }
    times.resize((size_t)total);
    if (total == 0) return;
    DevBuf dkoff(sizeof(int64_t) * koff.size(), stream), dtimes(sizeof(int64_t) * (size_t)total, stream);
    MS3_CUDA(cudaMemcpyAsync(dkoff.get(), koff.data(), sizeof(int64_t) * koff.size(), cudaMemcpyHostToDevice, stream));
    detect_greedy<true><<<gg, 128, 0, stream>>>(M, N, chunk, pad, nchunks, detect_interval, doff.as<int64_t>(),
                                                cn.as<int64_t>(), cv.as<double>(), use.as<uint8_t>(), nullptr,
                                                dkoff.as<int64_t>(), dtimes.as<int64_t>());
    MS3_LAUNCH_CHECK();
    MS3_CUDA(cudaMemcpyAsync(times.data(), dtimes.get(), sizeof(int64_t) * (size_t)total, cudaMemcpyDeviceToHost,
                             stream));
    MS3_CUDA(cudaStreamSynchronize(stream));
}

}  // namespace ms3gpu
