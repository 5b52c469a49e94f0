// Host-buffer entry points with copies overlapped with the kernels.
//
// The recording is cut into slabs of whole chunks (about 1 GiB of rows).
// Input slabs go host -> device on a copy stream; each slab's windows are
// filtered and their covariance partial tiles summed as soon as the rows
// they read have arrived (a window also reads 60000 rows of the next slab).
// When the covariance is complete the whitening matrix is formed, and output
// slabs are whitened and copied device -> host on a second copy stream while
// the next slab is being whitened.  Work is issued in an interleaved order so
// that pageable host buffers (whose copies block the host) overlap as well.
// The result is identical to the unstreamed path: the same kernels on the
// same windows, and the covariance slices are summed in a fixed order.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "bandpass.h"
#include "common.cuh"
#include "ms3gpu.h"
#include "pipeline.h"
#include "whiten.h"

namespace ms3gpu {

namespace {

constexpr int64_t kOverlapRows = 60000;
constexpr size_t kSlabBytes = size_t(1) << 30;

struct Streams {
    cudaStream_t h2d = nullptr, d2h = nullptr;
    std::vector<cudaEvent_t> events;
    Streams() {
        MS3_CUDA(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
        MS3_CUDA(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
    }
    ~Streams() {
        if (h2d) cudaStreamSynchronize(h2d);
        if (d2h) cudaStreamSynchronize(d2h);
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        if (h2d) cudaStreamDestroy(h2d);
        if (d2h) cudaStreamDestroy(d2h);
    }
    cudaEvent_t record(cudaStream_t s) {
        cudaEvent_t e;
        MS3_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        events.push_back(e);
        MS3_CUDA(cudaEventRecord(e, s));
        return e;
    }
};

// Slab k covers chunks [k*wps, (k+1)*wps) and rows [k*wps*chunk, ...).
struct Slabs {
    int64_t N = 0, chunk = 0, nchunks = 0, wps = 0, n = 0;
    Slabs(int64_t N_, int64_t M, int64_t chunk_) : N(N_), chunk(chunk_) {
        nchunks = ceil_div(N, chunk);
        const int64_t row_bytes = std::max<int64_t>(1, M) * (int64_t)sizeof(float);
        wps = std::max<int64_t>(1, (int64_t)kSlabBytes / (chunk * row_bytes));
        n = ceil_div(nchunks, wps);
    }
    int64_t row0(int64_t k) const { return std::min(N, k * wps * chunk); }
    int64_t row1(int64_t k) const { return std::min(N, (k + 1) * wps * chunk); }
    int64_t c0(int64_t k) const { return k * wps; }
    int64_t c1(int64_t k) const { return std::min(nchunks, (k + 1) * wps); }
    // last input slab read by the windows of slab k
    int64_t needs(int64_t k) const {
        const int64_t last_row = std::min(N, c1(k) * chunk + kOverlapRows) - 1;
        return std::min(n - 1, last_row / (wps * chunk));
    }
};

void copy_rows_h2d(float* dst_d, const float* src_h, int64_t M, int64_t r0, int64_t r1, cudaStream_t s) {
    if (r1 > r0)
        MS3_CUDA(cudaMemcpyAsync(dst_d + r0 * M, src_h + r0 * M, sizeof(float) * (size_t)((r1 - r0) * M),
                                 cudaMemcpyHostToDevice, s));
}

void copy_rows_d2h(void* dst_h, const void* src_d, int64_t M, int64_t r0, int64_t r1, size_t esz, cudaStream_t s) {
    if (r1 > r0)
        MS3_CUDA(cudaMemcpyAsync(static_cast<char*>(dst_h) + (size_t)(r0 * M) * esz,
                                 static_cast<const char*>(src_d) + (size_t)(r0 * M) * esz,
                                 esz * (size_t)((r1 - r0) * M), cudaMemcpyDeviceToHost, s));
}

}  // namespace

void bandpass_whiten_streamed(const float* raw_h, int64_t M, int64_t N, float* filt_h, void* pre_h,
                              const BandpassParams& bp, double q, bool mixed, cudaStream_t s) {
    if (M <= 0 || N <= 0) return;
    const int64_t chunk = bandpass_chunk_size(M, bp.num_threads);
    const Slabs sl(N, M, chunk);
    const size_t esz = q > 0 ? 2 : 4;
    DevBuf raw_d(sizeof(float) * (size_t)(M * N), s), filt_d(sizeof(float) * (size_t)(M * N), s);
    float* raw = raw_d.as<float>();
    float* filt = filt_d.as<float>();
    // declared after the buffers: on any exit the copy streams are drained
    // before the buffers go back to the pool
    Streams st;
    // the device buffers come from the stream-ordered pool of `s`: the copy
    // streams must not touch them before the allocation is ordered
    cudaEvent_t alloc_ev = st.record(s);
    MS3_CUDA(cudaStreamWaitEvent(st.h2d, alloc_ev, 0));
    MS3_CUDA(cudaStreamWaitEvent(st.d2h, alloc_ev, 0));

    const CovPlan cp = cov_plan(filt, M);
    std::vector<int64_t> slices((size_t)sl.n), soff((size_t)sl.n + 1, 0);
    for (int64_t k = 0; k < sl.n; k++) {
        slices[(size_t)k] = cov_slices(cp, sl.row1(k) - sl.row0(k));
        soff[(size_t)k + 1] = soff[(size_t)k] + slices[(size_t)k];
    }
    DevBuf partials(cov_partials_bytes(cp, soff[(size_t)sl.n]), s);
    DevBuf mats(sizeof(double) * (size_t)(2 * M * M), s);

    std::vector<cudaEvent_t> in_ev((size_t)sl.n, nullptr);
    auto issue_in = [&](int64_t k) {
        if (k < sl.n && !in_ev[(size_t)k]) {
            copy_rows_h2d(raw, raw_h, M, sl.row0(k), sl.row1(k), st.h2d);
            in_ev[(size_t)k] = st.record(st.h2d);
        }
    };
    // phase 1: copy in, filter, covariance partials
    issue_in(0);
    for (int64_t k = 0; k < sl.n; k++) {
        const int64_t need = sl.needs(k);
        for (int64_t j = k; j <= std::min(sl.n - 1, need + 1); j++) issue_in(j);
        MS3_CUDA(cudaStreamWaitEvent(s, in_ev[(size_t)need], 0));
        bandpass_device(raw, M, N, filt, bp, s, sl.c0(k), sl.c1(k));
        double* part_k = reinterpret_cast<double*>(partials.as<char>() + cov_partials_bytes(cp, soff[(size_t)k]));
        cov_partials(filt, M, sl.row0(k), sl.row1(k), cp, part_k, slices[(size_t)k], s);
        if (filt_h) {
            cudaEvent_t e = st.record(s);
            MS3_CUDA(cudaStreamWaitEvent(st.d2h, e, 0));
            copy_rows_d2h(filt_h, filt, M, sl.row0(k), sl.row1(k), sizeof(float), st.d2h);
        }
    }
    double* XXt = mats.as<double>();
    double* W = XXt + M * M;
    cov_finish(partials.as<double>(), soff[(size_t)sl.n], cp, M, N, XXt, s);
    whitening_matrix_device(XXt, M, W, nullptr, nullptr, s);
    // phase 2: whiten slab by slab into the (now unused) input buffer, copy
    // out; slab k+1 is issued before slab k's copy
    void* pre = raw;
    DevBuf errbuf(sizeof(int), s);
    MS3_CUDA(cudaMemsetAsync(errbuf.get(), 0, sizeof(int), s));
    std::vector<cudaEvent_t> out_ev((size_t)sl.n, nullptr);
    for (int64_t k = 0; k <= sl.n; k++) {
        if (k < sl.n) {
            const int64_t r0 = sl.row0(k), r1 = sl.row1(k);
            apply_whitening_device(filt + r0 * M, M, r1 - r0, W, q, mixed,
                                   static_cast<char*>(pre) + (size_t)(r0 * M) * esz, s, errbuf.as<int>());
            out_ev[(size_t)k] = st.record(s);
        }
        if (k >= 1) {
            MS3_CUDA(cudaStreamWaitEvent(st.d2h, out_ev[(size_t)k - 1], 0));
            copy_rows_d2h(pre_h, pre, M, sl.row0(k - 1), sl.row1(k - 1), esz, st.d2h);
        }
    }
    // buffers return to the pool on `s` only after the copies are done
    cudaEvent_t out_done = st.record(st.d2h);
    MS3_CUDA(cudaStreamWaitEvent(s, out_done, 0));
    int herr = 0;
    MS3_CUDA(cudaMemcpyAsync(&herr, errbuf.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    MS3_CUDA(cudaStreamSynchronize(s));
    if (herr) throw Error(MS3GPU_ERR_CUDA, "tensor-core apply: pipeline wait timed out");
    bandpass_check_timeout(s);
    covariance_check_timeout(s);
}

}  // namespace ms3gpu
