// Streaming forms of ms3.bandpass_filter, ms3.whiten and ms3.mask_out_artifacts.
//
// The reference reads its input in chunks through DiskReadMda32::readChunk
// (mda/diskreadmda32.cpp:615-661) and writes them with
// DiskWriteMda::writeChunk (mda/diskwritemda.cpp:255-265), so a recording
// never has to fit in memory (p_bandpass_filter.cpp:160-220,
// p_whiten.cpp:64-206).  Here the caller's read / write callbacks move slabs
// of rows through two pinned host buffers and two device buffers: slab k+1
// is read and slab k-1 written on the host while slab k is copied in,
// computed and copied out on the GPU.
//
// Bandpass slabs are whole windows (chunks) plus their 60000-row halos on
// each side; the windows are filtered by the same kernels as the in-memory
// path with the slab's first row as origin, so every output row is the same.
// Whitening reads the recording twice, as the reference does: covariance
// partial sums slab by slab, then the apply slab by slab.  Slabs of pass 1
// are whole covariance slices of the whole recording, so the sum is the one
// the in-memory path forms (when one slice fits in a slab).
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "artifacts.h"
#include "bandpass.h"
#include "common.cuh"
#include "ms3gpu.h"
#include "stream.h"
#include "whiten.h"

namespace ms3gpu {

namespace {

constexpr int64_t kOverlapRows = 60000;
constexpr int64_t kDefaultSlabBytes = int64_t(1) << 30;

int64_t slab_bytes_of(const ms3gpu_stream_io& io) {
    return io.slab_bytes > 0 ? io.slab_bytes : kDefaultSlabBytes;
}

void read_rows(const ms3gpu_stream_io& io, int64_t t0, int64_t nt, void* dst) {
    if (nt <= 0) return;
    if (io.read(io.read_ctx, t0, nt, dst) != 0)
        throw Error(MS3GPU_ERR_IO, "read callback failed for timepoints [" + std::to_string(t0) + ", " +
                                       std::to_string(t0 + nt) + ")");
}

void write_rows(const ms3gpu_stream_io& io, int64_t t0, int64_t nt, const void* src) {
    if (nt <= 0) return;
    if (io.write(io.write_ctx, t0, nt, src) != 0)
        throw Error(MS3GPU_ERR_IO, "write callback failed for timepoints [" + std::to_string(t0) + ", " +
                                       std::to_string(t0 + nt) + ")");
}

// Page-locked host memory (so the copies run asynchronously at full speed).
class Pinned {
public:
    explicit Pinned(size_t bytes) {
        if (bytes) MS3_CUDA(cudaHostAlloc(&p_, bytes, cudaHostAllocDefault));
    }
    ~Pinned() {
        if (p_) cudaFreeHost(p_);
    }
    Pinned(const Pinned&) = delete;
    Pinned& operator=(const Pinned&) = delete;
    void* get() const { return p_; }

private:
    void* p_ = nullptr;
};

// Input rows [a, b) of a slab and the output rows [o0, o1) it produces.
struct SlabRows {
    int64_t a = 0, b = 0, o0 = 0, o1 = 0;
};

// The double-buffered slab pipeline.  Buffers are sized once for the largest
// slab; run() may be called several times (the two passes of whitening).
class SlabPipe {
public:
    SlabPipe(size_t in_bytes, size_t out_bytes, cudaStream_t s)
        : s_(s), hin0_(in_bytes), hin1_(in_bytes), hout0_(out_bytes), hout1_(out_bytes), din0_(in_bytes, s),
          din1_(in_bytes, s), dout0_(out_bytes, s), dout1_(out_bytes, s), in_bytes_(in_bytes), out_bytes_(out_bytes) {
        MS3_CUDA(cudaStreamCreateWithFlags(&h2d_, cudaStreamNonBlocking));
        MS3_CUDA(cudaStreamCreateWithFlags(&d2h_, cudaStreamNonBlocking));
        for (cudaEvent_t* e : {&ev_alloc_, &ev_h2d_[0], &ev_h2d_[1], &ev_comp_[0], &ev_comp_[1], &ev_d2h_[0],
                               &ev_d2h_[1]})
            MS3_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        // the device buffers come from the stream-ordered pool of `s`: the
        // copy streams must not touch them before the allocation is ordered
        MS3_CUDA(cudaEventRecord(ev_alloc_, s_));
        MS3_CUDA(cudaStreamWaitEvent(h2d_, ev_alloc_, 0));
        MS3_CUDA(cudaStreamWaitEvent(d2h_, ev_alloc_, 0));
    }
    ~SlabPipe() {
        // drain every copy before the pinned and device buffers are released
        if (h2d_) cudaStreamSynchronize(h2d_);
        if (d2h_) cudaStreamSynchronize(d2h_);
        for (cudaEvent_t e : {ev_alloc_, ev_h2d_[0], ev_h2d_[1], ev_comp_[0], ev_comp_[1], ev_d2h_[0], ev_d2h_[1]})
            if (e) cudaEventDestroy(e);
        if (h2d_) cudaStreamDestroy(h2d_);
        if (d2h_) cudaStreamDestroy(d2h_);
    }
    SlabPipe(const SlabPipe&) = delete;
    SlabPipe& operator=(const SlabPipe&) = delete;

    // rows(k) -> SlabRows; compute(k, rows, din, dout) issues slab k's work
    // on the compute stream.  out_row_bytes == 0: no output (nothing written).
    template <class RowsF, class ComputeF>
    void run(int64_t n, size_t in_row_bytes, size_t out_row_bytes, const ms3gpu_stream_io& io, RowsF rows,
             ComputeF compute) {
        void* hin[2] = {hin0_.get(), hin1_.get()};
        void* hout[2] = {hout0_.get(), hout1_.get()};
        void* din[2] = {din0_.get(), din1_.get()};
        void* dout[2] = {dout0_.get(), dout1_.get()};
        const bool out = out_row_bytes > 0;
        SlabRows prev;
        for (int64_t k = 0; k < n; k++) {
            const int b = (int)(k & 1);
            const SlabRows r = rows(k);
            const size_t ib = in_row_bytes * (size_t)(r.b - r.a), ob = out_row_bytes * (size_t)(r.o1 - r.o0);
            if (ib > in_bytes_ || ob > out_bytes_) throw_invalid("slab larger than its buffers");
            // the pinned input buffer is free once slab k-2's copy is done
            if (k >= 2) MS3_CUDA(cudaEventSynchronize(ev_h2d_[b]));
            read_rows(io, r.a, r.b - r.a, hin[b]);
            // the device input buffer is free once slab k-2 is computed
            if (k >= 2) MS3_CUDA(cudaStreamWaitEvent(h2d_, ev_comp_[b], 0));
            if (ib) MS3_CUDA(cudaMemcpyAsync(din[b], hin[b], ib, cudaMemcpyHostToDevice, h2d_));
            MS3_CUDA(cudaEventRecord(ev_h2d_[b], h2d_));
            MS3_CUDA(cudaStreamWaitEvent(s_, ev_h2d_[b], 0));
            // the device output buffer is free once slab k-2 is copied out
            if (k >= 2 && out) MS3_CUDA(cudaStreamWaitEvent(s_, ev_d2h_[b], 0));
            compute(k, r, din[b], dout[b]);
            MS3_CUDA(cudaEventRecord(ev_comp_[b], s_));
            if (out) {
                MS3_CUDA(cudaStreamWaitEvent(d2h_, ev_comp_[b], 0));
                if (ob) MS3_CUDA(cudaMemcpyAsync(hout[b], dout[b], ob, cudaMemcpyDeviceToHost, d2h_));
                MS3_CUDA(cudaEventRecord(ev_d2h_[b], d2h_));
            }
            // slab k-1 is written while slab k is on the GPU
            if (k >= 1 && out) {
                MS3_CUDA(cudaEventSynchronize(ev_d2h_[1 - b]));
                write_rows(io, prev.o0, prev.o1 - prev.o0, hout[1 - b]);
            }
            prev = r;
        }
        if (n >= 1 && out) {
            MS3_CUDA(cudaEventSynchronize(ev_d2h_[(n - 1) & 1]));
            write_rows(io, prev.o0, prev.o1 - prev.o0, hout[(n - 1) & 1]);
        }
        MS3_CUDA(cudaStreamSynchronize(s_));
    }

private:
    cudaStream_t s_ = nullptr, h2d_ = nullptr, d2h_ = nullptr;
    cudaEvent_t ev_alloc_ = nullptr, ev_h2d_[2] = {nullptr, nullptr}, ev_comp_[2] = {nullptr, nullptr},
                ev_d2h_[2] = {nullptr, nullptr};
    Pinned hin0_, hin1_, hout0_, hout1_;
    DevBuf din0_, din1_, dout0_, dout1_;
    size_t in_bytes_ = 0, out_bytes_ = 0;
};

}  // namespace

void bandpass_stream(int64_t M, int64_t N, bool in_i16, const ms3gpu_stream_io& io, const BandpassParams& bp,
                     cudaStream_t s) {
    const size_t in_esz = in_i16 ? 2 : 4;
    const int64_t slab_bytes = slab_bytes_of(io);
    if (M <= 0 || N <= 0) return;
    if (bp.freq_max == 0) {
        // p_bandpass_filter.cpp:117-119: the input is copied unchanged, row
        // blocks through one host buffer (no device work)
        const int64_t rows = std::max<int64_t>(1, slab_bytes / (M * (int64_t)in_esz));
        Pinned buf(in_esz * (size_t)(std::min(rows, N) * M));
        for (int64_t t = 0; t < N; t += rows) {
            const int64_t nt = std::min(rows, N - t);
            read_rows(io, t, nt, buf.get());
            write_rows(io, t, nt, buf.get());
        }
        return;
    }
    const int sub = bp.subsample_factor ? bp.subsample_factor : 1;
    const int64_t N2 = N / sub;
    if (N2 <= 0) return;
    const size_t out_esz = bp.quantization_unit != 0 ? 2 : 4;
    const int64_t chunk = bandpass_chunk_size(M, bp.num_threads);
    const int64_t nchunks = ceil_div(N, chunk);
    // windows per slab: the slab's own rows fill about slab_bytes
    const int64_t wps = std::max<int64_t>(1, slab_bytes / (chunk * M * (int64_t)in_esz));
    const int64_t n = ceil_div(nchunks, wps);
    const int64_t in_rows_max = std::min(N, wps * chunk + 2 * kOverlapRows);
    const int64_t out_rows_max = std::min(N2, wps * chunk / sub + 1);
    const size_t in_row_bytes = in_esz * (size_t)M, out_row_bytes = out_esz * (size_t)M;
    SlabPipe pipe(in_row_bytes * (size_t)in_rows_max, out_row_bytes * (size_t)out_rows_max, s);
    auto rows = [&](int64_t k) {
        const int64_t c0 = k * wps, c1 = std::min(nchunks, c0 + wps);
        SlabRows r;
        r.a = std::max<int64_t>(0, c0 * chunk - kOverlapRows);
        r.b = std::min(N, c1 * chunk + kOverlapRows);
        bandpass_output_rows(N, chunk, sub, c0, c1, r.o0, r.o1);
        return r;
    };
    pipe.run(n, in_row_bytes, out_row_bytes, io, rows, [&](int64_t k, const SlabRows& r, void* din, void* dout) {
        const int64_t c0 = k * wps, c1 = std::min(nchunks, c0 + wps);
        bandpass_device(din, M, N, dout, bp, s, c0, c1, in_i16, r.a, r.o0);
    });
    bandpass_check_timeout(s);
}

void whiten_stream(int64_t M, int64_t N, const ms3gpu_stream_io& io, double quantization_unit, bool mixed,
                   cudaStream_t s) {
    if (M <= 0 || N <= 0) return;
    const int64_t slab_bytes = slab_bytes_of(io);
    const size_t row_bytes = sizeof(float) * (size_t)M;
    const size_t out_row_bytes = (quantization_unit > 0 ? 2 : 4) * (size_t)M;
    // the slab buffers are pool allocations (256-byte aligned): plan for an
    // aligned pointer
    const CovPlan cp = cov_plan(nullptr, M);
    int64_t tslice = cov_tslice(cp, N);
    const int64_t slab_rows = std::max<int64_t>(1, slab_bytes / (int64_t)row_bytes);
    if (tslice > slab_rows) tslice = std::max<int64_t>(32, slab_rows / 32 * 32);
    const int64_t R = std::max<int64_t>(1, slab_rows / tslice) * tslice;  // rows per slab, whole slices
    const int64_t n = ceil_div(N, R);
    const int64_t slices_per_slab = R / tslice;
    const int64_t S_total = ceil_div(N, tslice);
    const int64_t rows_max = std::min(N, R);
    SlabPipe pipe(row_bytes * (size_t)rows_max, out_row_bytes * (size_t)rows_max, s);
    DevBuf partials(cov_partials_bytes(cp, S_total), s);
    DevBuf mats(sizeof(double) * (size_t)(2 * M * M), s);
    double* XXt = mats.as<double>();
    double* W = XXt + M * M;
    auto rows = [&](int64_t k) {
        SlabRows r;
        r.a = r.o0 = k * R;
        r.b = r.o1 = std::min(N, (k + 1) * R);
        return r;
    };
    // pass 1 (p_whiten.cpp:64-118): covariance partial sums
    pipe.run(n, row_bytes, 0, io, rows, [&](int64_t k, const SlabRows& r, void* din, void*) {
        double* part = reinterpret_cast<double*>(partials.as<char>() + cov_partials_bytes(cp, k * slices_per_slab));
        cov_partials_sliced(static_cast<const float*>(din), M, 0, r.b - r.a, cp, part, tslice, s);
    });
    cov_finish(partials.as<double>(), S_total, cp, M, N, XXt, s);
    whitening_matrix_device(XXt, M, W, nullptr, nullptr, s);
    // pass 2 (p_whiten.cpp:153-206): the apply
    DevBuf errbuf(sizeof(int), s);
    MS3_CUDA(cudaMemsetAsync(errbuf.get(), 0, sizeof(int), s));
    pipe.run(n, row_bytes, out_row_bytes, io, rows, [&](int64_t, const SlabRows& r, void* din, void* dout) {
        apply_whitening_device(static_cast<const float*>(din), M, r.b - r.a, W, quantization_unit, mixed, dout, s,
                               errbuf.as<int>());
    });
    int herr = 0;
    MS3_CUDA(cudaMemcpyAsync(&herr, errbuf.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
    MS3_CUDA(cudaStreamSynchronize(s));
    covariance_check_timeout(s);
    if (herr) throw Error(MS3GPU_ERR_CUDA, "tensor-core apply: pipeline wait timed out");
}

int64_t mask_out_artifacts_stream(int64_t M, int64_t N, double threshold, int64_t I, const ms3gpu_stream_io& io,
                                  cudaStream_t s) {
    if (M <= 0 || N <= 0) return 0;
    const int64_t nint = N / I;
    const size_t row_bytes = sizeof(float) * (size_t)M;
    // slabs of whole intervals
    const int64_t R = std::max<int64_t>(1, slab_bytes_of(io) / (int64_t)row_bytes / I) * I;
    const int64_t rows_max = std::min(N, R);
    SlabPipe pipe(row_bytes * (size_t)rows_max, row_bytes * (size_t)rows_max, s);
    DevBuf norms(sizeof(double) * (size_t)std::max<int64_t>(1, nint * M), s);
    DevBuf exceed(sizeof(int) * (size_t)(nint + 2), s);
    // pass 1 (p_mask_out_artifacts.cpp:37-58): norms of the whole intervals,
    // which end at timepoint nint * I
    const int64_t covered = nint * I;
    pipe.run(ceil_div(covered, R), row_bytes, 0, io,
             [&](int64_t k) {
                 SlabRows r;
                 r.a = k * R;
                 r.b = std::min(covered, (k + 1) * R);
                 return r;
             },
             [&](int64_t, const SlabRows& r, void* din, void*) {
                 artifact_norms_device(static_cast<const float*>(din), M, I, (r.b - r.a) / I,
                                       norms.as<double>() + (r.a / I) * M, s);
             });
    artifact_flags_device(norms.as<double>(), M, nint, threshold, exceed.as<int>(), s);
    // pass 2 (:60-99): the masked copy, zeros beyond the last whole interval
    pipe.run(ceil_div(N, R), row_bytes, row_bytes, io,
             [&](int64_t k) {
                 SlabRows r;
                 r.a = r.o0 = k * R;
                 r.b = r.o1 = std::min(N, (k + 1) * R);
                 return r;
             },
             [&](int64_t, const SlabRows& r, void* din, void* dout) {
                 artifact_write_device(static_cast<const float*>(din), M, r.b - r.a, r.a, I, nint,
                                       exceed.as<int>(), static_cast<float*>(dout), s);
             });
    return artifact_kept(exceed.as<int>(), nint, I, s);
}

}  // namespace ms3gpu
