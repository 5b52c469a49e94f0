// C ABI of libms3gpu (declared in include/ms3gpu.h).
//
// Each entry point validates its arguments, classifies every buffer as host
// or device memory, stages host buffers through stream-ordered device
// allocations, runs the device stages, copies results back and synchronises
// the stream.  C++ exceptions never cross the boundary: they become status
// codes plus the per-thread text returned by ms3gpu_last_error().
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <new>
#include <utility>
#include <string>
#include <vector>

#include "artifacts.h"
#include "bandpass.h"
#include "detect.h"
#include "common.cuh"
#include "ms3gpu.h"
#include "pipeline.h"
#include "ptrkind.h"
#include "stream.h"
#include "whiten.h"

namespace ms3gpu {

namespace {
thread_local std::string g_last_error;
std::mutex g_pool_mu;
bool g_pool_configured[64] = {false};
}  // namespace

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line) {
    cudaGetLastError();  // clear a non-sticky error so later calls can proceed
    const int code = (e == cudaErrorMemoryAllocation) ? MS3GPU_ERR_NOMEM : MS3GPU_ERR_CUDA;
    throw Error(code, std::string("CUDA error ") + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) +
                          ") in " + what + " at " + file + ":" + std::to_string(line));
}

[[noreturn]] void throw_invalid(const std::string& msg) { throw Error(MS3GPU_ERR_INVALID, msg); }

static unsigned long long g_launches = 0;
void count_launch() { __atomic_fetch_add(&g_launches, 1ULL, __ATOMIC_RELAXED); }
[[noreturn]] void throw_unsupported(const std::string& msg) { throw Error(MS3GPU_ERR_UNSUPPORTED, msg); }

// Test hook: MS3GPU_FAIL_ALLOC_AFTER=n makes the (n+1)-th device allocation
// of the process fail as if the device were out of memory.
static long long fail_alloc_countdown() {
    static long long v = [] {
        const char* s = std::getenv("MS3GPU_FAIL_ALLOC_AFTER");
        return (s && *s) ? std::atoll(s) : -1LL;
    }();
    return v;
}
static long long g_alloc_count = 0;

static void configure_pool() {
    int dev = 0;
    MS3_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (dev < 64 && !g_pool_configured[dev]) {
        cudaMemPool_t pool;
        MS3_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        uint64_t thr = std::numeric_limits<uint64_t>::max();
        MS3_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
        g_pool_configured[dev] = true;
    }
}

void DevBuf::alloc(size_t bytes, cudaStream_t s) {
    release();
    s_ = s;
    if (bytes == 0) return;
    const long long lim = fail_alloc_countdown();
    if (lim >= 0 && __atomic_fetch_add(&g_alloc_count, 1, __ATOMIC_RELAXED) >= lim)
        throw Error(MS3GPU_ERR_NOMEM, "device allocation of " + std::to_string(bytes) +
                                          " bytes failed (MS3GPU_FAIL_ALLOC_AFTER test hook)");
    configure_pool();
    MS3_CUDA(cudaMallocAsync(&p_, bytes, s));
    n_ = bytes;
}

void DevBuf::release() {
    if (p_) cudaFreeAsync(p_, s_);
    p_ = nullptr;
    n_ = 0;
}

namespace {

// True for memory the current device reaches in place (its own device
// memory, managed memory), false for host memory, which is staged.  Device
// memory of another GPU is rejected: a kernel given it would fault rather
// than fail cleanly.
bool is_device_ptr(const void* p) {
    if (!p) return false;
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    int cur = 0;
    MS3_CUDA(cudaGetDevice(&cur));
    switch (classify_pointer((int)a.type, a.device, cur)) {
    case PtrKind::DeviceHere:
    case PtrKind::Managed:
        return true;
    case PtrKind::DeviceElsewhere:
        throw_invalid("buffer is device memory of GPU " + std::to_string(a.device) + ", but the call runs on GPU " +
                      std::to_string(cur) + " (make that device current or copy the buffer)");
    default:
        return false;
    }
}

// A read-only view of a caller buffer on the device.
struct InView {
    const void* ptr = nullptr;
    DevBuf own;
};

void stage_in(InView& v, const void* p, size_t bytes, cudaStream_t s) {
    if (bytes == 0 || is_device_ptr(p)) {
        v.ptr = p;
        return;
    }
    v.own.alloc(bytes, s);
    MS3_CUDA(cudaMemcpyAsync(v.own.get(), p, bytes, cudaMemcpyHostToDevice, s));
    v.ptr = v.own.get();
}

// A writable device buffer for a caller output; copied back by finish().
struct OutView {
    void* user = nullptr;
    void* ptr = nullptr;
    size_t bytes = 0;
    bool host = false;
    DevBuf own;
    void setup(void* p, size_t b, cudaStream_t s, DevBuf* reuse = nullptr) {
        user = p;
        bytes = b;
        if (b == 0 || is_device_ptr(p)) {
            ptr = p;
            return;
        }
        host = true;
        if (reuse && reuse->get() && reuse->size() >= b) {
            ptr = reuse->get();
        } else {
            own.alloc(b, s);
            ptr = own.get();
        }
    }
    void finish(cudaStream_t s) {
        if (host && bytes) MS3_CUDA(cudaMemcpyAsync(user, ptr, bytes, cudaMemcpyDeviceToHost, s));
    }
};

// An NVTX range names each entry point on a profiler timeline (nvtx3 is
// header-only: without a tool attached the calls return at once).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
};

template <class F>
int guarded(F&& f);

template <class F>
int guarded(const char* name, F&& f) {
    NvtxRange range(name);
    return guarded(std::forward<F>(f));
}

// Bounds-checked build: a recorded index-check failure of any unit becomes
// this call's error (after the device has finished the call's work).
void bounds_check_all() {
#ifdef MS3GPU_BOUNDS_CHECK
    MS3_CUDA(cudaDeviceSynchronize());
    const int sites[4] = {bounds_site_bandpass(0), bounds_site_whiten(0), bounds_site_apply(0), bounds_site_cov(0)};
    for (int v : sites)
        if (v) throw Error(MS3GPU_ERR_CUDA, "bounds check failed at site " + std::to_string(v));
#endif
}

template <class F>
int guarded(F&& f) {
    try {
        f();
        bounds_check_all();
        g_last_error.clear();
        return MS3GPU_OK;
    } catch (const Error& e) {
        g_last_error = e.what();
        return e.code;
    } catch (const std::bad_alloc&) {
        g_last_error = "host memory exhausted";
        return MS3GPU_ERR_NOMEM;
    } catch (const std::exception& e) {
        g_last_error = e.what();
        return MS3GPU_ERR_INVALID;
    } catch (...) {
        g_last_error = "unknown error";
        return MS3GPU_ERR_INVALID;
    }
}

void check_shape(int64_t M, int64_t N) {
    if (M < 0 || N < 0) throw_invalid("negative dimension (M=" + std::to_string(M) + ", N=" + std::to_string(N) + ")");
    if (M > 0 && N > std::numeric_limits<int64_t>::max() / 8 / M) throw_invalid("timeseries too large");
}

void require(const void* p, const char* name, bool needed) {
    if (needed && !p) throw_invalid(std::string(name) + " is NULL");
}

BandpassParams to_params(const ms3gpu_bandpass_opts* o) {
    if (!o) throw_invalid("bandpass opts is NULL");
    BandpassParams p;
    p.samplerate = o->samplerate;
    p.freq_min = o->freq_min;
    p.freq_max = o->freq_max;
    p.freq_wid = o->freq_wid;
    p.quantization_unit = o->quantization_unit;
    p.subsample_factor = o->subsample_factor ? o->subsample_factor : 1;
    p.num_threads = o->num_threads;
    if (p.subsample_factor < 1) throw_invalid("subsample_factor must be >= 1");
    if (p.freq_max != 0) {
        if (!(p.samplerate > 0)) throw_invalid("samplerate must be > 0");
        if (p.num_threads < 1) throw_invalid("num_threads must be >= 1");
    }
    return p;
}

cudaStream_t as_stream(void* s) { return static_cast<cudaStream_t>(s); }

bool check_precision(int32_t p) {
    if (p != MS3GPU_PRECISION_PLAIN && p != MS3GPU_PRECISION_MIXED)
        throw_invalid("precision must be MS3GPU_PRECISION_PLAIN (0) or MS3GPU_PRECISION_MIXED (1)");
    return p == MS3GPU_PRECISION_MIXED;
}

}  // namespace
}  // namespace ms3gpu

using namespace ms3gpu;

extern "C" {

const char* ms3gpu_last_error(void) { return g_last_error.c_str(); }

const char* ms3gpu_version(void) { return "ms3gpu 0.1.0 (sm_100a)"; }

uint64_t ms3gpu_launch_count(void) { return __atomic_load_n(&g_launches, __ATOMIC_RELAXED); }

int ms3gpu_release_cached_memory(void) {
    return guarded(__func__, [&] {
        int dev = 0;
        MS3_CUDA(cudaGetDevice(&dev));
        cudaMemPool_t pool;
        MS3_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
        MS3_CUDA(cudaDeviceSynchronize());
        MS3_CUDA(cudaMemPoolTrimTo(pool, 0));
    });
}

int64_t ms3gpu_bandpass_chunk_size(int64_t M, int32_t num_threads) {
    if (M < 1 || num_threads < 1) return -1;
    return bandpass_chunk_size(M, num_threads);
}

int ms3gpu_bandpass_output_dims(int64_t M, int64_t N, const ms3gpu_bandpass_opts* opts, int64_t* M_out,
                                int64_t* N_out, int32_t* dtype_out) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        if (!opts) throw_invalid("opts is NULL");
        const int sub = opts->subsample_factor ? opts->subsample_factor : 1;
        if (sub < 1) throw_invalid("subsample_factor must be >= 1");
        if (M_out) *M_out = M;
        if (opts->freq_max == 0) {  // the input is copied unchanged
            if (N_out) *N_out = N;
            if (dtype_out) *dtype_out = MS3GPU_DTYPE_FLOAT32;
            return;
        }
        if (N_out) *N_out = N / sub;
        if (dtype_out) *dtype_out = opts->quantization_unit != 0 ? MS3GPU_DTYPE_INT16 : MS3GPU_DTYPE_FLOAT32;
    });
}

int ms3gpu_bandpass_requirements(int64_t M, int64_t N, const ms3gpu_bandpass_opts* opts, double* peak_ram_mb) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        if (!opts || !peak_ram_mb) throw_invalid("NULL argument");
        if (opts->num_threads < 1) throw_invalid("num_threads must be >= 1");
        // p_bandpass_filter.cpp:149-158
        const int overhead = 6;
        const int64_t chunk = bandpass_chunk_size(M, opts->num_threads);
        const double bytes = overhead * sizeof(float) * (double)M * opts->num_threads * (double)(chunk + 2 * 60000);
        *peak_ram_mb = bytes / (1024 * 1024);
    });
}

int ms3gpu_whiten_requirements(int64_t M, int64_t N, double* peak_ram_mb) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        if (!peak_ram_mb) throw_invalid("NULL argument");
        // p_whiten.cpp:53-57
        *peak_ram_mb = 3.0 * 1e5 * (double)M * sizeof(float) / (1024 * 1024);
    });
}

namespace {
void bandpass_any(const void* timeseries, bool in_i16, int64_t M, int64_t N, void* timeseries_out,
                  const ms3gpu_bandpass_opts* opts, void* stream) {
    check_shape(M, N);
    BandpassParams p = to_params(opts);
    cudaStream_t s = as_stream(stream);
    const bool copy = p.freq_max == 0;
    const int64_t N2 = copy ? N : N / p.subsample_factor;
    const size_t in_esz = in_i16 ? 2 : 4;
    const size_t esz = copy ? in_esz : (p.quantization_unit != 0 ? 2 : 4);
    const size_t in_bytes = in_esz * (size_t)(M * N);
    const size_t out_bytes = esz * (size_t)(M * N2);
    require(timeseries, "timeseries", in_bytes > 0);
    require(timeseries_out, "timeseries_out", out_bytes > 0);
    InView in;
    stage_in(in, timeseries, in_bytes, s);
    OutView out;
    out.setup(timeseries_out, out_bytes, s);
    bandpass_device(in.ptr, M, N, out.ptr, p, s, 0, -1, in_i16);
    out.finish(s);
    MS3_CUDA(cudaStreamSynchronize(s));
    bandpass_check_timeout(s);
}
}  // namespace

int ms3gpu_bandpass_filter(const float* timeseries, int64_t M, int64_t N, void* timeseries_out,
                           const ms3gpu_bandpass_opts* opts, void* stream) {
    return guarded(__func__, [&] { bandpass_any(timeseries, false, M, N, timeseries_out, opts, stream); });
}

int ms3gpu_bandpass_filter_i16(const int16_t* timeseries, int64_t M, int64_t N, void* timeseries_out,
                               const ms3gpu_bandpass_opts* opts, void* stream) {
    return guarded(__func__, [&] { bandpass_any(timeseries, true, M, N, timeseries_out, opts, stream); });
}

namespace {
// Device state of one batch job between its compute and its copy-back.
// The filtered signal's device buffer for a filter + whiten call without a
// caller filt buffer: a library buffer, or, when that does not fit beside the
// caller's buffers and the output is float32, the output buffer itself
// (in_place).  Returns nullptr with in_place set in that case.
float* alloc_filt_or_in_place(size_t in_bytes, double q, DevBuf& filt_own, cudaStream_t s, bool& in_place) {
    in_place = false;
    if (!in_bytes) return nullptr;
    const char* force = std::getenv("MS3GPU_FILT_IN_PLACE");  // testing: take the in-place path
    if (force && force[0] == '1' && q <= 0) {
        in_place = true;
        return nullptr;
    }
    try {
        filt_own.alloc(in_bytes, s);
        return filt_own.as<float>();
    } catch (const Error& e) {
        if (e.code != MS3GPU_ERR_NOMEM || q > 0) throw;
    }
    in_place = true;
    return nullptr;
}

// pre = W filt.  In place (filt_d is the float32 output buffer itself), the
// output is whitened in time slabs of whole 128-row tiles through a 256 MiB
// buffer and copied back: each output row depends only on its own filtered
// row, so the values are those of the one-pass apply.
void apply_maybe_in_place(const float* filt_d, bool in_place, int64_t M, int64_t N, const double* W, double q,
                          bool mixed, void* pre_d, cudaStream_t s, int* err) {
    if (!in_place) {
        apply_whitening_device(filt_d, M, N, W, q, mixed, pre_d, s, err);
        return;
    }
    const int64_t rows = std::max<int64_t>(128, (((int64_t)256 << 20) / (4 * std::max<int64_t>(1, M))) / 128 * 128);
    DevBuf slab(sizeof(float) * (size_t)(std::min(rows, N) * M), s);
    DevBuf own_err;
    if (!err) {
        own_err.alloc(sizeof(int), s);
        MS3_CUDA(cudaMemsetAsync(own_err.get(), 0, sizeof(int), s));
        err = own_err.as<int>();
    }
    float* pre_f = static_cast<float*>(pre_d);
    for (int64_t r0 = 0; r0 < N; r0 += rows) {
        const int64_t n = std::min(rows, N - r0);
        apply_whitening_device(pre_f + r0 * M, M, n, W, q, mixed, slab.get(), s, err);
        MS3_CUDA(cudaMemcpyAsync(pre_f + r0 * M, slab.get(), sizeof(float) * (size_t)(n * M), cudaMemcpyDeviceToDevice,
                                 s));
    }
    if (own_err.get()) {
        int herr = 0;
        MS3_CUDA(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, s));
        MS3_CUDA(cudaStreamSynchronize(s));
        if (herr) throw Error(MS3GPU_ERR_CUDA, "tensor-core apply: pipeline wait timed out");
    }
}

struct BatchJob {
    cudaStream_t s = nullptr;
    InView in;
    OutView filt, pre;
    DevBuf filt_own, mats, err;
};

// Issues one job's device work on js (no copy back, no synchronisation).
void issue_batch_job(const ms3gpu_job& j, BatchJob& st) {
    check_shape(j.M, j.N);
    BandpassParams p = to_params(&j.bp);
    if (p.subsample_factor != 1 || p.quantization_unit != 0)
        throw_invalid("bandpass_whiten needs subsample_factor 1 and quantization_unit 0");
    const int64_t M = j.M, N = j.N;
    const double q = j.wh.quantization_unit;
    const bool mixed = check_precision(j.wh.precision);
    const size_t in_bytes = sizeof(float) * (size_t)(M * N);
    const size_t pre_bytes = (q > 0 ? 2 : 4) * (size_t)(M * N);
    require(j.timeseries, "timeseries", in_bytes > 0);
    require(j.pre_out, "pre_out", pre_bytes > 0);
    cudaStream_t s = st.s;
    stage_in(st.in, j.timeseries, in_bytes, s);
    float* filt_d = nullptr;
    bool in_place = false;
    if (j.filt_out) {
        st.filt.setup(j.filt_out, in_bytes, s);
        filt_d = static_cast<float*>(st.filt.ptr);
    } else {
        filt_d = alloc_filt_or_in_place(in_bytes, q, st.filt_own, s, in_place);
    }
    st.pre.setup(j.pre_out, pre_bytes, s);
    if (in_place) filt_d = static_cast<float*>(st.pre.ptr);
    bandpass_device(static_cast<const float*>(st.in.ptr), M, N, filt_d, p, s);
    st.mats.alloc(sizeof(double) * (size_t)(2 * M * M), s);
    double* XXt = st.mats.as<double>();
    double* W = XXt + M * M;
    covariance_device(filt_d, M, N, XXt, s);
    whitening_matrix_device(XXt, M, W, nullptr, nullptr, s);
    st.err.alloc(sizeof(int), s);
    MS3_CUDA(cudaMemsetAsync(st.err.get(), 0, sizeof(int), s));
    apply_maybe_in_place(filt_d, in_place, M, N, W, q, mixed, st.pre.ptr, s, st.err.as<int>());
}
}  // namespace

int ms3gpu_bandpass_whiten_batch(ms3gpu_job* jobs, int32_t n_jobs, void* stream) {
    std::string first_error;
    int first_code = MS3GPU_OK;
    const int rc = guarded([&] {
        if (n_jobs < 0) throw_invalid("n_jobs is negative");
        require(jobs, "jobs", n_jobs > 0);
        if (n_jobs == 0) return;
        cudaStream_t s0 = as_stream(stream);
        // Jobs of at least `large` ch-samples (default 3e8, 384 channels x 26 s)
        // fill the GPU by themselves (their persistent kernels take one CTA per
        // SM): they run one after another on the first stream, before the
        // smaller jobs, which are spread over K streams so that their short and
        // latency-bound kernels overlap.
        const char* ks = std::getenv("MS3GPU_BATCH_STREAMS");
        const char* ls = std::getenv("MS3GPU_BATCH_LARGE");
        const int K = std::max(1, std::min<int>(n_jobs, (ks && *ks) ? std::atoi(ks) : 4));
        const double large = (ls && *ls) ? std::atof(ls) : 3e8;
        std::vector<cudaStream_t> streams((size_t)K, nullptr);
        cudaEvent_t start = nullptr;
        MS3_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
        MS3_CUDA(cudaEventRecord(start, s0));
        for (auto& st : streams) {
            MS3_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            MS3_CUDA(cudaStreamWaitEvent(st, start, 0));
        }
        std::vector<std::unique_ptr<BatchJob>> state((size_t)n_jobs);
        auto record = [&](int i, int code, const std::string& msg) {
            jobs[i].status = code;
            if (code != MS3GPU_OK && first_code == MS3GPU_OK) {
                first_code = code;
                first_error = "job " + std::to_string(i) + ": " + msg;
            }
        };
        // phase 1: every job's device work, round-robin over the streams
        std::vector<int> order;
        for (int i = 0; i < n_jobs; i++)
            if ((double)jobs[i].M * (double)jobs[i].N >= large) order.push_back(i);
        const size_t nlarge = order.size();
        for (int i = 0; i < n_jobs; i++)
            if ((double)jobs[i].M * (double)jobs[i].N < large) order.push_back(i);
        cudaEvent_t large_done = nullptr;
        for (size_t k = 0; k < order.size(); k++) {
            const int i = order[k];
            if (k == nlarge && nlarge > 0) {  // the small jobs start once the large ones are done
                MS3_CUDA(cudaEventCreateWithFlags(&large_done, cudaEventDisableTiming));
                MS3_CUDA(cudaEventRecord(large_done, streams[0]));
                for (int t = 1; t < K; t++) MS3_CUDA(cudaStreamWaitEvent(streams[(size_t)t], large_done, 0));
            }
            state[(size_t)i].reset(new BatchJob);
            state[(size_t)i]->s = streams[k < nlarge ? 0 : (size_t)((k - nlarge) % K)];
            jobs[i].status = MS3GPU_OK;
            const int code = guarded([&] { issue_batch_job(jobs[i], *state[(size_t)i]); });
            if (code != MS3GPU_OK) record(i, code, ms3gpu_last_error());
        }
        // phase 2: copies back (a copy into pageable memory waits for its job)
        for (int i = 0; i < n_jobs; i++) {
            if (jobs[i].status != MS3GPU_OK) continue;
            BatchJob& st = *state[(size_t)i];
            const int code = guarded([&] {
                if (jobs[i].filt_out) st.filt.finish(st.s);
                st.pre.finish(st.s);
            });
            if (code != MS3GPU_OK) record(i, code, ms3gpu_last_error());
        }
        for (auto& st : streams) MS3_CUDA(cudaStreamSynchronize(st));
        for (int i = 0; i < n_jobs; i++) {
            if (jobs[i].status != MS3GPU_OK) continue;
            int herr = 0;
            const int code = guarded([&] {
                MS3_CUDA(cudaMemcpy(&herr, state[(size_t)i]->err.get(), sizeof(int), cudaMemcpyDeviceToHost));
                if (herr) throw Error(MS3GPU_ERR_CUDA, "tensor-core apply: pipeline wait timed out");
            });
            if (code != MS3GPU_OK) record(i, code, ms3gpu_last_error());
        }
        state.clear();  // device buffers go back to the pools of their streams
        for (auto& st : streams) {
            MS3_CUDA(cudaStreamSynchronize(st));
            MS3_CUDA(cudaStreamDestroy(st));
        }
        MS3_CUDA(cudaEventDestroy(start));
        if (large_done) MS3_CUDA(cudaEventDestroy(large_done));
        bandpass_check_timeout(s0);
        covariance_check_timeout(s0);
    });
    if (rc != MS3GPU_OK) return rc;
    if (first_code != MS3GPU_OK) {
        g_last_error = first_error;
        return first_code;
    }
    return MS3GPU_OK;
}

int ms3gpu_whiten_covariance(const float* timeseries, int64_t M, int64_t N, double* XXt, void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        cudaStream_t s = as_stream(stream);
        const size_t in_bytes = sizeof(float) * (size_t)(M * N);
        require(timeseries, "timeseries", in_bytes > 0);
        require(XXt, "XXt", M > 0);
        InView in;
        stage_in(in, timeseries, in_bytes, s);
        OutView out;
        out.setup(XXt, sizeof(double) * (size_t)(M * M), s);
        covariance_device(static_cast<const float*>(in.ptr), M, N, static_cast<double*>(out.ptr), s);
        out.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
        covariance_check_timeout(s);
    });
}

int ms3gpu_whiten_covariance_noalloc(const float* timeseries, int64_t M, int64_t N, double* XXt,
                                     void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        cudaStream_t s = as_stream(stream);
        require(timeseries, "timeseries", M * N > 0);
        require(XXt, "XXt", M > 0);
        // Staging host memory would allocate device buffers: only memory the
        // current device reaches in place is accepted.
        if (M * N > 0 && !is_device_ptr(timeseries))
            throw_invalid("ms3gpu_whiten_covariance_noalloc needs timeseries in device memory");
        if (M > 0 && !is_device_ptr(XXt)) throw_invalid("ms3gpu_whiten_covariance_noalloc needs XXt in device memory");
        // Queued on the caller's stream; the caller decides when to wait for it.
        covariance_device_noalloc(timeseries, M, N, XXt, s);
    });
}

int ms3gpu_whitening_matrix(const double* XXt, int64_t M, double* W, double* components, double* sigma,
                            void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, 0);
        cudaStream_t s = as_stream(stream);
        const size_t mm = sizeof(double) * (size_t)(M * M);
        require(XXt, "XXt", M > 0);
        require(W, "W", M > 0);
        InView in;
        stage_in(in, XXt, mm, s);
        OutView w, c, sg;
        w.setup(W, mm, s);
        if (components) c.setup(components, mm, s);
        if (sigma) sg.setup(sigma, sizeof(double) * (size_t)M, s);
        whitening_matrix_device(static_cast<const double*>(in.ptr), M, static_cast<double*>(w.ptr),
                                components ? static_cast<double*>(c.ptr) : nullptr,
                                sigma ? static_cast<double*>(sg.ptr) : nullptr, s);
        w.finish(s);
        if (components) c.finish(s);
        if (sigma) sg.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
        whitening_check_timeout(s);
    });
}

int ms3gpu_apply_whitening_matrix(const float* timeseries, int64_t M, int64_t N, const double* W,
                                  double quantization_unit, int32_t precision, void* timeseries_out,
                                  void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        cudaStream_t s = as_stream(stream);
        const size_t in_bytes = sizeof(float) * (size_t)(M * N);
        const size_t out_bytes = (quantization_unit > 0 ? 2 : 4) * (size_t)(M * N);
        require(timeseries, "timeseries", in_bytes > 0);
        require(timeseries_out, "timeseries_out", out_bytes > 0);
        require(W, "W", M > 0);
        InView in, w;
        stage_in(in, timeseries, in_bytes, s);
        stage_in(w, W, sizeof(double) * (size_t)(M * M), s);
        OutView out;
        out.setup(timeseries_out, out_bytes, s);
        apply_whitening_device(static_cast<const float*>(in.ptr), M, N, static_cast<const double*>(w.ptr),
                               quantization_unit, check_precision(precision), out.ptr, s);
        out.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
    });
}

int ms3gpu_compute_whitening_matrix(const float* const* timeseries_list, const int64_t* N_list, int32_t n_inputs,
                                    int64_t M, const int32_t* channels, int32_t n_channels, double* W_out,
                                    void* stream) {
    return guarded(__func__, [&] {
        if (n_inputs < 1) throw_invalid("timeseries_list is empty");
        require(timeseries_list, "timeseries_list", true);
        require(N_list, "N_list", true);
        if (M <= 0) throw_invalid("M must be positive");
        if (n_channels < 0) throw_invalid("n_channels is negative");
        require(channels, "channels", n_channels > 0);
        require(W_out, "W_out", true);
        const int64_t M2 = n_channels > 0 ? n_channels : M;
        std::vector<int32_t> ch0((size_t)M2);
        for (int64_t j = 0; j < M2; j++) {
            const int64_t c = n_channels > 0 ? channels[j] : j + 1;
            if (c < 1 || c > M)
                throw_invalid("channel " + std::to_string(c) + " is outside 1.." + std::to_string(M));
            ch0[(size_t)j] = (int32_t)(c - 1);
        }
        int64_t Ntot = 0;
        for (int32_t i = 0; i < n_inputs; i++) {
            check_shape(M, N_list[i]);
            require(timeseries_list[i], "timeseries_list entry", N_list[i] > 0);
            Ntot += N_list[i];
        }
        cudaStream_t s = as_stream(stream);
        DevBuf chmap;
        if (n_channels > 0) {
            chmap.alloc(sizeof(int32_t) * (size_t)M2, s);
            MS3_CUDA(cudaMemcpyAsync(chmap.get(), ch0.data(), sizeof(int32_t) * (size_t)M2, cudaMemcpyHostToDevice, s));
        }
        // the recordings' partial tiles go to consecutive slices of one buffer
        const CovPlan plan = cov_plan(nullptr, M2);
        std::vector<int64_t> slices((size_t)n_inputs);
        int64_t Stot = 0;
        for (int32_t i = 0; i < n_inputs; i++) Stot += (slices[(size_t)i] = cov_slices(plan, N_list[i]));
        DevBuf partials(cov_partials_bytes(plan, Stot), s);
        int64_t done = 0;
        for (int32_t i = 0; i < n_inputs; i++) {
            const int64_t Ni = N_list[i];
            if (Ni == 0) continue;
            InView in;
            stage_in(in, timeseries_list[i], sizeof(float) * (size_t)(M * Ni), s);
            const float* X = static_cast<const float*>(in.ptr);
            DevBuf sub;
            if (n_channels > 0) {
                sub.alloc(sizeof(float) * (size_t)(M2 * Ni), s);
                gather_channels_device(X, M, Ni, chmap.as<int32_t>(), M2, sub.as<float>(), s);
                X = sub.as<float>();
            }
            double* part_i = reinterpret_cast<double*>(partials.as<char>() + cov_partials_bytes(plan, done));
            cov_partials(X, M2, 0, Ni, cov_plan(X, M2), part_i, slices[(size_t)i], s);
            done += slices[(size_t)i];
        }
        DevBuf xxt(sizeof(double) * (size_t)(M2 * M2), s);
        cov_finish(partials.as<double>(), Stot, plan, M2, Ntot, xxt.as<double>(), s);
        OutView w;
        w.setup(W_out, sizeof(double) * (size_t)(M2 * M2), s);
        whitening_matrix_device(xxt.as<double>(), M2, static_cast<double*>(w.ptr), nullptr, nullptr, s);
        w.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
        covariance_check_timeout(s);
    });
}

int ms3gpu_whiten_blocks(const float* timeseries, int64_t M, int64_t N, const int32_t* channels,
                         const int32_t* block_sizes, int32_t n_blocks, void* timeseries_out,
                         const ms3gpu_whiten_opts* opts, void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        if (!opts) throw_invalid("whiten opts is NULL");
        if (n_blocks < 1) throw_invalid("n_blocks must be positive");
        require(block_sizes, "block_sizes", true);
        require(channels, "channels", true);
        int64_t total = 0;
        for (int32_t k = 0; k < n_blocks; k++) {
            if (block_sizes[k] < 1) throw_invalid("block " + std::to_string(k) + " is empty");
            total += block_sizes[k];
        }
        if (total != M) throw_invalid("the blocks must name every channel exactly once");
        std::vector<int32_t> ch0((size_t)M);
        std::vector<char> seen((size_t)M, 0);
        for (int64_t j = 0; j < M; j++) {
            const int64_t c = channels[j];
            if (c < 1 || c > M) throw_invalid("channel " + std::to_string(c) + " is outside 1.." + std::to_string(M));
            if (seen[(size_t)(c - 1)]++) throw_invalid("channel " + std::to_string(c) + " is in two blocks");
            ch0[(size_t)j] = (int32_t)(c - 1);
        }
        cudaStream_t s = as_stream(stream);
        const double q = opts->quantization_unit;
        const bool mixed = check_precision(opts->precision);
        const size_t esz = q > 0 ? 2 : 4;
        const size_t in_bytes = sizeof(float) * (size_t)(M * N);
        require(timeseries, "timeseries", in_bytes > 0);
        require(timeseries_out, "timeseries_out", M * N > 0);
        InView in;
        stage_in(in, timeseries, in_bytes, s);
        OutView out;
        out.setup(timeseries_out, esz * (size_t)(M * N), s);
        DevBuf chmap(sizeof(int32_t) * (size_t)M, s);
        MS3_CUDA(cudaMemcpyAsync(chmap.get(), ch0.data(), sizeof(int32_t) * (size_t)M, cudaMemcpyHostToDevice, s));
        DevBuf err(sizeof(int), s);
        MS3_CUDA(cudaMemsetAsync(err.get(), 0, sizeof(int), s));
        int64_t off = 0;
        for (int32_t k = 0; k < n_blocks; k++) {
            const int64_t Mb = block_sizes[k];
            const int32_t* chk = chmap.as<int32_t>() + off;
            DevBuf xb(sizeof(float) * (size_t)(Mb * N), s), yb(esz * (size_t)(Mb * N), s);
            DevBuf mats(sizeof(double) * (size_t)(2 * Mb * Mb), s);
            gather_channels_device(static_cast<const float*>(in.ptr), M, N, chk, Mb, xb.as<float>(), s);
            double* XXt = mats.as<double>();
            double* W = XXt + Mb * Mb;
            covariance_device(xb.as<float>(), Mb, N, XXt, s);
            whitening_matrix_device(XXt, Mb, W, nullptr, nullptr, s);
            apply_whitening_device(xb.as<float>(), Mb, N, W, q, mixed, yb.get(), s, err.as<int>());
            scatter_channels_device(yb.get(), Mb, N, chk, M, out.ptr, esz, s);
            off += Mb;
        }
        out.finish(s);
        int herr = 0;
        MS3_CUDA(cudaMemcpyAsync(&herr, err.get(), sizeof(int), cudaMemcpyDeviceToHost, s));
        MS3_CUDA(cudaStreamSynchronize(s));
        covariance_check_timeout(s);
        if (herr) throw Error(MS3GPU_ERR_CUDA, "tensor-core apply: pipeline wait timed out");
    });
}

int ms3gpu_mask_out_artifacts(const float* timeseries, int64_t M, int64_t N, double threshold,
                              int64_t interval_size, float* timeseries_out, int64_t* timepoints_kept,
                              void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        // p_mask_out_artifacts.cpp:26-29
        if (threshold == 0 || interval_size <= 0)
            throw_invalid("Problem with input parameters. Either threshold or interval_size is zero.");
        cudaStream_t s = as_stream(stream);
        const size_t bytes = sizeof(float) * (size_t)(M * N);
        require(timeseries, "timeseries", bytes > 0);
        require(timeseries_out, "timeseries_out", bytes > 0);
        InView in;
        stage_in(in, timeseries, bytes, s);
        OutView out;
        out.setup(timeseries_out, bytes, s);
        const int64_t kept = mask_out_artifacts_device(static_cast<const float*>(in.ptr), M, N, threshold,
                                                       interval_size, static_cast<float*>(out.ptr), s);
        out.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
        if (timepoints_kept) *timepoints_kept = kept;
    });
}

int ms3gpu_detect_events(const float* timeseries, int64_t M, int64_t N, double detect_threshold,
                         double detect_interval, int32_t detect_sign, int64_t chunk_size, int64_t* counts,
                         int64_t* times, int64_t capacity, void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        require(counts, "counts", M > 0);
        cudaStream_t s = as_stream(stream);
        const size_t bytes = sizeof(float) * (size_t)(M * N);
        require(timeseries, "timeseries", bytes > 0);
        const int64_t chunk = chunk_size > 0 ? chunk_size : detect_chunk_size(M, N, 1);
        InView in;
        stage_in(in, timeseries, bytes, s);
        std::vector<int64_t> c, t;
        detect_events_device(static_cast<const float*>(in.ptr), M, N, detect_threshold, detect_interval, detect_sign,
                             chunk, 1000, c, t, s);
        for (int64_t m = 0; m < M; m++) counts[m] = c[(size_t)m];
        if (!times) return;
        if ((int64_t)t.size() > capacity)
            throw_invalid("times needs " + std::to_string(t.size()) + " entries (capacity " +
                          std::to_string(capacity) + ")");
        std::copy(t.begin(), t.end(), times);
    });
}

int ms3gpu_whiten_clips(const float* clips, int64_t M, int64_t T, int64_t L, const double* W,
                        double quantization_unit, int32_t precision, void* clips_out, void* stream) {
    return guarded(__func__, [&] {
        if (T < 0 || L < 0) throw_invalid("negative dimension");
        if (T > 0 && L > std::numeric_limits<int64_t>::max() / T) throw_invalid("clips too large");
        const int64_t N = T * L;
        check_shape(M, N);
        cudaStream_t s = as_stream(stream);
        const size_t in_bytes = sizeof(float) * (size_t)(M * N);
        const size_t out_bytes = (quantization_unit > 0 ? 2 : 4) * (size_t)(M * N);
        require(clips, "clips", in_bytes > 0);
        require(clips_out, "clips_out", out_bytes > 0);
        require(W, "W", M > 0);
        InView in, w;
        stage_in(in, clips, in_bytes, s);
        stage_in(w, W, sizeof(double) * (size_t)(M * M), s);
        OutView out;
        out.setup(clips_out, out_bytes, s);
        // the clips' timepoints, clip after clip, are one M x (T*L) array
        apply_whitening_device(static_cast<const float*>(in.ptr), M, N, static_cast<const double*>(w.ptr),
                               quantization_unit, check_precision(precision), out.ptr, s, nullptr,
                               /*round_1e4=*/false);
        out.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
    });
}

int ms3gpu_whiten(const float* timeseries, int64_t M, int64_t N, void* timeseries_out,
                  const ms3gpu_whiten_opts* opts, void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        if (!opts) throw_invalid("whiten opts is NULL");
        cudaStream_t s = as_stream(stream);
        const double q = opts->quantization_unit;
        const size_t in_bytes = sizeof(float) * (size_t)(M * N);
        const size_t out_bytes = (q > 0 ? 2 : 4) * (size_t)(M * N);
        require(timeseries, "timeseries", in_bytes > 0);
        require(timeseries_out, "timeseries_out", out_bytes > 0);
        InView in;
        stage_in(in, timeseries, in_bytes, s);
        OutView out;
        out.setup(timeseries_out, out_bytes, s);
        DevBuf mats(sizeof(double) * (size_t)(2 * M * M), s);
        double* XXt = mats.as<double>();
        double* W = XXt + M * M;
        covariance_device(static_cast<const float*>(in.ptr), M, N, XXt, s);
        whitening_matrix_device(XXt, M, W, nullptr, nullptr, s);
        apply_whitening_device(static_cast<const float*>(in.ptr), M, N, W, q, check_precision(opts->precision),
                               out.ptr, s);
        out.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
        covariance_check_timeout(s);
    });
}

int ms3gpu_bandpass_whiten(const float* timeseries, int64_t M, int64_t N, float* filt_out, void* pre_out,
                           const ms3gpu_bandpass_opts* bp, const ms3gpu_whiten_opts* wh, void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        BandpassParams p = to_params(bp);
        if (!wh) throw_invalid("whiten opts is NULL");
        if (p.subsample_factor != 1 || p.quantization_unit != 0)
            throw_invalid("bandpass_whiten needs subsample_factor 1 and quantization_unit 0");
        cudaStream_t s = as_stream(stream);
        const double q = wh->quantization_unit;
        const size_t in_bytes = sizeof(float) * (size_t)(M * N);
        const size_t pre_bytes = (q > 0 ? 2 : 4) * (size_t)(M * N);
        require(timeseries, "timeseries", in_bytes > 0);
        require(pre_out, "pre_out", pre_bytes > 0);
        // host buffers: stream the recording through the device with overlapped copies
        const char* nostream = std::getenv("MS3GPU_NO_STREAMING");
        if (in_bytes > 0 && !is_device_ptr(timeseries) && !is_device_ptr(pre_out) &&
            (!filt_out || !is_device_ptr(filt_out)) && !(nostream && nostream[0] == '1')) {
            bandpass_whiten_streamed(timeseries, M, N, filt_out, pre_out, p, q, check_precision(wh->precision), s);
            return;
        }
        InView in;
        stage_in(in, timeseries, in_bytes, s);
        OutView filt;
        DevBuf filt_own;
        float* filt_d = nullptr;
        bool in_place = false;
        if (filt_out) {
            filt.setup(filt_out, in_bytes, s);
            filt_d = static_cast<float*>(filt.ptr);
        } else {
            filt_d = alloc_filt_or_in_place(in_bytes, q, filt_own, s, in_place);
        }
        OutView pre;
        if (in_place) {  // the filtered signal goes into the output buffer (never the staged input)
            pre.setup(pre_out, pre_bytes, s);
            filt_d = static_cast<float*>(pre.ptr);
        }
        bandpass_device(static_cast<const float*>(in.ptr), M, N, filt_d, p, s);
        // The staged raw input is dead once filtered: the whitened output may reuse it.
        if (!in_place) pre.setup(pre_out, pre_bytes, s, &in.own);
        DevBuf mats(sizeof(double) * (size_t)(2 * M * M), s);
        double* XXt = mats.as<double>();
        double* W = XXt + M * M;
        covariance_device(filt_d, M, N, XXt, s);
        whitening_matrix_device(XXt, M, W, nullptr, nullptr, s);
        apply_maybe_in_place(filt_d, in_place, M, N, W, q, check_precision(wh->precision), pre.ptr, s, nullptr);
        if (filt_out) filt.finish(s);
        pre.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
        bandpass_check_timeout(s);
        covariance_check_timeout(s);
    });
}

int ms3gpu_bandpass_filter_windows(const void* timeseries, int32_t in_dtype, int64_t M, int64_t N, int64_t row0,
                                   int64_t rows, int64_t c_begin, int64_t c_end, void* timeseries_out,
                                   int64_t out_row0, int64_t out_rows, const ms3gpu_bandpass_opts* opts,
                                   void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        BandpassParams p = to_params(opts);
        if (in_dtype != MS3GPU_DTYPE_FLOAT32 && in_dtype != MS3GPU_DTYPE_INT16)
            throw_invalid("in_dtype must be MS3GPU_DTYPE_FLOAT32 or MS3GPU_DTYPE_INT16");
        if (p.freq_max == 0) throw_invalid("freq_max 0 copies whole recordings: use ms3gpu_bandpass_filter");
        const int64_t chunk = bandpass_chunk_size(M, p.num_threads);
        const int64_t nchunks = N > 0 ? ceil_div(N, chunk) : 0;
        if (c_begin < 0 || c_end > nchunks || c_begin > c_end)
            throw_invalid("windows [" + std::to_string(c_begin) + ", " + std::to_string(c_end) + ") outside [0, " +
                          std::to_string(nchunks) + ")");
        if (c_begin == c_end || M == 0) return;
        const int sub = p.subsample_factor;
        const int64_t need0 = std::max<int64_t>(0, c_begin * chunk - 60000);
        const int64_t need1 = std::min<int64_t>(N, c_end * chunk + 60000);
        if (row0 < 0 || rows < 0 || row0 > need0 || row0 + rows < need1)
            throw_invalid("input rows [" + std::to_string(row0) + ", " + std::to_string(row0 + rows) +
                          ") do not hold the windows' rows [" + std::to_string(need0) + ", " +
                          std::to_string(need1) + ")");
        int64_t o0 = 0, o1 = 0;
        bandpass_output_rows(N, chunk, sub, c_begin, c_end, o0, o1);
        if (out_row0 < 0 || out_rows < 0 || out_row0 > o0 || out_row0 + out_rows < o1)
            throw_invalid("output rows [" + std::to_string(out_row0) + ", " + std::to_string(out_row0 + out_rows) +
                          ") do not hold the windows' output rows [" + std::to_string(o0) + ", " +
                          std::to_string(o1) + ")");
        const bool in_i16 = in_dtype == MS3GPU_DTYPE_INT16;
        const size_t in_bytes = (in_i16 ? 2 : 4) * (size_t)(rows * M);
        const size_t out_bytes = (p.quantization_unit != 0 ? 2 : 4) * (size_t)(out_rows * M);
        require(timeseries, "timeseries", in_bytes > 0);
        require(timeseries_out, "timeseries_out", out_bytes > 0);
        cudaStream_t s = as_stream(stream);
        InView in;
        stage_in(in, timeseries, in_bytes, s);
        OutView out;
        out.setup(timeseries_out, out_bytes, s);
        // rows of the output buffer outside the windows' rows keep what the caller had there
        if (out.host && out_bytes) MS3_CUDA(cudaMemcpyAsync(out.ptr, timeseries_out, out_bytes, cudaMemcpyHostToDevice, s));
        bandpass_device(in.ptr, M, N, out.ptr, p, s, c_begin, c_end, in_i16, row0, out_row0);
        out.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
        bandpass_check_timeout(s);
    });
}

int ms3gpu_whiten_covariance_sum(const float* timeseries, int64_t M, int64_t N, double* XXt_sum, void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        require(XXt_sum, "XXt_sum", M > 0);
        cudaStream_t s = as_stream(stream);
        const size_t in_bytes = sizeof(float) * (size_t)(M * N);
        require(timeseries, "timeseries", in_bytes > 0);
        if (M == 0) return;
        InView in;
        stage_in(in, timeseries, in_bytes, s);
        OutView out;
        out.setup(XXt_sum, sizeof(double) * (size_t)(M * M), s);
        if (N == 0)
            MS3_CUDA(cudaMemsetAsync(out.ptr, 0, sizeof(double) * (size_t)(M * M), s));
        else
            covariance_sum_device(static_cast<const float*>(in.ptr), M, N, static_cast<double*>(out.ptr), s);
        out.finish(s);
        MS3_CUDA(cudaStreamSynchronize(s));
        covariance_check_timeout(s);
    });
}

namespace {
void check_stream_io(const ms3gpu_stream_io* io, bool needs_write) {
    if (!io) throw_invalid("stream io is NULL");
    if (!io->read) throw_invalid("stream io has no read callback");
    if (needs_write && !io->write) throw_invalid("stream io has no write callback");
    if (io->slab_bytes < 0) throw_invalid("slab_bytes must be >= 0");
}
}  // namespace

int ms3gpu_bandpass_filter_stream(int64_t M, int64_t N, int32_t in_dtype, const ms3gpu_stream_io* io,
                                  const ms3gpu_bandpass_opts* opts, void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        BandpassParams p = to_params(opts);
        check_stream_io(io, true);
        if (in_dtype != MS3GPU_DTYPE_FLOAT32 && in_dtype != MS3GPU_DTYPE_INT16)
            throw_invalid("in_dtype must be MS3GPU_DTYPE_FLOAT32 or MS3GPU_DTYPE_INT16");
        bandpass_stream(M, N, in_dtype == MS3GPU_DTYPE_INT16, *io, p, as_stream(stream));
    });
}

int ms3gpu_mask_out_artifacts_stream(int64_t M, int64_t N, double threshold, int64_t interval_size,
                                     const ms3gpu_stream_io* io, int64_t* timepoints_kept, void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        if (threshold == 0 || interval_size <= 0)
            throw_invalid("Problem with input parameters. Either threshold or interval_size is zero.");
        check_stream_io(io, true);
        const int64_t kept = mask_out_artifacts_stream(M, N, threshold, interval_size, *io, as_stream(stream));
        if (timepoints_kept) *timepoints_kept = kept;
    });
}

int ms3gpu_whiten_stream(int64_t M, int64_t N, const ms3gpu_stream_io* io, const ms3gpu_whiten_opts* opts,
                         void* stream) {
    return guarded(__func__, [&] {
        check_shape(M, N);
        if (!opts) throw_invalid("whiten opts is NULL");
        check_stream_io(io, true);
        whiten_stream(M, N, *io, opts->quantization_unit, check_precision(opts->precision), as_stream(stream));
    });
}

}  // extern "C"
