// Internal helpers shared by the ms3gpu CUDA sources.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <stdexcept>
#include <string>

namespace ms3gpu {

// Error carried from the implementation to the C ABI boundary, where it is
// turned into a status code and the per-thread last-error text.
struct Error : public std::runtime_error {
    int code;
    Error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

[[noreturn]] void throw_cuda(cudaError_t e, const char* what, const char* file, int line);
[[noreturn]] void throw_invalid(const std::string& msg);
[[noreturn]] void throw_unsupported(const std::string& msg);

#define MS3_CUDA(x)                                                              \
    do {                                                                         \
        cudaError_t e_ = (x);                                                    \
        if (e_ != cudaSuccess) ::ms3gpu::throw_cuda(e_, #x, __FILE__, __LINE__); \
    } while (0)

// Kernel launches issued by this library (reported by ms3gpu_launch_count).
void count_launch();

// Checks the launch just issued (configuration errors surface here) and
// counts it.
#define MS3_LAUNCH_CHECK()                \
    do {                                  \
        MS3_CUDA(cudaGetLastError());     \
        ::ms3gpu::count_launch();         \
    } while (0)

// Index checks of the bounds-checked build (-DMS3GPU_BOUNDS_CHECK, built as
// libms3gpu_checked.so beside libms3gpu.so by mountainsort_b200.build and
// loaded by the Python binding when MS3GPU_LIBRARY=checked):
// MS3_IN_BOUNDS(i, n, site) is true when 0 <= i < n; otherwise it records
// the first failing site in its translation unit's bounds word and is false,
// and the caller skips the access, so a wrong index becomes an error status
// (MS3GPU_ERR_CUDA, "bounds check failed at site ...") instead of a fault.
// In the ordinary build it is the constant true and costs nothing.
#ifdef MS3GPU_BOUNDS_CHECK
static __device__ int g_bounds_site;  // one per translation unit (no relocatable device code)
__device__ __forceinline__ bool bounds_ok(int64_t i, int64_t n, int site) {
    if ((uint64_t)i < (uint64_t)n) return true;
    atomicCAS(&g_bounds_site, 0, site);
    return false;
}
// The translation unit's recorded site (0: none), cleared; synchronizes `s`.
static inline int take_bounds_site(cudaStream_t s) {
    int h = 0;
    if (cudaMemcpyFromSymbolAsync(&h, g_bounds_site, sizeof(int), 0, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return -1;
    if (h) {
        const int zero = 0;
        cudaMemcpyToSymbolAsync(g_bounds_site, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s);
        cudaStreamSynchronize(s);
    }
    return h;
}
#define MS3_IN_BOUNDS(i, n, site) ::ms3gpu::bounds_ok((int64_t)(i), (int64_t)(n), (site))
#else
#define MS3_IN_BOUNDS(i, n, site) true
#endif
// Per translation unit of the library: its recorded bounds-check site, cleared
// (0 in the ordinary build).
int bounds_site_bandpass(cudaStream_t s);
int bounds_site_whiten(cudaStream_t s);
int bounds_site_apply(cudaStream_t s);
int bounds_site_cov(cudaStream_t s);

// Stream-ordered device allocation owned by one call.  Freed on the same
// stream when it goes out of scope, so later work on the stream may not use it.
class DevBuf {
public:
    DevBuf() = default;
    DevBuf(size_t bytes, cudaStream_t s) { alloc(bytes, s); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p_(o.p_), n_(o.n_), s_(o.s_) { o.p_ = nullptr; o.n_ = 0; }
    void alloc(size_t bytes, cudaStream_t s);
    void release();
    template <class T>
    T* as() const { return static_cast<T*>(p_); }
    void* get() const { return p_; }
    size_t size() const { return n_; }

private:
    void* p_ = nullptr;
    size_t n_ = 0;
    cudaStream_t s_ = nullptr;
};

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// float -> int16 exactly as the reference's writer converts (std::copy on
// x86-64, packages/ms3/mda/mdaio.cpp:232-243): truncation to int32 with
// 0x80000000 for NaN / out-of-range values, low 16 bits stored.
__host__ __device__ inline int16_t x86_float_to_int16(float v) {
    int32_t i;
    if (!(v > -2147483648.0f && v < 2147483648.0f))
        i = INT32_MIN;
    else
        i = (int32_t)v;
    return (int16_t)(uint16_t)(uint32_t)i;
}

// (int)(d) for a double as cvttsd2si does it (0x80000000 when out of range).
__host__ __device__ inline int32_t x86_double_to_int32(double d) {
    if (!(d > -2147483649.0 && d < 2147483648.0)) return INT32_MIN;
    return (int32_t)d;
}

}  // namespace ms3gpu
