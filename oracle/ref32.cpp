// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// A Qt-free CPU restatement of the reference's ms3.bandpass_filter and
// ms3.whiten processors ("ref32").  It is the parity checker for the CUDA
// library and the timed CPU baseline; the product never links or calls it.
// Only tests/, __graft_entry__.smoke() and bench.py (cpu baseline / reference
// arm) load it.
//
// Every function follows the reference's arithmetic step by step: the same
// chunk geometry, the same float/double choices, the same loop orders and the
// same OpenMP work split.  Citations are paths inside the reference project.
// Parity status: the reference cannot be compiled here (it needs Qt5 and
// FFTW3f) and its tests hold no golden vectors for this path, so the numeric
// part of this restatement is "parity unpinned"; the .mda format it shares is
// pinned against files written by the reference's own Python writer.
//
// Compiled with -ffp-contract=off so that no multiply-add is fused: the
// reference is built for plain x86-64 SSE2, where float*float rounds to
// float and float += double rounds through double.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <omp.h>

#include "fft_ref.hpp"

using ms3ref::BatchedFft;

// float -> int16 as the reference's std::copy compiles on x86-64
// (mda/mdaio.cpp:232-243): cvttss2si to int32 (0x80000000 for NaN and
// out-of-range values), then the low 16 bits are stored.
static inline int16_t x86_float_to_int16(float v) {
    int32_t i;
    if (!(v > -2147483648.0f && v < 2147483648.0f))
        i = INT32_MIN;
    else
        i = (int32_t)v;
    return (int16_t)(uint16_t)(uint32_t)i;
}

extern "C" {

int16_t ref32_float_to_int16(float v) { return x86_float_to_int16(v); }

// packages/ms3/p_bandpass_filter.cpp:421-447 (define_kernel)
void ref32_define_kernel(int64_t N, double* kernel, double samplefreq, double freq_min,
                         double freq_max, double freq_wid) {
    double T = N / samplefreq;
    double df = 1 / T;
    double relwid = 3.0;
    for (int64_t i = 0; i < N; i++) {
        const double fgrid = (i <= (N + 1) / 2) ? df * i : df * (i - N);
        const double absf = std::fabs(fgrid);
        double val = 1.0;
        if (freq_min != 0) {
            if (i == 0)
                val = 0.0;
            else
                val *= (1 + std::erf(relwid * (absf - freq_min) / freq_min)) / 2;
        }
        if (freq_max != 0) {
            val *= (1 - std::erf((absf - freq_max) / freq_wid)) / 2;
        }
        kernel[i] = std::sqrt(val);
    }
}

// packages/ms3/p_bandpass_filter.cpp:147-155 (chunk geometry; T is
// omp_get_max_threads() in the reference)
int64_t ref32_bandpass_chunk_size(int64_t M, int64_t num_threads) {
    int overhead = 6;
    int64_t overlap_size = 60000;
    int64_t min_chunk_size = overlap_size * 2;
    double target_ram_bytes = 1.0 * (1024 * 1024 * 1024);
    double target_chunk_size =
        target_ram_bytes / (overhead * sizeof(float) * M * num_threads) - 2 * overlap_size;
    int64_t chunk_size = (int64_t)(target_chunk_size);
    if (chunk_size < min_chunk_size) chunk_size = min_chunk_size;
    return chunk_size;
}

// packages/ms3/p_bandpass_filter.cpp:157-158
double ref32_bandpass_peak_ram_mb(int64_t M, int64_t num_threads) {
    int overhead = 6;
    int64_t chunk_size = ref32_bandpass_chunk_size(M, num_threads);
    double expected_ram_bytes = overhead * sizeof(float) * M * num_threads * (chunk_size + 2 * 60000);
    return expected_ram_bytes / (1024 * 1024);
}

// packages/ms3/p_whiten.cpp:53-57
double ref32_whiten_peak_ram_mb(int64_t M) {
    int64_t processing_chunk_size = 100000;
    int overhead = 3;
    double expected_peak_ram_bytes = overhead * processing_chunk_size * M * sizeof(float);
    return expected_peak_ram_bytes / (1024 * 1024);
}

// Test hook: batched FFT of `howmany` interleaved complex signals.
int ref32_fft(float* data, int64_t L, int64_t howmany, int sign) {
    try {
        BatchedFft f(L, sign);
        std::vector<float> work((size_t)(2 * L * howmany));
        f.execute(data, work.data(), howmany);
    } catch (...) {
        return -1;
    }
    return 0;
}

// ms3.bandpass_filter on an in-memory M x N timeseries (element (m,t) at
// X[m + M t]).  Follows packages/ms3/p_bandpass_filter.cpp:115-229 with
// Kernel_runner::init/apply (:34-110), multiply_by_factor (:233-248) and
// subsample (:480-491).
//   geometry_threads: the T of the chunk-size formula (omp_get_max_threads()
//                     in the reference, or --_request_num_threads)
//   exec_threads:     OpenMP threads actually used here (0 = default)
// Output: M x (N / subsample_factor).  When quantization_unit != 0 the values
// are the float chunk after multiply_by_factor and, if out_i16 is given, the
// int16 file content (std::copy truncation, mda/mdaio.cpp:232-243).
// Returns 0 on success.
int ref32_bandpass_filter(const float* X, int64_t M, int64_t Naa, double samplerate,
                          double freq_min, double freq_max, double freq_wid,
                          double quantization_unit, int subsample_factor,
                          int64_t geometry_threads, int exec_threads, float* out_f32,
                          int16_t* out_i16) {
    if (subsample_factor == 0) subsample_factor = 1;
    const int64_t N2 = Naa / subsample_factor;
    if (freq_max == 0) {  // :117-119 -- the file is copied unchanged
        if (out_f32) std::memcpy(out_f32, X, sizeof(float) * M * Naa);
        return 0;
    }
    const int64_t overlap_size = 60000;
    const int64_t chunk_size = ref32_bandpass_chunk_size(M, geometry_threads);
    const int64_t L = chunk_size + 2 * overlap_size;
    const int64_t MN = M * L;

    std::vector<double> kernel0((size_t)L);
    ref32_define_kernel(L, kernel0.data(), samplerate, freq_min, freq_max, freq_wid);

    if (exec_threads > 0) omp_set_num_threads(exec_threads);
    BatchedFft fwd(L, -1), inv(L, +1);
    int ret = 0;
    const int64_t nchunks = (Naa + chunk_size - 1) / chunk_size;
#pragma omp parallel
    {
        std::vector<float> buf((size_t)(2 * MN)), work((size_t)(2 * MN));
        std::vector<float> chunk2;
#pragma omp for schedule(static)
        for (int64_t c = 0; c < nchunks; c++) {
            const int64_t timepoint = c * chunk_size;
            // DiskReadMda32::readChunk zero-fills outside [0, N)
            // (mda/diskreadmda32.cpp:615-661)
            const int64_t t0 = timepoint - overlap_size;
            for (int64_t i = 0; i < L; i++) {
                const int64_t t = t0 + i;
                float* dst = &buf[(size_t)(i * M * 2)];
                if (t < 0 || t >= Naa) {
                    for (int64_t m = 0; m < M; m++) { dst[2 * m] = 0.f; dst[2 * m + 1] = 0.f; }
                } else {
                    const float* src = X + t * M;
                    for (int64_t m = 0; m < M; m++) { dst[2 * m] = src[m]; dst[2 * m + 1] = 0.f; }
                }
            }
            fwd.execute(buf.data(), work.data(), M);
            // data_out[aa] *= kernel0[i] * factor   (float *= double)
            const double factor = 1.0 / L;
            for (int64_t i = 0; i < L; i++) {
                const double kf = kernel0[(size_t)i] * factor;
                float* row = &buf[(size_t)(i * M * 2)];
                for (int64_t m = 0; m < 2 * M; m++) row[m] = (float)((double)row[m] * kf);
            }
            inv.execute(buf.data(), work.data(), M);
            // getChunk(chunk2, 0, overlap_size, M, chunk_size) then subsample /
            // quantize / writeChunk truncated at the end of the file.
            const int64_t nsub = chunk_size / subsample_factor;
            const int64_t out_t0 = timepoint / subsample_factor;
            for (int64_t j = 0; j < nsub; j++) {
                const int64_t ot = out_t0 + j;
                if (ot >= N2) break;
                const int64_t src_i = overlap_size + j * subsample_factor;
                const float* src = &buf[(size_t)(src_i * M * 2)];
                for (int64_t m = 0; m < M; m++) {
                    float v = src[2 * m];
                    if (quantization_unit) v = (float)((double)v * (1.0 / quantization_unit));
                    if (out_f32) out_f32[ot * M + m] = v;
                    if (out_i16) out_i16[ot * M + m] = x86_float_to_int16(v);
                }
            }
        }
    }
    return ret;
}

// ms3.whiten pass 1: XXt = sum_t x_t x_t^T with float products accumulated
// in double per 1e5-timepoint chunk, chunk sums added into the total, then
// divided by N-1 when N > 1 (packages/ms3/p_whiten.cpp:64-118).  Chunks are
// added in index order (the reference adds them in completion order).
void ref32_whiten_xxt(const float* X, int64_t M, int64_t N, int exec_threads, double* XXt) {
    int64_t chunk_size = 100000;
    if (N < chunk_size) chunk_size = N;
    std::fill(XXt, XXt + M * M, 0.0);
    if (N == 0) return;
    const int64_t nchunks = (N + chunk_size - 1) / chunk_size;
    std::vector<double> parts((size_t)(nchunks * M * M), 0.0);
    if (exec_threads > 0) omp_set_num_threads(exec_threads);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; c++) {
        const int64_t timepoint = c * chunk_size;
        const int64_t n = std::min(chunk_size, N - timepoint);
        const float* chunkptr = X + timepoint * M;
        double* XXt0ptr = &parts[(size_t)(c * M * M)];
        for (int64_t i = 0; i < n; i++) {
            int64_t aa = M * i;
            int64_t bb = 0;
            for (int64_t m1 = 0; m1 < M; m1++) {
                for (int64_t m2 = 0; m2 < M; m2++) {
                    float prod = chunkptr[aa + m1] * chunkptr[aa + m2];
                    XXt0ptr[bb] += prod;
                    bb++;
                }
            }
        }
    }
    for (int64_t c = 0; c < nchunks; c++)
        for (int64_t bb = 0; bb < M * M; bb++) XXt[bb] += parts[(size_t)(c * M * M + bb)];
    if (N > 1)
        for (int64_t ii = 0; ii < M * M; ii++) XXt[ii] /= (N - 1);
}

// --- packages/ms3/pca.cpp, double-precision overloads -----------------------

// common/mlcompute.cpp:131-139 (norm = sqrt(inner_product))
static double ml_norm(int64_t N, const double* X) {
    double s = 0.0;
    for (int64_t i = 0; i < N; i++) s = s + X[i] * X[i];
    return std::sqrt(s);
}

// pca.cpp:457-466
static void normalize_vector(std::vector<double>& V) {
    double norm = ml_norm((int64_t)V.size(), V.data());
    if (!norm) return;
    for (double& v : V) v /= norm;
}

// pca.cpp:479-491
static void matvec(int64_t M, int64_t N, double* ret, const double* A, const double* x) {
    for (int64_t m = 0; m < M; m++) ret[m] = 0;
    int64_t iA = 0;
    for (int64_t n = 0; n < N; n++) {
        double xval = x[n];
        for (int64_t m = 0; m < M; m++) {
            ret[m] += A[iA] * xval;
            iA++;
        }
    }
}

// pca.cpp:220-243 (A is M x L, B is L x N, column-major)
static std::vector<double> mult_AB(const std::vector<double>& A, const std::vector<double>& B,
                                   int64_t M, int64_t L, int64_t N) {
    std::vector<double> C((size_t)(M * N), 0.0);
    int64_t iC = 0;
    for (int64_t n = 0; n < N; n++) {
        for (int64_t m = 0; m < M; m++) {
            double acc = 0.0;
            for (int64_t l = 0; l < L; l++) acc += A[(size_t)(m + l * M)] * B[(size_t)(l + L * n)];
            C[(size_t)iC] += acc;
            iC++;
        }
    }
    return C;
}

// pca.cpp:319-342 (A is M x L, B is N x L)
static std::vector<double> mult_ABtrans(const std::vector<double>& A, const std::vector<double>& B,
                                        int64_t M, int64_t L, int64_t N) {
    std::vector<double> C((size_t)(M * N), 0.0);
    int64_t iC = 0;
    for (int64_t n = 0; n < N; n++) {
        for (int64_t m = 0; m < M; m++) {
            double acc = 0.0;
            for (int64_t l = 0; l < L; l++) acc += A[(size_t)(m + l * M)] * B[(size_t)(n + l * N)];
            C[(size_t)iC] += acc;
            iC++;
        }
    }
    return C;
}

// pca.cpp:542-558
static void iterate_XXt_to_get_top_component(std::vector<double>& C, double& sigma,
                                             const std::vector<double>& XXt, int64_t M,
                                             int64_t num_iterations) {
    C.assign((size_t)M, 0.0);
    for (int64_t i = 0; i < M; i++) C[(size_t)i] = std::sin((double)(i + 1));
    normalize_vector(C);
    std::vector<double> tmp((size_t)M);
    for (int64_t it = 0; it < num_iterations; it++) {
        matvec(M, M, tmp.data(), XXt.data(), C.data());
        C = tmp;
        sigma = ml_norm(M, C.data());
        normalize_vector(C);
    }
}

// pca.cpp:409-431 (XXt <- (I - CC') XXt (I - CC'))
static void subtract_out_rank_1_from_XXt(std::vector<double>& XXt, const std::vector<double>& C,
                                         int64_t M) {
    std::vector<double> B((size_t)(M * M));
    for (int64_t j = 0; j < M; j++)
        for (int64_t i = 0; i < M; i++)
            B[(size_t)(i + M * j)] = (i == j) ? 1 - C[(size_t)i] * C[(size_t)j] : -C[(size_t)i] * C[(size_t)j];
    std::vector<double> tmp = mult_AB(XXt, B, M, M, M);
    XXt = mult_AB(B, tmp, M, M, M);
}

// pca.cpp:172-195 (pca_from_XXt, 10 iterations per component) and
// pca.cpp:635-651 (whitening_matrix_from_XXt: W = (C D) C', D = diag(1/sqrt(sigma)),
// 0 where sigma == 0).  Also returns the components and sigmas when asked.
void ref32_whitening_matrix(const double* XXt_in, int64_t M, double* W_out, double* comps_out,
                            double* sigma_out) {
    const int64_t K = M;
    const int64_t num_iterations_per_component = 10;
    std::vector<double> XXtw(XXt_in, XXt_in + M * M);
    std::vector<double> C((size_t)(M * K), 0.0), sigma((size_t)K, 0.0);
    for (int64_t k = 0; k < K; k++) {
        std::vector<double> C0;
        double sigma0 = 0;
        iterate_XXt_to_get_top_component(C0, sigma0, XXtw, M, num_iterations_per_component);
        for (int64_t m = 0; m < M; m++) C[(size_t)(m + M * k)] = C0[(size_t)m];
        sigma[(size_t)k] = sigma0;
        subtract_out_rank_1_from_XXt(XXtw, C0, M);
    }
    std::vector<double> D((size_t)(M * M), 0.0);
    for (int64_t i = 0; i < M; i++) {
        double val = 0;
        if (sigma[(size_t)i]) val = 1 / std::sqrt(sigma[(size_t)i]);
        D[(size_t)(i + M * i)] = val;
    }
    std::vector<double> tmp = mult_AB(C, D, M, M, M);
    std::vector<double> W = mult_ABtrans(tmp, C, M, M, M);
    std::memcpy(W_out, W.data(), sizeof(double) * M * M);
    if (comps_out) std::memcpy(comps_out, C.data(), sizeof(double) * M * M);
    if (sigma_out) std::memcpy(sigma_out, sigma.data(), sizeof(double) * M);
}

// ms3.whiten pass 2 (packages/ms3/p_whiten.cpp:153-206): out[m1] += in[m2] *
// W[m1*M + m2] accumulated in float (each += rounds through double), then
// quantize(x, 1e-4) = floor(x/1e-4 + 0.5)*1e-4 (:31-41) and, when
// quantization_unit > 0, scale_for_quantization (:445-451).
void ref32_whiten_apply(const float* X, int64_t M, int64_t N, const double* WW,
                        double quantization_unit, int exec_threads, float* out) {
    int64_t chunk_size = 100000;
    if (N < chunk_size) chunk_size = N;
    if (N == 0) return;
    const int64_t nchunks = (N + chunk_size - 1) / chunk_size;
    if (exec_threads > 0) omp_set_num_threads(exec_threads);
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < nchunks; c++) {
        const int64_t timepoint = c * chunk_size;
        const int64_t n = std::min(chunk_size, N - timepoint);
        const float* chunk_in_ptr = X + timepoint * M;
        float* chunk_out_ptr = out + timepoint * M;
        for (int64_t i = 0; i < n * M; i++) chunk_out_ptr[i] = 0.f;
        for (int64_t i = 0; i < n; i++) {
            int64_t aa = M * i;
            int64_t bb = 0;
            for (int64_t m1 = 0; m1 < M; m1++) {
                for (int64_t m2 = 0; m2 < M; m2++) {
                    chunk_out_ptr[aa + m1] =
                        (float)((double)chunk_out_ptr[aa + m1] + (double)chunk_in_ptr[aa + m2] * WW[bb]);
                    bb++;
                }
            }
        }
        for (int64_t i = 0; i < n * M; i++) {
            float x = chunk_out_ptr[i];
            x = (float)(std::floor(x / 0.0001 + 0.5) * 0.0001);
            if (quantization_unit > 0) {
                // (int)(x/q + 0.5): cvttsd2si, 0x80000000 when out of range
                double v = (x / quantization_unit) + 0.5;
                int iv = (v > -2147483649.0 && v < 2147483648.0) ? (int)v : INT32_MIN;
                x = (float)iv;
            }
            chunk_out_ptr[i] = x;
        }
    }
}

// ms3.compute_whitening_matrix (packages/ms3/p_whiten.cpp:208-298): the
// recordings Xs[0..n_inputs) (each M x Ns[i], column-major) read as one
// array concatenated in time (DiskReadMda32 over a file list), in chunks of
// 1e7 timepoints (the last chunk shorter); each chunk restricted to
// `channels` (1-based, :421-433) when n_channels > 0, float products summed in
// a per-chunk double M2 x M2 matrix, chunk matrices added in index order (the
// reference adds them in completion order), divided by N-1 when N > 1; then
// whitening_matrix_from_XXt.  Returns -1 for a channel outside [1, M].
int ref32_compute_whitening_matrix(const float* const* Xs, const int64_t* Ns, int n_inputs, int64_t M,
                                   const int32_t* channels, int n_channels, double* W_out, double* XXt_out) {
    const int64_t M2 = n_channels > 0 ? n_channels : M;
    std::vector<int64_t> ch((size_t)M2);
    for (int64_t j = 0; j < M2; j++) {
        ch[(size_t)j] = n_channels > 0 ? (int64_t)channels[j] - 1 : j;
        if (ch[(size_t)j] < 0 || ch[(size_t)j] >= M) return -1;
    }
    int64_t N = 0;
    for (int i = 0; i < n_inputs; i++) N += Ns[i];
    // timepoint t of the concatenation -> (input, row)
    std::vector<int64_t> start((size_t)n_inputs + 1, 0);
    for (int i = 0; i < n_inputs; i++) start[(size_t)i + 1] = start[(size_t)i] + Ns[i];
    auto row = [&](int64_t t) -> const float* {
        int i = 0;
        while (t >= start[(size_t)i + 1]) i++;
        return Xs[i] + (t - start[(size_t)i]) * M;
    };
    const int64_t processing_chunk_size = 10000000;
    const int64_t chunk_size = N < processing_chunk_size ? N : processing_chunk_size;
    std::vector<double> XXt((size_t)(M2 * M2), 0.0), XXt0((size_t)(M2 * M2));
    std::vector<float> x((size_t)M2);
    for (int64_t timepoint = 0; timepoint < N; timepoint += chunk_size) {
        const int64_t n = std::min(chunk_size, N - timepoint);
        std::fill(XXt0.begin(), XXt0.end(), 0.0);
        for (int64_t i = 0; i < n; i++) {
            const float* r = row(timepoint + i);
            for (int64_t j = 0; j < M2; j++) x[(size_t)j] = r[ch[(size_t)j]];
            int64_t bb = 0;
            for (int64_t m1 = 0; m1 < M2; m1++) {
                for (int64_t m2 = 0; m2 < M2; m2++) {
                    float prod = x[(size_t)m1] * x[(size_t)m2];
                    XXt0[(size_t)bb] += prod;
                    bb++;
                }
            }
        }
        for (int64_t bb = 0; bb < M2 * M2; bb++) XXt[(size_t)bb] += XXt0[(size_t)bb];
    }
    if (N > 1)
        for (int64_t ii = 0; ii < M2 * M2; ii++) XXt[(size_t)ii] /= (N - 1);
    ref32_whitening_matrix(XXt.data(), M2, W_out, nullptr, nullptr);
    if (XXt_out) std::memcpy(XXt_out, XXt.data(), sizeof(double) * (size_t)(M2 * M2));
    return 0;
}

// ms3.whiten_clips (packages/ms3/p_whiten.cpp:300-345): clips M x T x L; for
// each clip and timepoint out(m1) += x(m2) * WW[m1*M + m2] in float (the same
// accumulation as the apply), no 1e-4 rounding (commented out there, :336-341),
// then scale_for_quantization when quantization_unit > 0 (:445-451).
void ref32_whiten_clips(const float* clips, int64_t M, int64_t T, int64_t L, const double* WW,
                        double quantization_unit, float* out) {
    for (int64_t i = 0; i < L; i++) {
        const float* chunk_ptr = clips + i * M * T;
        float* chunk_out_ptr = out + i * M * T;
        for (int64_t k = 0; k < M * T; k++) chunk_out_ptr[k] = 0.f;
        for (int64_t t = 0; t < T; t++) {
            int64_t aa = 0;
            const int64_t bb = M * t;
            for (int64_t m1 = 0; m1 < M; m1++) {
                for (int64_t m2 = 0; m2 < M; m2++) {
                    chunk_out_ptr[bb + m1] =
                        (float)((double)chunk_out_ptr[bb + m1] + (double)chunk_ptr[bb + m2] * WW[aa]);
                    aa++;
                }
            }
        }
        if (quantization_unit > 0) {
            for (int64_t k = 0; k < M * T; k++) {
                double v = (chunk_out_ptr[k] / quantization_unit) + 0.5;
                int iv = (v > -2147483649.0 && v < 2147483648.0) ? (int)v : INT32_MIN;
                chunk_out_ptr[k] = (float)iv;
            }
        }
    }
}

// ms3.mask_out_artifacts (packages/ms3/p_mask_out_artifacts.cpp:24-104) on
// an M x N column-major float32 timeseries: interval norms in double (the
// reader delivers doubles), MLCompute::mean / stdev (common/mlcompute.cpp:
// 67-85), flagged intervals masked with their neighbours (the reference's
// write to use_it[-1] for interval 0 is out of bounds and dropped here),
// output zero on masked intervals and after the last whole interval.
// Returns the number of timepoints kept, or -1 for a zero threshold or
// interval size (the reference returns false).
int64_t ref32_mask_out_artifacts(const float* X, int64_t M, int64_t N, double threshold, int64_t interval_size,
                                 float* out) {
    if (!threshold || !interval_size) return -1;
    const int64_t I = interval_size, nint = N / I;
    std::vector<double> norms((size_t)(M * nint));
    for (int64_t i = 0; i < nint; i++) {
        for (int64_t m = 0; m < M; m++) {
            double sumsqr = 0;
            for (int64_t aa = 0; aa < I; aa++) {
                const double v = X[(i * I + aa) * M + m];
                sumsqr += v * v;
            }
            norms[(size_t)(m + M * i)] = std::sqrt(sumsqr);
        }
    }
    std::vector<int> use_it((size_t)(nint + 1), 1);
    for (int64_t m = 0; m < M; m++) {
        double sum = 0, sumsqr = 0;
        for (int64_t i = 0; i < nint; i++) {
            const double v = norms[(size_t)(m + M * i)];
            sum = sum + v;
            sumsqr = sumsqr + v * v;
        }
        const double mean0 = nint ? sum / nint : 0;
        const double sigma0 = nint >= 2 ? std::sqrt((sumsqr - sum * sum / nint) / (nint - 1)) : 0;
        for (int64_t i = 0; i < nint; i++) {
            if (norms[(size_t)(m + M * i)] > mean0 + sigma0 * threshold) {
                if (i >= 1) use_it[(size_t)(i - 1)] = 0;
                use_it[(size_t)i] = 0;
                use_it[(size_t)(i + 1)] = 0;
            }
        }
    }
    std::fill(out, out + M * N, 0.f);
    int64_t kept = 0;
    for (int64_t i = 0; i < nint; i++) {
        if (!use_it[(size_t)i]) continue;
        kept += I;
        std::memcpy(out + i * I * M, X + i * I * M, sizeof(float) * (size_t)(I * M));
    }
    return kept;
}

// mountainsortalg's detect_events (detect_events.cpp:69-135) on one vector.
static std::vector<int64_t> detect_events_vec(const std::vector<double>& X, double detect_threshold,
                                              double detect_interval, int sign) {
    const int64_t ct = (int64_t)X.size();
    double sum = 0, sumsqr = 0;
    for (double v : X) sum = sum + v;
    for (double v : X) sumsqr = sumsqr + v * v;
    const double mean = ct ? sum / ct : 0;
    const double stdev = ct >= 2 ? std::sqrt((sumsqr - sum * sum / ct) / (ct - 1)) : 0;
    const double threshold2 = detect_threshold * stdev;
    std::vector<int64_t> tc;
    std::vector<double> vc;
    for (int64_t n = 0; n < ct; n++) {
        double val = X[(size_t)n] - mean;
        if (sign < 0)
            val = -val;
        else if (sign == 0)
            val = std::fabs(val);
        if (val > threshold2) {
            tc.push_back(n);
            vc.push_back(val);
        }
    }
    std::vector<char> to_use(tc.size(), 0);
    int64_t last_best_ind = -1;
    for (int64_t i = 0; i < (int64_t)tc.size(); i++) {
        if (last_best_ind >= 0) {
            if (tc[(size_t)last_best_ind] < tc[(size_t)i] - detect_interval) {
                last_best_ind = -1;
                if ((i > 0) && (tc[(size_t)i - 1] >= tc[(size_t)i] - detect_interval)) {
                    last_best_ind = i - 1;
                    int64_t jj = last_best_ind;
                    while ((jj - 1 >= 0) && (tc[(size_t)jj - 1] >= tc[(size_t)i] - detect_interval)) {
                        if (vc[(size_t)jj - 1] > vc[(size_t)last_best_ind]) last_best_ind = jj - 1;
                        jj--;
                    }
                }
            }
        }
        if (last_best_ind >= 0) {
            if (vc[(size_t)i] > vc[(size_t)last_best_ind]) {
                to_use[(size_t)i] = 1;
                to_use[(size_t)last_best_ind] = 0;
                last_best_ind = i;
            } else {
                to_use[(size_t)i] = 0;
            }
        } else {
            to_use[(size_t)i] = 1;
            last_best_ind = i;
        }
    }
    std::vector<int64_t> times;
    for (size_t i = 0; i < tc.size(); i++)
        if (to_use[i]) times.push_back(tc[i]);
    return times;
}

// detect_events on every channel over mountainsort3's time chunks (chunk
// timepoints, `pad` of padding each side, zeros outside [0, N); times kept
// inside the unpadded chunk, neighborhoodsorter.cpp:74-100).  counts[m] and
// times channel after channel; returns the total (times written up to
// capacity).
int64_t ref32_detect_events(const float* X, int64_t M, int64_t N, double detect_threshold, double detect_interval,
                            int sign, int64_t chunk, int64_t pad, int64_t* counts, int64_t* times, int64_t capacity) {
    int64_t total = 0;
    for (int64_t m = 0; m < M; m++) {
        counts[m] = 0;
        for (int64_t t1 = 0; t1 < N; t1 += chunk) {
            const int64_t size = std::min(chunk, N - t1);
            std::vector<double> X0((size_t)(size + 2 * pad));
            for (int64_t n = 0; n < size + 2 * pad; n++) {
                const int64_t t = t1 - pad + n;
                X0[(size_t)n] = (t >= 0 && t < N) ? (double)X[t * M + m] : 0.0;
            }
            for (int64_t t0 : detect_events_vec(X0, detect_threshold, detect_interval, sign)) {
                if ((0 <= t0 - pad) && (t0 - pad < size)) {
                    if (total < capacity) times[total] = t0 - pad + t1;
                    total++;
                    counts[m]++;
                }
            }
        }
    }
    return total;
}

// Whole ms3.whiten on an in-memory timeseries.  Also returns XXt and W when
// the caller passes buffers for them.
int ref32_whiten(const float* X, int64_t M, int64_t N, double quantization_unit, int exec_threads,
                 float* out, double* XXt_out, double* W_out) {
    std::vector<double> XXt((size_t)(M * M)), W((size_t)(M * M));
    ref32_whiten_xxt(X, M, N, exec_threads, XXt.data());
    ref32_whitening_matrix(XXt.data(), M, W.data(), nullptr, nullptr);
    ref32_whiten_apply(X, M, N, W.data(), quantization_unit, exec_threads, out);
    if (XXt_out) std::memcpy(XXt_out, XXt.data(), sizeof(double) * M * M);
    if (W_out) std::memcpy(W_out, W.data(), sizeof(double) * M * M);
    return 0;
}

}  // extern "C"
