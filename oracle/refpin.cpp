// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// C entry points over the reference's own processor functions, compiled from
// the reference's sources (packages/ms3/p_bandpass_filter.cpp, p_whiten.cpp,
// pca.cpp, p_mask_out_artifacts.cpp, common/mlcompute.cpp and the mda/
// classes) against the Qt subset in refshim/ and the FFTW interface in
// refshim/fftw3.h (the oracle's FFT).  Built into oracle/_ref/libmsref.so by
// `make -C oracle ref` where the reference checkout is present.  The tests
// use it to pin the restatement (ref32) to the reference's code and to make
// the committed golden vectors; bench.py's reference arm times it.
//
// The processors read and write .mda files, as the reference does; the
// Python side (oracle/refpin.py) writes the inputs and reads the outputs.
#include <omp.h>

#include <cstdint>
#include <exception>

#include "mda.h"
#include "p_bandpass_filter.h"
#include "p_mask_out_artifacts.h"
#include "p_whiten.h"
#include "pca.h"

extern "C" {

// ms3.bandpass_filter (p_bandpass_filter.cpp:115-229).  The chunk geometry
// follows omp_get_max_threads() (:147), so geometry_threads is set as the
// OpenMP thread count, as --_request_num_threads does in the executable
// (mountainsort3_main.cpp:428-434).  Returns 0 on success.
int msref_bandpass_filter(const char* in, const char* out, double samplerate, double freq_min, double freq_max,
                          double freq_wid, double quantization_unit, int subsample_factor, int geometry_threads) {
    try {
        omp_set_num_threads(geometry_threads);
        Bandpass_filter_opts o;
        o.samplerate = samplerate;
        o.freq_min = freq_min;
        o.freq_max = freq_max;
        o.freq_wid = freq_wid;
        o.quantization_unit = quantization_unit;
        o.subsample_factor = subsample_factor;
        return p_bandpass_filter(in, out, o) ? 0 : -1;
    } catch (const std::exception&) {
        return -2;
    }
}

// ms3.whiten (p_whiten.cpp:45-206), on exec_threads OpenMP threads.
int msref_whiten(const char* in, const char* out, double quantization_unit, int exec_threads) {
    try {
        if (exec_threads > 0) omp_set_num_threads(exec_threads);
        Whiten_opts o;
        o.quantization_unit = quantization_unit;
        return p_whiten(in, out, o) ? 0 : -1;
    } catch (const std::exception&) {
        return -2;
    }
}

// whitening_matrix_from_XXt (pca.cpp:635-651) on an M x M column-major XXt.
int msref_whitening_matrix(const double* XXt, int64_t M, double* W) {
    try {
        Mda C(M, M);
        for (int64_t i = 0; i < M * M; i++) C.set(XXt[i], i);
        Mda Wm;
        whitening_matrix_from_XXt(Wm, C);
        if (Wm.N1() != M || Wm.N2() != M) return -1;
        for (int64_t i = 0; i < M * M; i++) W[i] = Wm.get(i);
        return 0;
    } catch (const std::exception&) {
        return -2;
    }
}

// ms3.compute_whitening_matrix (p_whiten.cpp:208-293): channels are 1-based,
// n_channels == 0 means all.
int msref_compute_whitening_matrix(const char* const* inputs, int n_inputs, const int* channels, int n_channels,
                                   const char* out) {
    try {
        QStringList list;
        for (int i = 0; i < n_inputs; i++) list << QString(inputs[i]);
        QList<int> ch;
        for (int i = 0; i < n_channels; i++) ch << channels[i];
        Whiten_opts o;
        return p_compute_whitening_matrix(list, ch, out, o) ? 0 : -1;
    } catch (const std::exception&) {
        return -2;
    }
}

// ms3.apply_whitening_matrix (p_whiten.cpp:357-429).
int msref_apply_whitening_matrix(const char* in, const char* W, const char* out, double quantization_unit) {
    try {
        Whiten_opts o;
        o.quantization_unit = quantization_unit;
        return p_apply_whitening_matrix(in, W, out, o) ? 0 : -1;
    } catch (const std::exception&) {
        return -2;
    }
}

// ms3.whiten_clips (p_whiten.cpp:295-355).
int msref_whiten_clips(const char* clips, const char* W, const char* out, double quantization_unit) {
    try {
        Whiten_opts o;
        o.quantization_unit = quantization_unit;
        return p_whiten_clips(clips, W, out, o) ? 0 : -1;
    } catch (const std::exception&) {
        return -2;
    }
}

// ms3.mask_out_artifacts (p_mask_out_artifacts.cpp:24-104).
int msref_mask_out_artifacts(const char* in, const char* out, double threshold, int interval_size) {
    try {
        return p_mask_out_artifacts(in, out, threshold, interval_size) ? 0 : -1;
    } catch (const std::exception&) {
        return -2;
    }
}

}  // extern "C"
