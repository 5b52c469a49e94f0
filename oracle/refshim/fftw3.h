// ORACLE / TEST INFRASTRUCTURE ONLY -- never linked into the product library.
//
// The FFTW 3 single-precision interface that packages/ms3/p_bandpass_filter.cpp
// calls (fftwf_plan_many_dft / fftwf_execute and the allocation and thread
// helpers), implemented over the oracle's own FFT (oracle/fft_ref.hpp: the
// unnormalised DFT in FP32 arithmetic with FP64 twiddles).  FFTW itself is a
// third-party dependency that the reference does not vendor and that is not
// installed here; this header states its published interface and computes the
// transform it defines.
#pragma once

#include <cstddef>

typedef float fftwf_complex[2];
typedef struct ms3ref_fftwf_plan* fftwf_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

void* fftwf_malloc(size_t n);
void fftwf_free(void* p);
fftwf_plan fftwf_plan_many_dft(int rank, const int* n, int howmany, fftwf_complex* in, const int* inembed,
                               int istride, int idist, fftwf_complex* out, const int* onembed, int ostride,
                               int odist, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup_threads(void);
