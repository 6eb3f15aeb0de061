#pragma once
// Oracle build shim (test infrastructure only).
//
// The reference's include/loki/utils/fft.hpp includes <fftw3.h> for the
// Fourier-domain FFA and the matched-filter templates, both off the
// time-domain FP32 path. FFTW is not installed here; this header declares the
// handful of single-precision entry points that lib/fft.cpp names, and
// oracle/ref_stubs.cpp defines them: batched 1-D r2c / c2r plans compute the
// DFT definition in double (FFTW's unscaled conventions), the 2-D plans and
// FFTW's allocators throw, clean-up calls do nothing.

#include <cstddef>

extern "C" {
typedef float fftwf_complex[2];
typedef struct fftwf_plan_s* fftwf_plan;

#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)

int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int nthreads);
void fftwf_cleanup_threads(void);
void fftwf_cleanup(void);
void fftw_cleanup(void);
fftwf_complex* fftwf_alloc_complex(std::size_t n);
float* fftwf_alloc_real(std::size_t n);
void fftwf_free(void* p);
void fftwf_destroy_plan(fftwf_plan p);
void fftwf_execute(const fftwf_plan p);
void fftwf_execute_dft_r2c(const fftwf_plan p, float* in, fftwf_complex* out);
void fftwf_execute_dft_c2r(const fftwf_plan p, fftwf_complex* in, float* out);
fftwf_plan fftwf_plan_many_dft_r2c(int rank, const int* n, int howmany, float* in,
                                   const int* inembed, int istride, int idist,
                                   fftwf_complex* out, const int* onembed,
                                   int ostride, int odist, unsigned flags);
fftwf_plan fftwf_plan_many_dft_c2r(int rank, const int* n, int howmany,
                                   fftwf_complex* in, const int* inembed,
                                   int istride, int idist, float* out,
                                   const int* onembed, int ostride, int odist,
                                   unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float* in, fftwf_complex* out,
                                 unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex* in, float* out,
                                 unsigned flags);
}
