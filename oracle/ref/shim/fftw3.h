/* Declaration-only stand-in for FFTW3, written for this project so that the
 * reference library's headers compile for the oracle build.  The gauge
 * hot path never performs an FFT; these stubs do nothing.  Test
 * infrastructure for the oracle only. */
#pragma once
#include <stdlib.h>
typedef double fftw_complex[2];
typedef struct qshim_fftw_plan_s* fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
static inline void* fftw_malloc(size_t n) { return malloc(n); }
static inline void fftw_free(void* p) { free(p); }
static inline fftw_plan fftw_plan_many_dft(int, const int*, int, fftw_complex*, const int*, int, int,
                                           fftw_complex*, const int*, int, int, int, unsigned)
{ return (fftw_plan)0; }
static inline void fftw_execute(const fftw_plan) {}
static inline void fftw_execute_dft(const fftw_plan, fftw_complex*, fftw_complex*) {}
static inline void fftw_destroy_plan(fftw_plan) {}
static inline int fftw_init_threads(void) { return 1; }
static inline void fftw_plan_with_nthreads(int) {}
typedef float fftwf_complex[2];
typedef struct qshim_fftwf_plan_s* fftwf_plan;
static inline void* fftwf_malloc(size_t n) { return malloc(n); }
static inline void fftwf_free(void* p) { free(p); }
static inline fftwf_plan fftwf_plan_many_dft(int, const int*, int, fftwf_complex*, const int*, int, int,
                                             fftwf_complex*, const int*, int, int, int, unsigned)
{ return (fftwf_plan)0; }
static inline void fftwf_execute(const fftwf_plan) {}
static inline void fftwf_execute_dft(const fftwf_plan, fftwf_complex*, fftwf_complex*) {}
static inline void fftwf_destroy_plan(fftwf_plan) {}
