/* Declaration-only stand-in for FFTW3's MPI interface (oracle build only;
 * no FFT runs on the gauge hot path). */
#pragma once
#include <fftw3.h>
#include <mpi.h>
static inline void fftw_mpi_init(void) {}
static inline void fftw_mpi_cleanup(void) {}
static inline ptrdiff_t fftw_mpi_local_size_many(int, const ptrdiff_t*, ptrdiff_t, ptrdiff_t, MPI_Comm,
                                                 ptrdiff_t* n0, ptrdiff_t* s0)
{ *n0 = 0; *s0 = 0; return 1; }
static inline fftw_plan fftw_mpi_plan_many_dft(int, const ptrdiff_t*, ptrdiff_t, ptrdiff_t, ptrdiff_t, fftw_complex*,
                                               fftw_complex*, MPI_Comm, int, unsigned)
{ return (fftw_plan)0; }
static inline ptrdiff_t fftwf_mpi_local_size_many(int, const ptrdiff_t*, ptrdiff_t, ptrdiff_t, MPI_Comm,
                                                  ptrdiff_t* n0, ptrdiff_t* s0)
{ *n0 = 0; *s0 = 0; return 1; }
static inline fftwf_plan fftwf_mpi_plan_many_dft(int, const ptrdiff_t*, ptrdiff_t, ptrdiff_t, ptrdiff_t,
                                                 fftwf_complex*, fftwf_complex*, MPI_Comm, int, unsigned)
{ return (fftwf_plan)0; }
