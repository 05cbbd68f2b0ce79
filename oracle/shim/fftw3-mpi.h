/*
 * oracle/shim/fftw3-mpi.h -- fftw3_mpi plans with one rank (the whole array
 * is local), backed by oracle/fft64.c.  TEST INFRASTRUCTURE ONLY.
 *
 * Layouts follow the fftw3_mpi contract the reference relies on
 * (src/CosmoBEC_MPI.cpp:88,174-177): r2c input is padded real
 * [n0][n1][2(n2/2+1)], output half-complex [n0][n1][n2/2+1]; c2r the reverse;
 * c2c is in place when in == out.
 */
#ifndef IFDM_SHIM_FFTW3_MPI_H
#define IFDM_SHIM_FFTW3_MPI_H

#include "fftw3.h"
#include "mpi.h"

#ifdef __cplusplus
extern "C" {
#endif

void fftw_mpi_init(void);
fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in, fftw_complex *out,
                               MPI_Comm comm, int sign, unsigned flags);
fftw_plan fftw_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double *in, fftw_complex *out,
                                   MPI_Comm comm, unsigned flags);
fftw_plan fftw_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in, double *out,
                                   MPI_Comm comm, unsigned flags);

#ifdef __cplusplus
}
#endif
#endif
