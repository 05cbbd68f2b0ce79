/*
 * oracle/fft64.h -- FP64 mixed-radix FFT used by the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker's FFT: the oracle
 * restatement (oracle/ifdm_oracle.c) and the single-rank FFTW shim
 * (oracle/shim/fftw_shim.c) both call it.  Nothing on the product path
 * links it.
 *
 * The reference calls FFTW3 / fftw3_mpi (version unpinned: `module load
 * fftw3`, job.sh:10; `-lfftw3 -lfftw3_mpi`, src/Makefile:2).  FFTW is not in
 * the reference tree; what the reference relies on is the mathematical
 * contract of its plans (src/CosmoBEC_MPI.cpp:174-177):
 *   forward  X[k] = sum_n x[n] exp(-2 pi i n k / N)     (FFTW_FORWARD = -1)
 *   backward x[n] = sum_k X[k] exp(+2 pi i n k / N)     (FFTW_BACKWARD = +1)
 * unnormalised, row-major, last index fastest.  r2c keeps k = 0..N/2 of the
 * last axis; c2r reads that half spectrum and assumes Hermitian symmetry
 * (the imaginary parts of the k=0 and k=N/2 coefficients of each last-axis
 * line are ignored, as in FFTW's halfcomplex backward transforms).
 *
 * Algorithm: Stockham autosort (self-sorting) decimation in frequency,
 * radices 4 / 2 / 3 / 5 specialised and a direct DFT for any other prime,
 * twiddles from a long-double table rounded once to double.
 */
#ifndef IFDM_ORACLE_FFT64_H
#define IFDM_ORACLE_FFT64_H

#include <complex.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex ocplx;

/* 3-D complex transform, in place on a[n0][n1][n2] (pitch n2), sign -1 / +1. */
void offt_c2c_3d(ocplx *a, int n0, int n1, int n2, int sign);

/* 3-D real -> half-complex: in[n0][n1][in_pitch] (in_pitch >= n2 doubles),
 * out[n0][n1][n2/2+1].  Forward sign. */
void offt_r2c_3d(const double *in, ocplx *out, int n0, int n1, int n2, int in_pitch);

/* 3-D half-complex -> real (backward sign), destroys `in`:
 * in[n0][n1][n2/2+1] -> out[n0][n1][out_pitch] (first n2 entries written). */
void offt_c2r_3d(ocplx *in, double *out, int n0, int n1, int n2, int out_pitch);

/* 1-D helper on a contiguous line (tests). */
void offt_c2c_1d(ocplx *line, int n, int sign);

/* Number of OpenMP threads the transforms use (1 if built without OpenMP). */
int offt_num_threads(void);

#ifdef __cplusplus
}
#endif
#endif
