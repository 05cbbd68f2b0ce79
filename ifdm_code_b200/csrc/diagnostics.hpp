// diagnostics.hpp -- device diagnostics of the wave function (diagnostics.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>

namespace ifdm {

constexpr int kMaxBins = 64;

// P(k) of delta = |psi|^2 / <|psi|^2> - 1 in nbins bins of |kappa| (kappa
// the integer wave vector, k = 2 pi kappa / L, L the box side): bin b holds
// edges[b] <= |kappa| < edges[b+1]; edges null: log-spaced from 1 to N/2.
// work: psi as complex128 N^3 on the device, overwritten.
// k_out: mean k of each bin's modes; pk_out: <|delta_k|^2> L^3 / N^6;
// modes_out: modes per bin; mean_rho: <|psi|^2>.  Any output may be null.
std::string power_spectrum(double2 *work, int N, double L, int nbins, const double *edges, double *k_out,
                           double *pk_out, long long *modes_out, double *mean_rho, cudaStream_t s);

// Means over the grid of |psi|^2, |grad psi|^2 (spectral derivative, k = pi
// kappa / xmax with kappa per axis in -N/2 .. N/2-1, xmax the half box), phi
// |psi|^2 and |psi|^4: out[0..3].  psi_work: psi as complex128 N^3 on the
// device, overwritten by its FFT; phi: N^3 doubles on the device.
std::string field_means(double2 *psi_work, const double *phi, int N, double xmax, double out[4], cudaStream_t s);

}  // namespace ifdm
