// ic_pipeline.hpp -- device IC pre-processing (see ic_pipeline.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

namespace ifdm {

struct IcInput {
    int N = 0;
    double Lg = 0, box = 0;  // cell size and box [kpc/h]
    double pmass = 0;        // particle mass [Msun/h] (mass[1] * 1e10)
    double L3 = 0;           // pow(Lg, 3) as the host evaluates it
    double a = 0;            // header.time
    double xmax = 0, dx = 0; // half box and cell size [Mpc]
    double mfdm_solar = 0;
    double kf = 0;           // mfdm / pow(c,2) / hbar
    double uc_rho = 0;       // pow(h_0,2) * pow(1e3,3)
    double uc_vel = 0;       // 1e3 / m2Mpc * s2Myr
    const float *d_pos = nullptr, *d_vel = nullptr;  // device, 3 floats per particle, in the
    long np = 0;                                     // reference's processing order
    cudaStream_t stream = nullptr;
};

// Deposits, solves the velocity phase and writes psi (complex128, device,
// N^3) and the x-velocity grid (host) for voutput.dat.
std::string ic_pipeline(const IcInput &in, double *d_psi_out, std::vector<float> *vx_out);

}  // namespace ifdm
