// physics.hpp -- the reference's unit system and constants, evaluated as the
// reference evaluates them (src/Cosmoinput3D.h:1-22; conversions of the CLI
// arguments at src/CosmoBEC_MPI.cpp:329-339).  The numbers must match bit for bit: they
// set the time step, the drift phase and the snapshot header, so they are
// kept as the same expressions in the same order.
#pragma once

#include <cmath>

namespace ifdm {
namespace phys {

const double m2kpc = 3.086e19;                          // m
const double m2Mpc = 3.086e22;                          // m
const double cm2Mpc = 3.086e24;                         // cm
const double s2Myr = 60.0 * 60.0 * 24.0 * 365.0 * 1e6;  // s
const double kg2eV = 1.783e-36;                         // kg
const double kg2solar = 1.989e30;                       // solar
const double rhoc = 3.51059e+10;                        // Msun / Mpc^3
const double h_0 = 0.677;
const double H_0 = h_0 * 100 * s2Myr / m2Mpc * 1e3;     // 1/Myr
const double hbar = 6.58211928e-16 / s2Myr;             // eV Myr
const double Omega_m0 = 0.276;
const double bigG = 6.674e-11 * kg2solar / pow(m2Mpc, 3) * pow(s2Myr, 2);  // Mpc^3/Msun/Myr^2
const double c = 2.99792458e8 / m2Mpc * s2Myr;          // Mpc/Myr

}  // namespace phys
}  // namespace ifdm
