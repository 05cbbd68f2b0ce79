// state_types.hpp -- plain structs shared by host code and the kernels.
#pragma once

namespace ifdm {

// Time-integration state shared between the timestep kernel and the passes.
struct TState {
    double a;                   // scale factor after the latest timestep
    double dt_KE, dt_PE, dt_QI; // integrated weights of the current step
    double cand_KE, cand_PE, cand_QI, da; // criteria of the latest timestep (stdout)
    double coefP, coefQ;        // phase = coefP*phi_s + coefQ*|psi_s|^2 for P1 (merged half kicks)
    double snapP, snapQ;        // half kick owed by the state at this step's start (snapshots)
    double pendP, pendQ;        // half kick owed after this step's P9
    double drift_s;             // drift phase per unit kappa^2
    double cre, cim;            // offset c removed before the forward FFT, added after the inverse
    double cnext_re, cnext_im;  // mean of the kicked field, from the k = 0 coefficient (next step's c)
    double mu;                  // mean |psi_s|^2 (conserved), subtracted from the Poisson source
    double alpha;               // dither phase added to this step's kick (FP32 mode, else 0)
    double gphase, gphase_prev; // accumulated dither after / before this step's kick (mod 2 pi)
    double maxphi, maxrho;      // natural units, inputs of the latest timestep
    unsigned long long maxphi_bits, maxrho_bits; // atomicMax targets (scaled, non-negative doubles)
    long long steps;
    int crit;
    int err;
};

// Constants of the timestep kernel, computed on the host in FP64.
struct Phys {
    double A_KE;      // 4/(3 pi) (m/c^2)/hbar dx^2       (dt_KE = A_KE a^2)
    double B_PE;      // 2 pi hbar/(m/c^2)                (dt_PE = B_PE a / max|phi|)
    double C_QI;      // 2 pi hbar/|g|, 0 when g == 0     (dt_QI = C_QI a^3 / max|psi|^2)
    double g;
    double H0, Om;
    double kP;        // (m/(c^2 hbar)) * Phi0: phase per (dt_PE * phi_s)
    double kQ;        // (g/hbar) * S^2:        phase per (dt_QI * |psi_s|^2)
    double kin;       // 0.5 hbar/(m/c^2) (pi/xmax)^2: drift phase per (dt_KE * kappa^2)
    double Phi0, S2;  // natural units of phi_s and |psi_s|^2
    double dt_scale;  // fixed-step mode multiplier (1 = reference)
    int N;
    int dither;       // 1: rotate psi by a pseudo-random global phase every step (FP32 mode)
    int limit;        // quadrature interval limit on the device
};

}  // namespace ifdm
