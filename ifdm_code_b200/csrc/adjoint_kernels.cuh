// adjoint_kernels.cuh -- pieces of the adjoint leap-frog step.
//
// One forward step maps psi_n to psi_{n+1} = U_n K_n psi_n with the kick
//   K_n psi = psi exp(-i theta),  theta = a phi_s[|psi|^2] + b |psi|^2 + alpha
// (phi_s the linear, symmetric Poisson operator -F^-1[F[.]/kappa^2]/N^3 with
// k = 0 removed) and the unitary drift U_n = F^-1 diag(exp(-i s kappa^2)) F / N^3.
// For a real loss L and g = dL/dRe psi + i dL/dIm psi:
//   g' = U_n^H g_{n+1}                          (drift with exp(+i s kappa^2))
//   w  = Im(conj(g') psi'),  psi' = K_n psi_n
//   u  = a phi_s[w] + b w                        (one more Poisson solve)
//   g_n = exp(+i theta) g' + 2 u psi_n.
// The Delta-t schedule is the one recorded in the forward pass (it depends on
// max reductions, which are not differentiated).
#pragma once

#include "step_kernels.cuh"

namespace ifdm {

// Coefficients of one recorded step, as its passes used them.
struct StepLog {
    double coefP;        // kick coefficient of the stored phi
    double coefQ;        // kick coefficient of |psi_s|^2
    double alpha;        // dither phase of the kick
    double drift_s;      // drift phase per unit kappa^2
    double cre, cim;     // offset c of this step
    double pendP, pendQ; // half kick owed after this step
    double gphase;       // accumulated dither after this step's kick
    double a, dt_KE, dt_PE, dt_QI;
};

// Load one recorded step into the pass state and rebuild its drift tables;
// conj != 0 writes the conjugate tables (the adjoint drift) instead.
__global__ void k_replay_step(TState *__restrict__ ts, const StepLog *__restrict__ lg, int N, int conj,
                              long long steps, double2 *__restrict__ drift64, float2 *__restrict__ drift32) {
    const StepLog e = *lg;
    if (threadIdx.x == 0) {
        ts->steps = steps;
        ts->coefP = e.coefP;
        ts->coefQ = e.coefQ;
        ts->alpha = e.alpha;
        ts->drift_s = e.drift_s;
        ts->cre = e.cre;
        ts->cim = e.cim;
        ts->pendP = e.pendP;
        ts->pendQ = e.pendQ;
        ts->gphase = e.gphase;
        ts->a = e.a;
    }
    const double twopi = 6.283185307179586476925286766559;
    for (int i = threadIdx.x; i < N; i += blockDim.x) {
        const double k = (double)kappa(i, N);
        double p = e.drift_s * (k * k);
        p -= twopi * rint(p * (1.0 / twopi));
        double sn, cs;
        sincos(p, &sn, &cs);
        if (conj) sn = -sn;
        drift64[i] = make_double2(cs, -sn);
        drift32[i] = make_float2((float)cs, (float)-sn);
    }
}

// Append the step the timestep kernel just prepared to the log.
__global__ void k_log_step(const TState *__restrict__ ts, StepLog *__restrict__ lg) {
    StepLog e;
    e.coefP = ts->coefP;
    e.coefQ = ts->coefQ;
    e.alpha = ts->alpha;
    e.drift_s = ts->drift_s;
    e.cre = ts->cre;
    e.cim = ts->cim;
    e.pendP = ts->pendP;
    e.pendQ = ts->pendQ;
    e.gphase = ts->gphase;
    e.a = ts->a;
    e.dt_KE = ts->dt_KE;
    e.dt_PE = ts->dt_PE;
    e.dt_QI = ts->dt_QI;
    *lg = e;
}

// w = Im(conj(g') psi'), psi' = psi exp(-i theta), theta = a phi + b |psi|^2 + alpha
template <typename R, typename K>
__global__ void k_adj_w(const cx<R> *__restrict__ g, const cx<R> *__restrict__ psi, const R *__restrict__ phi,
                        double a, double b, double alpha, R *__restrict__ w, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double px = (double)psi[i].x, py = (double)psi[i].y;
        const double th = a * (double)phi[i] + b * (px * px + py * py) + alpha;
        double s, c;
        sincos(th, &s, &c);
        const double qx = px * c + py * s, qy = py * c - px * s;  // psi'
        const double gx = (double)g[i].x, gy = (double)g[i].y;
        w[i] = (R)(gx * qy - gy * qx);
    }
}

// g <- exp(+i theta) g + 2 (aP pw + b w) psi, pw = phi_s[w]
template <typename R, typename K>
__global__ void k_adj_combine(cx<R> *__restrict__ g, const cx<R> *__restrict__ psi, const R *__restrict__ phi,
                              const R *__restrict__ pw, const R *__restrict__ w, double a, double aP, double b,
                              double alpha, size_t n, uint32_t salt) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double px = (double)psi[i].x, py = (double)psi[i].y;
        const double th = a * (double)phi[i] + b * (px * px + py * py) + alpha;
        double s, c;
        sincos(th, &s, &c);
        const double gx = (double)g[i].x, gy = (double)g[i].y;
        const double u = aP * (double)pw[i] + b * (double)w[i];
        const double ox = gx * c - gy * s + 2.0 * u * px;
        const double oy = gy * c + gx * s + 2.0 * u * py;
        g[i] = Cvt<R, double>::out(make_double2(ox, oy), salt, i);
    }
}

// Real source field -> half spectrum along z (the r2c half of the density pass).
template <typename R, typename K, int N>
__global__ void __launch_bounds__(TileZ<R, K, N>::NT)
    k_source_r2c_z(const R *__restrict__ src, cx<R> *__restrict__ rhok, const TState *__restrict__ ts,
                   const cx<K> *__restrict__ tw, const cx<K> *__restrict__ twh) {
    using TL = TileZ<R, K, N>;
    using C = typename TL::C;
    constexpr int NH = N / 2 + 1, NHP = half_pitch<R>(N), M = N / 2;
    extern __shared__ __align__(16) unsigned char smraw[];
    C *sm = reinterpret_cast<C *>(smraw);
    K *smr = reinterpret_cast<K *>(sm);
    const size_t row0 = size_t(blockIdx.x) * TL::L;
    const uint32_t salt = pass_salt(ts, 11);
    for (int f = threadIdx.x; f < TL::L * N; f += TL::NT) {
        const int l = f / N, n = f % N;
        smr[2 * ((n >> 1) * TL::LP + l) + (n & 1)] = (K)src[row0 * N + f];
    }
    __syncthreads();
    fft_tile<C, M, TL::EH, -1, TL::L, TL::LP, typename TL::HP>(sm, twh);
    constexpr int TPR = TL::NT / TL::L;  // threads per row: no division by N/2+1
    static_assert(TPR * TL::L == TL::NT, "whole rows per thread block");
    const int l = threadIdx.x / TPR;
    for (int k = threadIdx.x % TPR; k < NH; k += TPR) {
        const C zk = sm[(k % M) * TL::LP + l];
        const C zc = cconj(sm[((M - k) % M) * TL::LP + l]);
        const C e = cscale(zk + zc, K(0.5));
        const C o = cscale(zk - zc, K(0.5));
        const C wo = post_tw<-1, N>(tw, k % N, o);
        const size_t gi = (row0 + l) * NHP + k;
        rhok[gi] = Cvt<R, K>::out(mkc(e.x + wo.y, e.y - wo.x), salt, gi);
    }
}

// max |x_i| over n doubles into *out (the ordered bits of a non-negative
// double; *out zeroed before); NaN entries are skipped
__global__ void k_absmax(const double *__restrict__ x, size_t n, unsigned long long *__restrict__ out) {
    double m = 0.0;
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        m = fmax(m, fabs(x[i]));
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

// complex128 (natural units) <-> storage type, with a real scale
template <typename R>
__global__ void k_scale_in(const double2 *__restrict__ in, cx<R> *__restrict__ out, double f, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = mkc((R)(in[i].x * f), (R)(in[i].y * f));
}
template <typename R>
__global__ void k_scale_out(const cx<R> *__restrict__ in, double2 *__restrict__ out, double f, size_t n) {
    for (size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = make_double2((double)in[i].x * f, (double)in[i].y * f);
}

}  // namespace ifdm
