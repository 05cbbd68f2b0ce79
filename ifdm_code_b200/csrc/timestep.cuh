// timestep.cuh -- Timestep_criteria (src/CosmoBEC_MPI.cpp:19-78) on the device.
//
// One block.  Thread 0 turns the max reductions of the previous passes into
// the three step criteria and advances the scale factor; three warps integrate
//   dt_KE = int da/(H a^3), dt_PE = int da/(H a^2), dt_QI = int da/(H a^4)
// (integrands src/struct3D.h:127-146) with the QUADPACK method the reference
// gets from GSL's qags: one 21-point Gauss-Kronrod rule, accepted when its
// error estimate meets epsrel = 1e-10, else bisection of the worst interval.
// It then writes the merged kick coefficients for the next z-pass and all
// threads fill the separable drift tables exp(-i s kappa_i^2).
#pragma once

#include "step_kernels.cuh"

namespace ifdm {

// ------------------------------------------------------------ quadrature --
__device__ __forceinline__ double qk_integrand(int n, double x, double H0, double Om) {
    const double H = H0 * sqrt(Om / pow(x, 3) + (1.0 - Om));
    return 1. / (H * pow(x, (double)n));
}

// 21-point Kronrod abscissae/weights and the embedded 10-point Gauss weights
// (QUADPACK qk21; x[1],x[3],..,x[9] are the Gauss nodes, x[10] = 0).
__device__ __constant__ double c_gk_x[11] = {
    0.995657163025808080735527280689003, 0.973906528517171720077964012084452,
    0.930157491355708226001207180059508, 0.865063366688984510732096688423493,
    0.780817726586416897063717578345042, 0.679409568299024406234327365114874,
    0.562757134668604683339000099272694, 0.433395394129247190799265943165784,
    0.294392862701460198131126603103866, 0.148874338981631210884826001129720,
    0.0};
__device__ __constant__ double c_gk_wk[11] = {
    0.011694638867371874278064396062192, 0.032558162307964727478818972459390,
    0.054755896574351996031381300244580, 0.075039674810919952767043140916190,
    0.093125454583697605535065465083366, 0.109387158802297641899210590325805,
    0.123491976262065851077958109831074, 0.134709217311473325928054001771707,
    0.142775938577060080797094273138717, 0.147739104901338491374841515972068,
    0.149445554002916905664936468389821};
__device__ __constant__ double c_gk_wg[5] = {
    0.066671344308688137593568809893332, 0.149451349150580593145776339657697,
    0.219086362515982043995534934228163, 0.269266719309996355091226921569469,
    0.295524224714752870173892994651338};

static __device__ void qk21(int n, double H0, double Om, double a, double b, double *res, double *abserr, double *resasc) {
    const double c = 0.5 * (a + b), h = 0.5 * (b - a);
    const double fc = qk_integrand(n, c, H0, Om);
    double kron = fc * c_gk_wk[10], gauss = 0.0, sabs = fabs(kron);
    double fl[10], fr[10];
    for (int j = 0; j < 10; ++j) {
        const double dxj = h * c_gk_x[j];
        fl[j] = qk_integrand(n, c - dxj, H0, Om);
        fr[j] = qk_integrand(n, c + dxj, H0, Om);
    }
    for (int j = 1; j < 10; j += 2) {
        const double s = fl[j] + fr[j];
        gauss += c_gk_wg[j / 2] * s;
        kron += c_gk_wk[j] * s;
        sabs += c_gk_wk[j] * (fabs(fl[j]) + fabs(fr[j]));
    }
    for (int j = 0; j < 10; j += 2) {
        const double s = fl[j] + fr[j];
        kron += c_gk_wk[j] * s;
        sabs += c_gk_wk[j] * (fabs(fl[j]) + fabs(fr[j]));
    }
    const double mean = 0.5 * kron;
    double sasc = c_gk_wk[10] * fabs(fc - mean);
    for (int j = 0; j < 10; ++j) sasc += c_gk_wk[j] * (fabs(fl[j] - mean) + fabs(fr[j] - mean));
    double err = fabs((kron - gauss) * h);
    kron *= h;
    sabs *= fabs(h);
    sasc *= fabs(h);
    if (sasc != 0.0 && err != 0.0) {
        const double scale = pow(200.0 * err / sasc, 1.5);
        err = (scale < 1.0) ? sasc * scale : sasc;
    }
    const double eps = 2.220446049250313e-16, dmin = 2.2250738585072014e-308;
    if (sabs > dmin / (50.0 * eps)) err = fmax(err, 50.0 * eps * sabs);
    *res = kron;
    *abserr = err;
    *resasc = sasc;
}

// The same rule evaluated by a whole warp: lanes 0-9 take the left nodes,
// 10-19 the right ones, 20 the centre (the integrand's two pow calls are the
// cost), then every lane sums the 21 values in qk21's order, so the results
// are bit-identical to qk21 and equal on all lanes.  Called by all 32 lanes.
static __device__ void qk21_warp(int n, double H0, double Om, double a, double b, double *res, double *abserr,
                                 double *resasc) {
    const int lane = threadIdx.x & 31;
    const double c = 0.5 * (a + b), h = 0.5 * (b - a);
    double x = c;
    if (lane < 20) {
        const double dxj = h * c_gk_x[lane % 10];
        x = lane < 10 ? c - dxj : c + dxj;
    }
    const double f = lane <= 20 ? qk_integrand(n, x, H0, Om) : 0.0;
    const double fc = __shfl_sync(0xffffffffu, f, 20);
    double kron = fc * c_gk_wk[10], gauss = 0.0, sabs = fabs(kron);
    double fl[10], fr[10];
#pragma unroll
    for (int j = 0; j < 10; ++j) {
        fl[j] = __shfl_sync(0xffffffffu, f, j);
        fr[j] = __shfl_sync(0xffffffffu, f, 10 + j);
    }
    for (int j = 1; j < 10; j += 2) {
        const double s = fl[j] + fr[j];
        gauss += c_gk_wg[j / 2] * s;
        kron += c_gk_wk[j] * s;
        sabs += c_gk_wk[j] * (fabs(fl[j]) + fabs(fr[j]));
    }
    for (int j = 0; j < 10; j += 2) {
        const double s = fl[j] + fr[j];
        kron += c_gk_wk[j] * s;
        sabs += c_gk_wk[j] * (fabs(fl[j]) + fabs(fr[j]));
    }
    const double mean = 0.5 * kron;
    double sasc = c_gk_wk[10] * fabs(fc - mean);
    for (int j = 0; j < 10; ++j) sasc += c_gk_wk[j] * (fabs(fl[j] - mean) + fabs(fr[j] - mean));
    double err = fabs((kron - gauss) * h);
    kron *= h;
    sabs *= fabs(h);
    sasc *= fabs(h);
    if (sasc != 0.0 && err != 0.0) {
        const double scale = pow(200.0 * err / sasc, 1.5);
        err = (scale < 1.0) ? sasc * scale : sasc;
    }
    const double eps = 2.220446049250313e-16, dmin = 2.2250738585072014e-308;
    if (sabs > dmin / (50.0 * eps)) err = fmax(err, 50.0 * eps * sabs);
    *res = kron;
    *abserr = err;
    *resasc = sasc;
}

#define IFDM_QLIMIT 64
// Returns 0 on success, 1 when the interval limit was reached.  WARP: the
// rule is evaluated by the calling warp (all 32 lanes call, every lane gets
// the result); else by the calling thread alone.
template <bool WARP = false>
static __device__ int qags_dev(int n, double H0, double Om, double a, double b, int limit, double *result) {
    auto rule = [&](double lo_, double hi_, double *r, double *e, double *sc) {
        if constexpr (WARP) qk21_warp(n, H0, Om, lo_, hi_, r, e, sc);
        else qk21(n, H0, Om, lo_, hi_, r, e, sc);
    };
    double r0, e0, s0;
    rule(a, b, &r0, &e0, &s0);
    if ((e0 <= 1e-10 * fabs(r0) && e0 != s0) || e0 == 0.0) {
        *result = r0;
        return 0;
    }
    double lo[IFDM_QLIMIT], hi[IFDM_QLIMIT], rr[IFDM_QLIMIT], ee[IFDM_QLIMIT];
    if (limit > IFDM_QLIMIT) limit = IFDM_QLIMIT;
    int cnt = 1;
    lo[0] = a; hi[0] = b; rr[0] = r0; ee[0] = e0;
    double tot = r0;
    while (cnt < limit) {
        int w = 0;
        for (int i = 1; i < cnt; ++i) if (ee[i] > ee[w]) w = i;
        const double m = 0.5 * (lo[w] + hi[w]);
        double r1, e1, r2, e2, t;
        rule(lo[w], m, &r1, &e1, &t);
        rule(m, hi[w], &r2, &e2, &t);
        lo[cnt] = m; hi[cnt] = hi[w]; rr[cnt] = r2; ee[cnt] = e2;
        hi[w] = m; rr[w] = r1; ee[w] = e1;
        ++cnt;
        double te = 0.0;
        tot = 0.0;
        for (int i = 0; i < cnt; ++i) { tot += rr[i]; te += ee[i]; }
        if (te <= 1e-10 * fabs(tot)) { *result = tot; return 0; }
    }
    *result = tot;
    return 1;
}

__device__ __forceinline__ double bits_to_double(unsigned long long b) { return __longlong_as_double((long long)b); }

// After the initial density pass: partial sums (3 per block, fixed order) ->
// first offset c = mean psi_s and the conserved mean mu = <|psi_s|^2>.
static __global__ void k_reduce_init(TState *__restrict__ ts, const double *__restrict__ part, int nblocks, double n3) {
    __shared__ double red[3][256];
    double a = 0, b = 0, c = 0;
    for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
        a += part[3 * i];
        b += part[3 * i + 1];
        c += part[3 * i + 2];
    }
    red[0][threadIdx.x] = a;
    red[1][threadIdx.x] = b;
    red[2][threadIdx.x] = c;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] += red[2][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        ts->cnext_re = red[0][0] / n3;
        ts->cnext_im = red[1][0] / n3;
        ts->mu = red[2][0] / n3;
    }
}

// The timestep.  drift64/drift32: tables exp(-i s kappa_i^2), i < N.  Run by
// one block: thread 0 does the scalar work, all threads fill the tables.
__device__ __forceinline__ void timestep_body(TState *ts, const Phys &ph, double2 *drift64, float2 *drift32) {
    __shared__ double s_drift, s_ai, s_da, s_int[3];
    __shared__ int s_bad[3];
    if (threadIdx.x == 0) {
        const double maxphi = ph.Phi0 * bits_to_double(ts->maxphi_bits);
        const double maxrho = ph.S2 * bits_to_double(ts->maxrho_bits);
        ts->maxphi_bits = 0ull;
        ts->maxrho_bits = 0ull;
        ts->maxphi = maxphi;
        ts->maxrho = maxrho;
        const double ai = ts->a;
        const double dt_KE = ph.A_KE * (ai * ai);
        const double dt_PE = ph.B_PE / maxphi * ai;
        double dt_QI = ph.C_QI / maxrho * (ai * ai * ai);
        if (ph.g == 0) dt_QI = 0.0;
        double max_dt = dt_KE;
        int crit = 3;
        if (max_dt > dt_PE) { max_dt = dt_PE; crit = 2; }
        if ((max_dt > dt_QI) && (ph.g != 0)) { max_dt = dt_QI; crit = 4; }
        max_dt *= ph.dt_scale;
        const double H = ph.H0 * sqrt(ph.Om / (ai * ai * ai) + (1.0 - ph.Om));
        const double da = H * ai * max_dt;
        s_ai = ai;
        s_da = da;
        ts->cand_KE = dt_KE;
        ts->cand_PE = dt_PE;
        ts->cand_QI = dt_QI;
        ts->da = da;
        ts->crit = crit;
    }
    __syncthreads();
    // the three integrals of a to a + da, one full warp each (with fewer full
    // warps they take them in turn; a partial last warp stays out, its
    // shuffles need all 32 lanes); each warp evaluates a 21-point rule in one go
    const int wid = (int)(threadIdx.x >> 5), nfull = (int)(blockDim.x >> 5);
    for (int q = wid; wid < nfull && q < 3; q += nfull) {
        double r;
        const int bad = qags_dev<true>(q == 0 ? 3 : (q == 1 ? 2 : 4), ph.H0, ph.Om, s_ai, s_ai + s_da, ph.limit, &r);
        if ((threadIdx.x & 31) == 0) {
            s_int[q] = r;
            s_bad[q] = bad;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const double ai = s_ai, da = s_da;
        const double iKE = s_int[0], iPE = s_int[1], iQI = s_int[2];
        if (s_bad[0] | s_bad[1] | s_bad[2]) ts->err |= 1;
        ts->dt_KE = iKE;
        ts->dt_PE = iPE;
        ts->dt_QI = iQI;
        ts->a = ai + da;
        const double hp = 0.5 * iPE * ph.kP, hq = 0.5 * iQI * ph.kQ;
        ts->snapP = ts->pendP;
        ts->snapQ = ts->pendQ;
        ts->coefP = ts->pendP + hp;
        ts->coefQ = ts->pendQ + hq;
        ts->pendP = hp;
        ts->pendQ = hq;
        ts->drift_s = ph.kin * iKE;
        // global-phase dither (FP32 mode): psi is stored as exp(-i gphase) psi
        // and this step's kick adds alpha, a pseudo-random phase in [0, 2 pi)
        // from the step count, so consecutive steps round different numbers;
        // the offset c (a mean of psi) rotates with it
        double alpha = 0.0;
        if (ph.dither) {
            const unsigned long long h = (unsigned long long)ts->steps * 0x9e3779b97f4a7c15ull + 0x632be59bd9b4e019ull;
            const unsigned long long m = (h ^ (h >> 31)) * 0xbf58476d1ce4e5b9ull;
            alpha = 6.283185307179586476925286766559 * (double)((m ^ (m >> 29)) >> 11) * 0x1.0p-53;
        }
        double sa, ca;
        sincos(alpha, &sa, &ca);
        ts->alpha = alpha;
        ts->gphase_prev = ts->gphase;
        ts->gphase = fmod(ts->gphase + alpha, 6.283185307179586476925286766559);
        ts->cre = ts->cnext_re * ca + ts->cnext_im * sa;
        ts->cim = ts->cnext_im * ca - ts->cnext_re * sa;
        ts->steps += 1;
        s_drift = ph.kin * iKE;
    }
    __syncthreads();
    const double s = s_drift;
    const double twopi = 6.283185307179586476925286766559;
    for (int i = threadIdx.x; i < ph.N; i += blockDim.x) {
        const double k = (double)kappa(i, ph.N);
        double p = s * (k * k);
        p -= twopi * rint(p * (1.0 / twopi));
        double sn, cs;
        sincos(p, &sn, &cs);
        drift64[i] = make_double2(cs, -sn);
        drift32[i] = make_float2((float)cs, (float)-sn);
    }
}

static __global__ void k_timestep(TState *__restrict__ ts, Phys ph, double2 *__restrict__ drift64,
                           float2 *__restrict__ drift32) {
    timestep_body(ts, ph, drift64, drift32);
}

}  // namespace ifdm
