/* oracle/qags.c -- QUADPACK-method adaptive quadrature (see qags.h).
 * TEST INFRASTRUCTURE ONLY. */
#include "qags.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>

/* 21-point Kronrod abscissae on [0,1): x[1],x[3],..,x[9] are the 10-point
 * Gauss-Legendre nodes, x[10] = 0 is the centre.  Verified in
 * tests/test_oracle_quadrature.py: the Kronrod rule integrates x^k exactly
 * for k <= 31, the Gauss rule for k <= 19. */
static const double gk_x[11] = {
    0.995657163025808080735527280689003, 0.973906528517171720077964012084452,
    0.930157491355708226001207180059508, 0.865063366688984510732096688423493,
    0.780817726586416897063717578345042, 0.679409568299024406234327365114874,
    0.562757134668604683339000099272694, 0.433395394129247190799265943165784,
    0.294392862701460198131126603103866, 0.148874338981631210884826001129720,
    0.000000000000000000000000000000000};
static const double gk_wk[11] = {
    0.011694638867371874278064396062192, 0.032558162307964727478818972459390,
    0.054755896574351996031381300244580, 0.075039674810919952767043140916190,
    0.093125454583697605535065465083366, 0.109387158802297641899210590325805,
    0.123491976262065851077958109831074, 0.134709217311473325928054001771707,
    0.142775938577060080797094273138717, 0.147739104901338491374841515972068,
    0.149445554002916905664936468389821};
static const double gk_wg[5] = {
    0.066671344308688137593568809893332, 0.149451349150580593145776339657697,
    0.219086362515982043995534934228163, 0.269266719309996355091226921569469,
    0.295524224714752870173892994651338};

void oq_qk21(oq_fn f, void *params, double a, double b, double *result, double *abserr,
             double *resabs, double *resasc) {
    const double c = 0.5 * (a + b);
    const double h = 0.5 * (b - a);
    const double fc = f(c, params);
    double kron = fc * gk_wk[10];
    double gauss = 0.0;
    double sabs = fabs(kron);
    double fl[10], fr[10];
    for (int j = 0; j < 10; ++j) {
        const double dxj = h * gk_x[j];
        fl[j] = f(c - dxj, params);
        fr[j] = f(c + dxj, params);
    }
    /* Gauss nodes (odd indices) first, then the Kronrod-only nodes. */
    for (int j = 1; j < 10; j += 2) {
        const double s = fl[j] + fr[j];
        gauss += gk_wg[j / 2] * s;
        kron += gk_wk[j] * s;
        sabs += gk_wk[j] * (fabs(fl[j]) + fabs(fr[j]));
    }
    for (int j = 0; j < 10; j += 2) {
        const double s = fl[j] + fr[j];
        kron += gk_wk[j] * s;
        sabs += gk_wk[j] * (fabs(fl[j]) + fabs(fr[j]));
    }
    const double mean = 0.5 * kron;
    double sasc = gk_wk[10] * fabs(fc - mean);
    for (int j = 0; j < 10; ++j) sasc += gk_wk[j] * (fabs(fl[j] - mean) + fabs(fr[j] - mean));
    double err = fabs((kron - gauss) * h);
    kron *= h;
    sabs *= fabs(h);
    sasc *= fabs(h);
    if (sasc != 0.0 && err != 0.0) {
        const double scale = pow(200.0 * err / sasc, 1.5);
        err = (scale < 1.0) ? sasc * scale : sasc;
    }
    if (sabs > DBL_MIN / (50.0 * DBL_EPSILON)) {
        const double floor_err = 50.0 * DBL_EPSILON * sabs;
        if (floor_err > err) err = floor_err;
    }
    *result = kron;
    *abserr = err;
    *resabs = sabs;
    *resasc = sasc;
}

int oq_qags(oq_fn f, void *params, double a, double b, double epsabs, double epsrel,
            int limit, double *result, double *abserr) {
    double r0, e0, ra0, rs0;
    oq_qk21(f, params, a, b, &r0, &e0, &ra0, &rs0);
    double tol = fmax(epsabs, epsrel * fabs(r0));
    if ((e0 <= tol && e0 != rs0) || e0 == 0.0 || limit <= 1) {
        *result = r0;
        *abserr = e0;
        return 0;
    }
    /* bisection on the interval with the largest error estimate */
    double *lo = (double *)malloc(sizeof(double) * (size_t)limit);
    double *hi = (double *)malloc(sizeof(double) * (size_t)limit);
    double *rr = (double *)malloc(sizeof(double) * (size_t)limit);
    double *ee = (double *)malloc(sizeof(double) * (size_t)limit);
    int n = 1;
    lo[0] = a; hi[0] = b; rr[0] = r0; ee[0] = e0;
    double tot_r = r0, tot_e = e0;
    int status = 1;
    while (n < limit) {
        int w = 0;
        for (int i = 1; i < n; ++i) if (ee[i] > ee[w]) w = i;
        const double m = 0.5 * (lo[w] + hi[w]);
        double r1, e1, r2, e2, t1, t2;
        oq_qk21(f, params, lo[w], m, &r1, &e1, &t1, &t2);
        oq_qk21(f, params, m, hi[w], &r2, &e2, &t1, &t2);
        hi[n] = hi[w]; lo[n] = m; rr[n] = r2; ee[n] = e2;
        hi[w] = m; rr[w] = r1; ee[w] = e1;
        ++n;
        tot_r = 0.0; tot_e = 0.0;
        for (int i = 0; i < n; ++i) { tot_r += rr[i]; tot_e += ee[i]; }
        tol = fmax(epsabs, epsrel * fabs(tot_r));
        if (tot_e <= tol) { status = 0; break; }
    }
    *result = tot_r;
    *abserr = tot_e;
    free(lo); free(hi); free(rr); free(ee);
    return status;
}
