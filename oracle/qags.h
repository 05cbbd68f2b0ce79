/*
 * oracle/qags.h -- adaptive Gauss-Kronrod quadrature for the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference integrates the scale-factor
 * integrals with GSL 2.4 `gsl_integration_qags(f, a, a+da, 0, 1e-10, 1000,
 * w, &res, &err)` (src/CosmoBEC_MPI.cpp:66-68; GSL pinned by job.sh:9).
 * GSL is not in the reference tree.  This file restates the published
 * QUADPACK method (Piessens, de Doncker-Kapenga, Ueberhuber, Kahaner 1983):
 *
 *  1. one 21-point Gauss-Kronrod rule (10-point Gauss embedded) on [a,b],
 *     with QUADPACK's error estimate
 *        err = resasc * min(1, (200 |K-G| / resasc)^1.5),
 *        err = max(err, 50 eps resabs);
 *  2. accept when err <= max(epsabs, epsrel |K|) and err != resasc, or err==0;
 *  3. otherwise bisect the interval with the largest error until the summed
 *     error meets the tolerance or `limit` intervals exist.
 *
 * QAGS adds Wynn epsilon extrapolation to step 3; it only changes results for
 * integrands with end-point singularities.  The integrands here,
 * 1/(H(a) a^n) on [a, a+da] with a > 0, are analytic, and step 2 accepts the
 * first rule (err ~ 1e-14 relative against epsrel = 1e-10), so the
 * extrapolation branch is never reached.  The product's device quadrature
 * implements the same three steps.
 */
#ifndef IFDM_ORACLE_QAGS_H
#define IFDM_ORACLE_QAGS_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double (*oq_fn)(double x, void *params);

/* Returns 0 on success, 1 when the limit was hit (result still written). */
int oq_qags(oq_fn f, void *params, double a, double b, double epsabs, double epsrel,
            int limit, double *result, double *abserr);

/* The 21-point rule alone (exposed for tests). */
void oq_qk21(oq_fn f, void *params, double a, double b, double *result, double *abserr,
             double *resabs, double *resasc);

#ifdef __cplusplus
}
#endif
#endif
