/*
 * oracle/shim/gsl/gsl_integration.h -- the GSL 2.4 quadrature API subset the
 * reference calls (src/CosmoBEC_MPI.cpp:23,66-68,196-202), backed by the
 * oracle's QUADPACK-method restatement (oracle/qags.c).
 * TEST INFRASTRUCTURE ONLY.
 */
#ifndef IFDM_SHIM_GSL_INTEGRATION_H
#define IFDM_SHIM_GSL_INTEGRATION_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    double (*function)(double x, void *params);
    void *params;
} gsl_function;

typedef struct {
    size_t limit;
} gsl_integration_workspace;

gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n);
void gsl_integration_workspace_free(gsl_integration_workspace *w);
int gsl_integration_qags(const gsl_function *f, double a, double b, double epsabs, double epsrel, size_t limit,
                         gsl_integration_workspace *workspace, double *result, double *abserr);

#ifdef __cplusplus
}
#endif
#endif
