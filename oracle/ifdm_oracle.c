/*
 * oracle/ifdm_oracle.c -- CPU restatement of the reference path (see
 * ifdm_oracle.h).  TEST INFRASTRUCTURE ONLY.
 *
 * Expressions keep the reference's operation order so that, with the same
 * FFT, this file and the shimmed reference binary round identically.
 */
#define _GNU_SOURCE
#include "ifdm_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fft64.h"
#include "qags.h"

/* --- constants: src/Cosmoinput3D.h:1-22 (macros keep them constant-folded
 * exactly as the reference's namespace-scope const doubles are) ------------ */
#define M2KPC 3.086e19
#define M2MPC 3.086e22
#define CM2MPC 3.086e24
#define S2MYR (60.0 * 60.0 * 24.0 * 365.0 * 1e6)
#define KG2EV 1.783e-36
#define KG2SOLAR 1.989e30
#define RHOC_CONST 3.51059e+10
#define H_LITTLE 0.677
#define H_0 (H_LITTLE * 100 * S2MYR / M2MPC * 1e3)
#define HBAR (6.58211928e-16 / S2MYR)
#define OMEGA_M0 0.276
#define BIGG (6.674e-11 * KG2SOLAR / pow(M2MPC, 3) * pow(S2MYR, 2))
#define C_LIGHT (2.99792458e8 / M2MPC * S2MYR)

typedef double _Complex cplx;

struct orc_sim {
    orc_args a;
    char opath[4096], icpath[4096];
    /* globals of main(): src/CosmoBEC_MPI.cpp:329-339 */
    double mfdm, mfdm_solar, g;
    /* Params: src/struct3D.h:17-89 */
    int N;
    double xmax, dx, fftnorm;
    double *x, *k;
    double ai, rhoc;
    double dt_KE, dt_PE, dt_QI;
    int timesteps, twrite, ti;
    /* Operators: src/struct3D.h:98-125 */
    cplx *wfc, *phikk, *phik;
    double *phi, *KE_phase;
    float *vxg;
    double last_maxphi, last_maxrho;
};

void orc_constants(double *o) {
    o[0] = H_0;
    o[1] = HBAR;
    o[2] = BIGG;
    o[3] = C_LIGHT;
    o[4] = OMEGA_M0;
    o[5] = H_LITTLE;
    o[6] = RHOC_CONST;
    o[7] = CM2MPC;
}

int orc_num_threads(void) { return offt_num_threads(); }

/* src/struct3D.h:127-146 */
static double Ha2(double x, void *p) {
    double *q = (double *)p;
    double H = q[0] * sqrt(q[1] / pow(x, 3) + (1.0 - q[1]));
    return 1. / (H * pow(x, 2));
}
static double Ha3(double x, void *p) {
    double *q = (double *)p;
    double H = q[0] * sqrt(q[1] / pow(x, 3) + (1.0 - q[1]));
    return 1. / (H * pow(x, 3));
}
static double Ha4(double x, void *p) {
    double *q = (double *)p;
    double H = q[0] * sqrt(q[1] / pow(x, 3) + (1.0 - q[1]));
    return 1. / (H * pow(x, 4));
}

orc_sim *orc_create(const orc_args *args) {
    orc_sim *s = (orc_sim *)calloc(1, sizeof(orc_sim));
    s->a = *args;
    snprintf(s->opath, sizeof s->opath, "%s", args->opath ? args->opath : "");
    snprintf(s->icpath, sizeof s->icpath, "%s", args->icpath ? args->icpath : "");
    /* src/CosmoBEC_MPI.cpp:329-339 */
    s->mfdm = args->mfdm;
    s->mfdm_solar = s->mfdm * KG2EV / KG2SOLAR;
    s->g = args->g_in / (pow(CM2MPC, 3));
    const double xmax = args->xmax_in / H_LITTLE;
    const unsigned res = (unsigned)args->res;
    s->twrite = args->t_write;
    s->timesteps = args->t_stop;
    s->ti = args->ti;
    /* src/struct3D.h:43-87 */
    s->N = (int)res;
    s->xmax = xmax;
    s->dx = 2.0 * xmax / res;
    s->fftnorm = 1. / (double)(pow(res, 3));
    s->x = (double *)malloc(sizeof(double) * res);
    s->k = (double *)malloc(sizeof(double) * res);
    for (size_t i = 0; i < res; ++i) {
        s->x[i] = xmax / res - xmax + i * (2.0 * xmax / res);
        if (i < res / 2) s->k[i] = i * M_PI / xmax;
        else s->k[i] = ((double)(i)-res) * M_PI / xmax;
    }
    const size_t N = res, P = 2 * (N / 2 + 1);
    s->wfc = (cplx *)calloc(N * N * N, sizeof(cplx));
    s->phik = (cplx *)calloc(N * N * N, sizeof(cplx));
    s->phikk = (cplx *)calloc(N * N * (N / 2 + 1), sizeof(cplx));
    s->phi = (double *)calloc(N * N * P, sizeof(double));
    s->KE_phase = (double *)malloc(sizeof(double) * N * N * N);
    s->vxg = NULL;
    /* src/struct3D.h:121 */
    for (size_t i = 0; i < N; ++i)
        for (size_t j = 0; j < N; ++j)
            for (size_t k = 0; k < N; ++k)
                s->KE_phase[k + N * (j + N * i)] =
                    (0.5 * HBAR / (s->mfdm / pow(C_LIGHT, 2)) *
                     (pow(s->k[i], 2) + pow(s->k[j], 2) + pow(s->k[k], 2)));
    return s;
}

void orc_destroy(orc_sim *s) {
    if (!s) return;
    free(s->x); free(s->k); free(s->wfc); free(s->phik); free(s->phikk);
    free(s->phi); free(s->KE_phase); free(s->vxg);
    free(s);
}

/* ------------------------------------------------ poisson :80-119 ------- */
void orc_poisson(orc_sim *s) {
    const int N = s->N;
    const long P = 2 * (N / 2 + 1);
    const long NH = N / 2 + 1;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            for (int k = 0; k < N; ++k)
                s->phi[k + P * (j + (long)i * N)] =
                    s->mfdm_solar * (pow(cabs(s->wfc[k + N * (j + (long)i * N)]), 2)) - s->rhoc;
    offt_r2c_3d(s->phi, s->phikk, N, N, N, (int)P);
    const double *kv = s->k;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            for (int k = 0; k < NH; ++k) {
                const long idx = k + NH * (j + (long)i * N);
                if (pow(kv[i], 2) + pow(kv[j], 2) + pow(kv[k], 2) == 0) {
                    s->phikk[idx] = 0.0;
                } else {
                    s->phikk[idx] = -4.0 * M_PI * BIGG * s->phikk[idx] /
                                    (pow(kv[i], 2) + pow(kv[j], 2) + pow(kv[k], 2));
                }
            }
    offt_c2r_3d(s->phikk, s->phi, N, N, N, (int)P);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            for (int k = 0; k < P; ++k) {
                if (k < N) s->phi[k + P * (j + (long)i * N)] *= s->fftnorm;
                else s->phi[k + P * (j + (long)i * N)] = 0.0;
            }
}

/* ------------------------------------- Timestep_criteria :19-78 --------- */
void orc_timestep(orc_sim *s, double dt_scale) {
    const int N = s->N;
    const long P = 2 * (N / 2 + 1);
    (void)P;
    /* The reference's phi vector holds only N^3 elements (src/struct3D.h:110,
     * :117 push one per cell) although it is indexed with the padded pitch
     * 2(N/2+1); max_element (src/CosmoBEC_MPI.cpp:26) therefore scans the
     * first N^3 doubles of the padded layout, i.e. rows (i*N+j) below
     * N^3 / (2(N/2+1)), pads included. */
    const long nphi = (long)N * N * N, nw = (long)N * N * N;
    /* max_element by |.|, first maximum (src/CosmoBEC_MPI.cpp:26-27) */
    double bphi = 0.0;
    long iphi = 0;
    for (long i = 0; i < nphi; ++i)
        if (fabs(s->phi[iphi]) < fabs(s->phi[i])) iphi = i;
    bphi = s->phi[iphi];
    long iw = 0;
    for (long i = 0; i < nw; ++i)
        if (cabs(s->wfc[iw]) < cabs(s->wfc[i])) iw = i;
    const double maxphi = fabs(bphi);
    const double maxrho = pow(cabs(s->wfc[iw]), 2);
    s->last_maxphi = maxphi;
    s->last_maxrho = maxrho;
    const double mfdm = s->mfdm, g = s->g;
    double dt_KE = 4. / (3. * M_PI) * (mfdm / pow(C_LIGHT, 2)) / HBAR * pow(s->dx, 2) * pow(s->ai, 2);
    double dt_PE = 2. * M_PI * HBAR / (mfdm / pow(C_LIGHT, 2)) / maxphi * s->ai;
    double dt_QI = 2. * M_PI * HBAR / fabs(g) / maxrho * pow(s->ai, 3);
    if (g == 0) dt_QI = 0.0;
    if (s->a.verbose) printf(" max dt_KE = %g max dt_PE = %g max dt_QI = %g\n", dt_KE, dt_PE, dt_QI);
    double max_dt = dt_KE;
    if (max_dt > dt_PE) max_dt = dt_PE;
    if ((max_dt > dt_QI) && (g != 0)) max_dt = dt_QI;
    /* fixed-step mode extension: scale the selected step (1.0 = reference) */
    max_dt *= dt_scale;
    double H = H_0 * sqrt(OMEGA_M0 / pow(s->ai, 3) + (1.0 - OMEGA_M0));
    double da = H * s->ai * max_dt;
    double a_next = s->ai + da;
    double prm[2] = {H_0, OMEGA_M0};
    double err;
    oq_qags(Ha3, prm, s->ai, s->ai + da, 0, 1e-10, 1000, &s->dt_KE, &err);
    oq_qags(Ha2, prm, s->ai, s->ai + da, 0, 1e-10, 1000, &s->dt_PE, &err);
    oq_qags(Ha4, prm, s->ai, s->ai + da, 0, 1e-10, 1000, &s->dt_QI, &err);
    s->ai = a_next;
}

/* ------------------------------------------- Split_op_MPI :121-159 ------ */
static void kick(orc_sim *s) {
    const int N = s->N;
    const long P = 2 * (N / 2 + 1);
    const double mfdm = s->mfdm, g = s->g, dt_PE = s->dt_PE, dt_QI = s->dt_QI;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            for (int k = 0; k < N; ++k) {
                cplx *w = &s->wfc[k + N * (j + (long)N * i)];
                *w *= cexp(-0.5 *
                           (dt_PE * s->phi[k + P * (j + (long)i * N)] * mfdm / pow(C_LIGHT, 2) / HBAR +
                            dt_QI * g / HBAR * pow(cabs(*w), 2)) *
                           I);
            }
}

void orc_split_op(orc_sim *s) {
    const int N = s->N;
    kick(s); /* :130-134 */
    offt_c2c_3d(s->wfc, N, N, N, -1); /* :136 */
    const double dt_KE = s->dt_KE, fftnorm = s->fftnorm;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < N; ++i) /* :138-142 */
        for (int j = 0; j < N; ++j)
            for (int k = 0; k < N; ++k) {
                const long idx = k + N * (j + (long)N * i);
                s->wfc[idx] *= cexp(-s->KE_phase[idx] * dt_KE * I) * fftnorm;
            }
    offt_c2c_3d(s->wfc, N, N, N, +1); /* :144 */
    orc_poisson(s);                   /* :146 */
    kick(s);                          /* :148-152 */
}

/* ---------------------------------------------------- write3D.h -------- */
static int write_params(orc_sim *s, int t) { /* src/write3D.h:7-22 */
    char fn[4200];
    snprintf(fn, sizeof fn, "%soutput%d.dat", s->opath, t);
    FILE *f = fopen(fn, "wb");
    if (!f) return -1;
    double gg = s->g * (pow(CM2MPC, 3));
    fwrite(&s->mfdm, sizeof(double), 1, f);
    fwrite(&gg, sizeof(double), 1, f);
    fwrite(&s->ai, sizeof(double), 1, f);
    fwrite(s->x, sizeof(double), (size_t)s->N, f);
    fclose(f);
    return 0;
}

int orc_writeall(orc_sim *s, int t) { /* src/write3D.h:86-97, :55-77 */
    if (write_params(s, t)) return -1;
    char fn[4200];
    snprintf(fn, sizeof fn, "%soutput%d.dat", s->opath, t);
    FILE *f = fopen(fn, "ab");
    if (!f) return -1;
    const size_t n = (size_t)s->N * s->N * s->N;
    fwrite(s->wfc, sizeof(cplx), n, f);
    fclose(f);
    return 0;
}

static int write_vg(orc_sim *s) { /* src/write3D.h:24-53 (one rank: offset 0) */
    char fn[4200];
    snprintf(fn, sizeof fn, "%svoutput.dat", s->opath);
    FILE *f = fopen(fn, "r+b");
    if (!f) f = fopen(fn, "wb");
    if (!f) return -1;
    const size_t n = (size_t)s->N * s->N * s->N;
    fwrite(s->vxg, sizeof(float), n, f);
    fclose(f);
    return 0;
}

/* ------------------------------------------------ Simulation :183-310 --- */
int orc_simulation(orc_sim *s) {
    int write_num = 0;
    int write_sten_counter = 2;
    for (int tn = s->ti; tn < s->timesteps; ++tn) {
        orc_poisson(s);
        orc_timestep(s, 1.0);
        const double a = s->ai;
        if (a > 1) {
            orc_writeall(s, 999999);
            write_num++;
            break;
        } else if (a > 0.714 && write_num == 4) {
            orc_writeall(s, 999998);
            write_num++;
        } else if (a > 0.5 && write_num == (s->a.stan ? 2 : 3)) {
            orc_writeall(s, 999997);
            write_num++;
            break;
        } else if (!s->a.stan && a > 0.333 && write_num == 2) {
            orc_writeall(s, 999996);
            write_num++;
        } else if (a > 0.25 && write_num == 2) {
            orc_writeall(s, write_sten_counter);
            write_sten_counter++;
        } else if (a > 0.25 && write_num == 1) {
            orc_writeall(s, 999995);
            write_num++;
        } else if (a > 0.105 && write_num == 0) {
            orc_writeall(s, 999994);
            write_num++;
        } else if (((tn % s->twrite == 0)) || tn == s->timesteps - 1) {
            orc_writeall(s, tn + 1);
        }
        orc_split_op(s);
    }
    return 0;
}

int orc_run_fixed(orc_sim *s, int nsteps, double dt_scale) {
    for (int n = 0; n < nsteps; ++n) {
        orc_poisson(s);
        orc_timestep(s, dt_scale);
        orc_split_op(s);
    }
    return 0;
}

/* ------------------------------------------------ rerun :709-750 -------- */
int orc_read_rerun(orc_sim *s, int t) {
    char fn[4200];
    snprintf(fn, sizeof fn, "%soutput%d.dat", s->icpath, t);
    FILE *f = fopen(fn, "rb");
    if (!f) return -1;
    const int N = s->N;
    double dummy;
    size_t ok = fread(&dummy, sizeof(double), 1, f);
    ok += fread(&dummy, sizeof(double), 1, f);
    ok += fread(&s->ai, sizeof(double), 1, f);
    ok += fread(s->x, sizeof(double), (size_t)N, f);
    fseek(f, (long)((N + 3) * sizeof(double)), SEEK_SET);
    const size_t n = (size_t)N * N * N;
    ok += fread(s->wfc, sizeof(cplx), n, f);
    fclose(f);
    s->rhoc = RHOC_CONST;
    return ok == 3 + (size_t)N + n ? 0 : -2;
}

int orc_set_psi(orc_sim *s, const double *psi, double a) {
    memcpy(s->wfc, psi, sizeof(cplx) * (size_t)s->N * s->N * s->N);
    s->ai = a;
    s->rhoc = RHOC_CONST;
    return 0;
}

void orc_get_psi(const orc_sim *s, double *psi) {
    memcpy(psi, s->wfc, sizeof(cplx) * (size_t)s->N * s->N * s->N);
}

void orc_get_phi(const orc_sim *s, double *phi) {
    const int N = s->N;
    const long P = 2 * (N / 2 + 1);
    for (long r = 0; r < (long)N * N; ++r) memcpy(phi + r * N, s->phi + r * P, sizeof(double) * N);
}

void orc_get_vxg(const orc_sim *s, float *vx) {
    if (s->vxg) memcpy(vx, s->vxg, sizeof(float) * (size_t)s->N * s->N * s->N);
}
void orc_get_theta(const orc_sim *s, double *th) {
    memcpy(th, s->phik, sizeof(cplx) * (size_t)s->N * s->N * s->N);
}
double orc_get_a(const orc_sim *s) { return s->ai; }
double orc_get_rhoc(const orc_sim *s) { return s->rhoc; }
void orc_get_dts(const orc_sim *s, double *d) { d[0] = s->dt_KE; d[1] = s->dt_PE; d[2] = s->dt_QI; }
void orc_get_maxes(const orc_sim *s, double *m) { m[0] = s->last_maxphi; m[1] = s->last_maxrho; }

/* ------------------------------------------------------ Gadget IC ------ */
typedef struct { /* src/gadget_IC.h:17-33 */
    int npart[6];
    double mass[6];
    double time;
    double redshift;
    int flag_sfr;
    int flag_feedback;
    int npartTotal[6];
    int flag_cooling;
    int num_files;
    double BoxSize;
    double Omega0;
    double OmegaLambda;
    double HubbleParam;
    char fill[256 - 6 * 4 - 6 * 8 - 2 * 8 - 2 * 4 - 6 * 4 - 2 * 4 - 4 * 8];
} gadget_header;

/* CIC_scheme src/gadget_IC.h:45-156, one rank (local_n0 = Ng, my_rank = 0) */
static void cic_one(orc_sim *s, const gadget_header *hd, double Lg, const double *xg, float xp, float yp, float zp,
                    float vxp, float vyp, float vzp, float *vx, float *vy, float *vz) {
    const int Ng = s->N;
    const double pmass = hd->mass[1];
    int gi = (int)floor((xp - 0.5 * Lg) / Lg);
    int gj = (int)floor((yp - 0.5 * Lg) / Lg);
    int gk = (int)floor((zp - 0.5 * Lg) / Lg);
    if (gi == -1) { gi = Ng - 1; xp += hd->BoxSize; }
    if (gj < 0) { gj = Ng - 1; yp += hd->BoxSize; }
    if (gk < 0) { gk = Ng - 1; zp += hd->BoxSize; }
    const double dx = fabs((double)xp - xg[gi]) / Lg;
    const double dy = fabs((double)yp - xg[gj]) / Lg;
    const double dz = fabs((double)zp - xg[gk]) / Lg;
    const double tx = 1. - dx, ty = 1. - dy, tz = 1. - dz;
    int gii = gi + 1., gjj = gj + 1., gkk = gk + 1.;
    if (gii == Ng) gii = 0;
    if (gjj == Ng) gjj = 0;
    if (gkk == Ng) gkk = 0;
    const double L3 = pow(Lg, 3);
    cplx *w = s->wfc;
#define W(a, b, c) w[(a) + (long)Ng * ((b) + (long)(c) * Ng)]
#define V(arr, a, b, c) arr[(a) + (long)Ng * ((b) + (long)(c) * Ng)]
    if (gi >= 0 && gi < Ng) {
        W(gk, gj, gi) += tx * ty * tz * pmass / L3;
        W(gk, gjj, gi) += tx * dy * tz * pmass / L3;
        W(gkk, gj, gi) += tx * ty * dz * pmass / L3;
        W(gkk, gjj, gi) += tx * dy * dz * pmass / L3;
        V(vx, gk, gj, gi) += tx * ty * tz * vxp / L3;
        V(vx, gk, gjj, gi) += tx * dy * tz * vxp / L3;
        V(vx, gkk, gj, gi) += tx * ty * dz * vxp / L3;
        V(vx, gkk, gjj, gi) += tx * dy * dz * vxp / L3;
        V(vy, gk, gj, gi) += tx * ty * tz * vyp / L3;
        V(vy, gk, gjj, gi) += tx * dy * tz * vyp / L3;
        V(vy, gkk, gj, gi) += tx * ty * dz * vyp / L3;
        V(vy, gkk, gjj, gi) += tx * dy * dz * vyp / L3;
        V(vz, gk, gj, gi) += tx * ty * tz * vzp / L3;
        V(vz, gk, gjj, gi) += tx * dy * tz * vzp / L3;
        V(vz, gkk, gj, gi) += tx * ty * dz * vzp / L3;
        V(vz, gkk, gjj, gi) += tx * dy * dz * vzp / L3;
    }
    if (gii >= 0 && gii < Ng) {
        W(gk, gjj, gii) += dx * dy * tz * pmass / L3;
        W(gk, gj, gii) += dx * ty * tz * pmass / L3;
        W(gkk, gj, gii) += dx * ty * dz * pmass / L3;
        W(gkk, gjj, gii) += dx * dy * dz * pmass / L3;
        V(vx, gk, gjj, gii) += dx * dy * tz * vxp / L3;
        V(vx, gk, gj, gii) += dx * ty * tz * vxp / L3;
        V(vx, gkk, gj, gii) += dx * ty * dz * vxp / L3;
        V(vx, gkk, gjj, gii) += dx * dy * dz * vxp / L3;
        V(vy, gk, gjj, gii) += dx * dy * tz * vyp / L3;
        V(vy, gk, gj, gii) += dx * ty * tz * vyp / L3;
        V(vy, gkk, gj, gii) += dx * ty * dz * vyp / L3;
        V(vy, gkk, gjj, gii) += dx * dy * dz * vyp / L3;
        V(vz, gk, gjj, gii) += dx * dy * tz * vzp / L3;
        V(vz, gk, gj, gii) += dx * ty * tz * vzp / L3;
        V(vz, gkk, gj, gii) += dx * ty * dz * vzp / L3;
        V(vz, gkk, gjj, gii) += dx * dy * dz * vzp / L3;
    }
#undef W
#undef V
}

/* read_PosVel src/gadget_IC.h:259-353.  Returns particle count or <0. */
static long read_chunk(orc_sim *s, int chunk, gadget_header *hd, float **pos, float **vel) {
    char fn[4200];
    snprintf(fn, sizeof fn, "%s.%d", s->icpath, chunk);
    FILE *f = fopen(fn, "rb");
    if (!f) return -1;
    int dummy;
    size_t ok = fread(&dummy, 4, 1, f);
    ok += fread(hd, sizeof(gadget_header), 1, f);
    ok += fread(&dummy, 4, 1, f);
    if (ok != 3) { fclose(f); return -3; }
    /* box check src/gadget_IC.h:309-314 */
    if (!(fabs(hd->BoxSize - 2 * s->xmax * 1e3 * H_LITTLE) < 0.001)) { fclose(f); return -2; }
    hd->mass[1] *= 1e10;
    s->ai = hd->time;
    s->rhoc = 4 * hd->npart[1] * hd->mass[1] / pow(hd->BoxSize, 3) * pow(1e3, 3) * pow(H_LITTLE, 2);
    const long n = hd->npart[1];
    /* one extra zeroed particle: the single-rank scatter reads it (ifdm_oracle.h) */
    *pos = (float *)calloc((size_t)(3 * n + 3), sizeof(float));
    *vel = (float *)calloc((size_t)(3 * n + 3), sizeof(float));
    ok = fread(&dummy, 4, 1, f);
    ok += fread(*pos, sizeof(float), (size_t)(3 * n), f);
    ok += fread(&dummy, 4, 1, f);
    ok += fread(&dummy, 4, 1, f);
    ok += fread(*vel, sizeof(float), (size_t)(3 * n), f);
    fclose(f);
    if (ok != (size_t)(6 * n + 3)) return -3;
    return n;
}

int orc_load_ic(orc_sim *s) {
    const int Ng = s->N;
    const size_t n3 = (size_t)Ng * Ng * Ng;
    double *xg = (double *)malloc(sizeof(double) * Ng);
    float *vy = (float *)calloc(n3, sizeof(float));
    float *vz = (float *)calloc(n3, sizeof(float));
    free(s->vxg);
    s->vxg = (float *)calloc(n3, sizeof(float));
    float *vx = s->vxg;
    memset(s->wfc, 0, sizeof(cplx) * n3);
    gadget_header hd;
    double Lg = 0;
    for (int chunk = 0; chunk < 4; ++chunk) { /* src/gadget_IC.h:610-642 */
        float *pos = NULL, *vel = NULL;
        long n = read_chunk(s, chunk, &hd, &pos, &vel);
        if (n < 0) { free(xg); free(vy); free(vz); free(pos); free(vel); return (int)n; }
        Lg = hd.BoxSize / Ng;
        for (int i = 0; i < Ng; i++) xg[i] = i * Lg + 0.5 * Lg;
        if (s->a.ic_mode == ORC_IC_REF1) {
            /* src/gadget_IC.h:445-448: trailing particles beyond the last cell
             * centre are left ghosts of rank 0 -- with one rank they are also
             * owned, so they deposit twice; ghosts first (:496-502) */
            long lg = 0;
            for (long pn = n - 1; pn > 0; pn--) {
                if (xg[Ng - 1] < pos[pn * 3]) lg++;
                else break;
            }
            for (long p = n - lg; p < n; ++p)
                cic_one(s, &hd, Lg, xg, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], vel[3 * p], vel[3 * p + 1],
                        vel[3 * p + 2], vx, vy, vz);
            /* owned: numpart + 1 particles (:431-432), the last one zeroed */
            for (long p = 0; p < n + 1; ++p)
                cic_one(s, &hd, Lg, xg, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], vel[3 * p], vel[3 * p + 1],
                        vel[3 * p + 2], vx, vy, vz);
        } else {
            for (long p = 0; p < n; ++p)
                cic_one(s, &hd, Lg, xg, pos[3 * p], pos[3 * p + 1], pos[3 * p + 2], vel[3 * p], vel[3 * p + 1],
                        vel[3 * p + 2], vx, vy, vz);
        }
        free(pos);
        free(vel);
    }
    /* mass-weighted velocity src/gadget_IC.h:645-651 */
    for (size_t i = 0; i < n3; i++) {
        if (creal(s->wfc[i]) != 0) {
            vx[i] *= hd.mass[1] / creal(s->wfc[i]);
            vy[i] *= hd.mass[1] / creal(s->wfc[i]);
            vz[i] *= hd.mass[1] / creal(s->wfc[i]);
        }
    }
    /* initial_velocity_Poisson_Solver src/gadget_IC.h:157-247, one rank:
     * the left/right ghost planes are the last/first planes (periodic) */
    const int N = Ng;
    const double unit_conversion = 1e3 / M2MPC * S2MYR;
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++)
            for (int k = 0; k < N; k++) {
                int im = i - 1, jm = j - 1, km = k - 1, ip = i + 1, jp = j + 1, kp = k + 1;
                if (j == 0) jm = N - 1;
                if (k == 0) km = N - 1;
                if (j == N - 1) jp = 0;
                if (k == N - 1) kp = 0;
                float dvx, dvy, dvz;
                const float *Lv = vx + (size_t)N * N * (N - 1); /* Lvelx = last plane */
                const float *Rv = vx;                            /* Rvelx = first plane */
                if (i == 0 && N == 1) dvx = Rv[k + N * j] - Lv[k + N * j];
                else if (i == 0) dvx = vx[k + N * (j + (long)ip * N)] - Lv[k + N * j];
                else if (i == N - 1) dvx = Rv[k + N * j] - vx[k + N * (j + (long)im * N)];
                else dvx = vx[k + N * (j + (long)ip * N)] - vx[k + N * (j + (long)im * N)];
                dvy = vy[k + N * (jp + (long)i * N)] - vy[k + N * (jm + (long)i * N)];
                dvz = vz[kp + N * (j + (long)i * N)] - vz[km + N * (j + (long)i * N)];
                s->phik[k + N * (j + (long)i * N)] = 0.5 * (dvx + dvy + dvz) * unit_conversion / (s->dx);
            }
    offt_c2c_3d(s->phik, N, N, N, -1);
    for (int i = 0; i < N; i++)
        for (int j = 0; j < N; j++)
            for (int k = 0; k < N; k++) {
                const long idx = k + N * (j + (long)i * N);
                if (pow(s->k[i], 2) + pow(s->k[j], 2) + pow(s->k[k], 2) == 0) s->phik[idx] = 0.0;
                else
                    s->phik[idx] = -pow(s->ai, 3. / 2) * s->phik[idx] /
                                   (pow(s->k[i], 2) + pow(s->k[j], 2) + pow(s->k[k], 2));
            }
    offt_c2c_3d(s->phik, N, N, N, +1);
    for (size_t i = 0; i < n3; ++i) s->phik[i] /= (double)(N * N * N);
    write_vg(s);
    /* psi build src/gadget_IC.h:659-670 */
    const double uc = pow(H_LITTLE, 2) * pow(1e3, 3);
    const double kf = s->mfdm / pow(C_LIGHT, 2) / HBAR;
    for (size_t i = 0; i < n3; ++i)
        s->wfc[i] = 1.225 * csqrt(s->wfc[i] * uc / s->mfdm_solar) * cexp(kf * s->phik[i] * I);
    free(xg);
    free(vy);
    free(vz);
    return 0;
}
