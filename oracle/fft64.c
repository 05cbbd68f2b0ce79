/*
 * oracle/fft64.c -- FP64 Stockham FFT for the CPU oracle (test infrastructure
 * only; see fft64.h for the contract it restates).
 */
#include "fft64.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define OFFT_MAXF 40

typedef struct {
    int n;
    int nf;
    int f[OFFT_MAXF];
    ocplx *tw; /* tw[m] = exp(-2 pi i m / n), m = 0..n-1 */
} offt_plan;

#define OFFT_CACHE 32
static offt_plan *g_plans[OFFT_CACHE];
static int g_nplans = 0;

static offt_plan *plan_build(int n) {
    offt_plan *p = (offt_plan *)calloc(1, sizeof(offt_plan));
    p->n = n;
    int m = n;
    /* radix-4 first, then 2, 3, 5, then any remaining primes */
    while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
    while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
    while (m % 3 == 0) { p->f[p->nf++] = 3; m /= 3; }
    while (m % 5 == 0) { p->f[p->nf++] = 5; m /= 5; }
    for (int q = 7; m > 1; q += 2)
        while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
    p->tw = (ocplx *)malloc(sizeof(ocplx) * (size_t)n);
    const long double twopi = 6.283185307179586476925286766559005768L;
    for (int i = 0; i < n; ++i) {
        long double ang = -twopi * (long double)i / (long double)n;
        p->tw[i] = (double)cosl(ang) + I * (double)sinl(ang);
    }
    return p;
}

/* Plans are created single-threaded (callers create before parallel loops). */
static offt_plan *plan_get(int n) {
    for (int i = 0; i < g_nplans; ++i)
        if (g_plans[i]->n == n) return g_plans[i];
    offt_plan *p = plan_build(n);
    if (g_nplans < OFFT_CACHE) g_plans[g_nplans++] = p;
    return p;
}

static inline ocplx tw_get(const offt_plan *p, long idx, int sign) {
    ocplx w = p->tw[idx % p->n];
    return sign < 0 ? w : conj(w);
}

/* One Stockham pass: radix R, Ns = product of previous radices. */
static void stockham_pass(const offt_plan *p, int R, int Ns, const ocplx *x, ocplx *y, int sign) {
    const int n = p->n;
    const int nr = n / R;
    const int span = Ns * R;
    const int tstep = n / span; /* twiddle index step for exp(-2 pi i k r / span) */
    ocplx v[64];
    ocplx *vv = v;
    ocplx *big = NULL;
    if (R > 64) { big = (ocplx *)malloc(sizeof(ocplx) * (size_t)R); vv = big; }
    for (int j = 0; j < nr; ++j) {
        const int k = j % Ns;
        for (int r = 0; r < R; ++r) {
            ocplx a = x[j + r * nr];
            if (k != 0 && r != 0) a *= tw_get(p, (long)k * r * tstep, sign);
            vv[r] = a;
        }
        /* radix-R DFT in registers */
        if (R == 2) {
            ocplx a0 = vv[0], a1 = vv[1];
            vv[0] = a0 + a1; vv[1] = a0 - a1;
        } else if (R == 4) {
            ocplx a0 = vv[0], a1 = vv[1], a2 = vv[2], a3 = vv[3];
            ocplx s02 = a0 + a2, d02 = a0 - a2, s13 = a1 + a3, d13 = a1 - a3;
            /* multiply d13 by -i*sign... forward (sign -1): -i ; backward: +i */
            ocplx rot = (sign < 0) ? (cimag(d13) - I * creal(d13)) : (-cimag(d13) + I * creal(d13));
            vv[0] = s02 + s13;
            vv[2] = s02 - s13;
            vv[1] = d02 + rot;
            vv[3] = d02 - rot;
        } else {
            /* direct DFT of length R using the plan's table: exp(-2 pi i m / R) = tw[m * n / R] */
            ocplx out[64];
            ocplx *o = out;
            ocplx *obig = NULL;
            if (R > 64) { obig = (ocplx *)malloc(sizeof(ocplx) * (size_t)R); o = obig; }
            const int step = n / R;
            for (int s = 0; s < R; ++s) {
                ocplx acc = vv[0];
                for (int r = 1; r < R; ++r) acc += vv[r] * tw_get(p, (long)((r * s) % R) * step, sign);
                o[s] = acc;
            }
            for (int s = 0; s < R; ++s) vv[s] = o[s];
            free(obig);
        }
        const int base = (j / Ns) * span + k;
        for (int r = 0; r < R; ++r) y[base + r * Ns] = vv[r];
    }
    free(big);
}

/* Transform one contiguous line in place; work has n entries. */
static void line_fft(const offt_plan *p, ocplx *line, ocplx *work, int sign) {
    ocplx *src = line, *dst = work;
    int Ns = 1;
    for (int s = 0; s < p->nf; ++s) {
        stockham_pass(p, p->f[s], Ns, src, dst, sign);
        Ns *= p->f[s];
        ocplx *t = src; src = dst; dst = t;
    }
    if (src != line) memcpy(line, src, sizeof(ocplx) * (size_t)p->n);
}

void offt_c2c_1d(ocplx *line, int n, int sign) {
    offt_plan *p = plan_get(n);
    ocplx *w = (ocplx *)malloc(sizeof(ocplx) * (size_t)n);
    line_fft(p, line, w, sign);
    free(w);
}

int offt_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/*
 * Transform along one axis: lines are a[o*ostride + i + m*stride], m = 0..len-1,
 * for o in [0,nouter), i in [0,ninner).  Lines adjacent in i are gathered in
 * blocks of B so strided axes read whole cache lines.
 */
static void axis_fft(ocplx *a, int len, long stride, int nouter, long ostride, int ninner, int sign) {
    offt_plan *p = plan_get(len);
    const int B = (stride == 1) ? 1 : 8;
    const int nblk = (ninner + B - 1) / B;
    const long total = (long)nouter * nblk;
#pragma omp parallel
    {
        ocplx *buf = (ocplx *)malloc(sizeof(ocplx) * (size_t)len * B);
        ocplx *work = (ocplx *)malloc(sizeof(ocplx) * (size_t)len);
#pragma omp for schedule(static)
        for (long t = 0; t < total; ++t) {
            const int o = (int)(t / nblk);
            const int i0 = (int)(t % nblk) * B;
            const int nb = (ninner - i0 < B) ? (ninner - i0) : B;
            ocplx *base = a + o * ostride + i0;
            if (stride == 1) {
                line_fft(p, base, work, sign);
                continue;
            }
            for (int m = 0; m < len; ++m)
                for (int b = 0; b < nb; ++b) buf[b * len + m] = base[m * stride + b];
            for (int b = 0; b < nb; ++b) line_fft(p, buf + b * len, work, sign);
            for (int m = 0; m < len; ++m)
                for (int b = 0; b < nb; ++b) base[m * stride + b] = buf[b * len + m];
        }
        free(buf);
        free(work);
    }
}

void offt_c2c_3d(ocplx *a, int n0, int n1, int n2, int sign) {
    plan_get(n0); plan_get(n1); plan_get(n2);
    /* last axis (contiguous) */
    axis_fft(a, n2, 1, n0 * n1, n2, 1, sign);
    /* middle axis */
    axis_fft(a, n1, n2, n0, (long)n1 * n2, n2, sign);
    /* first axis */
    axis_fft(a, n0, (long)n1 * n2, n1, n2, n2, sign);
}

void offt_r2c_3d(const double *in, ocplx *out, int n0, int n1, int n2, int in_pitch) {
    const int nh = n2 / 2 + 1;
    offt_plan *p = plan_get(n2);
    plan_get(n0); plan_get(n1);
    const long lines = (long)n0 * n1;
#pragma omp parallel
    {
        ocplx *line = (ocplx *)malloc(sizeof(ocplx) * (size_t)n2);
        ocplx *work = (ocplx *)malloc(sizeof(ocplx) * (size_t)n2);
#pragma omp for schedule(static)
        for (long l = 0; l < lines; ++l) {
            const double *src = in + l * in_pitch;
            for (int k = 0; k < n2; ++k) line[k] = src[k];
            line_fft(p, line, work, -1);
            ocplx *dst = out + l * nh;
            for (int k = 0; k < nh; ++k) dst[k] = line[k];
        }
        free(line);
        free(work);
    }
    axis_fft(out, n1, nh, n0, (long)n1 * nh, nh, -1);
    axis_fft(out, n0, (long)n1 * nh, n1, nh, nh, -1);
}

void offt_c2r_3d(ocplx *in, double *out, int n0, int n1, int n2, int out_pitch) {
    const int nh = n2 / 2 + 1;
    offt_plan *p = plan_get(n2);
    plan_get(n0); plan_get(n1);
    axis_fft(in, n0, (long)n1 * nh, n1, nh, nh, +1);
    axis_fft(in, n1, nh, n0, (long)n1 * nh, nh, +1);
    const long lines = (long)n0 * n1;
#pragma omp parallel
    {
        ocplx *line = (ocplx *)malloc(sizeof(ocplx) * (size_t)n2);
        ocplx *work = (ocplx *)malloc(sizeof(ocplx) * (size_t)n2);
#pragma omp for schedule(static)
        for (long l = 0; l < lines; ++l) {
            const ocplx *src = in + l * nh;
            line[0] = creal(src[0]);
            for (int k = 1; k < nh; ++k) line[k] = src[k];
            if (n2 % 2 == 0) line[n2 / 2] = creal(src[n2 / 2]);
            for (int k = nh; k < n2; ++k) line[k] = conj(src[n2 - k]);
            line_fft(p, line, work, +1);
            double *dst = out + l * out_pitch;
            for (int k = 0; k < n2; ++k) dst[k] = creal(line[k]);
        }
        free(line);
        free(work);
    }
}
