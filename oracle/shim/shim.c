/*
 * oracle/shim/shim.c -- single-rank MPI, FFTW3(-MPI) and GSL-qags stand-ins
 * linked into the checker binary oracle/_ref/BECMPI_ref.  TEST INFRASTRUCTURE
 * ONLY: the reference sources are compiled unmodified where they lie; these
 * functions only supply the third-party libraries they were written against.
 */
#define _GNU_SOURCE
#include <fcntl.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>
#include <unistd.h>

#include "../fft64.h"
#include "../qags.h"
#include "fftw3-mpi.h"
#include "gsl/gsl_integration.h"
#include "mpi.h"

/* ------------------------------------------------------------------ MPI -- */

static size_t dt_size(MPI_Datatype dt) {
    switch (dt) {
        case MPI_CHAR: return 1;
        case MPI_INT: return sizeof(int);
        case MPI_FLOAT: return sizeof(float);
        case MPI_DOUBLE: return sizeof(double);
        case MPI_LONG_LONG: return sizeof(long long);
        default:
            fprintf(stderr, "mpi shim: unknown datatype %d\n", dt);
            abort();
    }
}

int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }

/* Timestep_criteria makes exactly two Allreduce calls per step
 * (src/CosmoBEC_MPI.cpp:29-30); with IFDM_SHIM_TIMING=<file> each call appends
 * a CLOCK_MONOTONIC timestamp, which times the reference's own step loop. */
static void shim_timestamp(void) {
    static FILE *tf = NULL;
    static int checked = 0;
    if (!checked) {
        checked = 1;
        const char *path = getenv("IFDM_SHIM_TIMING");
        if (path && *path) tf = fopen(path, "w");
    }
    if (tf) {
        struct timespec ts;
        clock_gettime(CLOCK_MONOTONIC, &ts);
        fprintf(tf, "%lld.%09ld\n", (long long)ts.tv_sec, ts.tv_nsec);
        fflush(tf);
    }
}

int MPI_Allreduce(const void *sendbuf, void *recvbuf, int count, MPI_Datatype dt, MPI_Op op, MPI_Comm c) {
    (void)op; (void)c;
    shim_timestamp();
    if (sendbuf != recvbuf) memmove(recvbuf, sendbuf, (size_t)count * dt_size(dt));
    return 0;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype dt, int root, MPI_Comm c) {
    (void)buf; (void)count; (void)dt; (void)root; (void)c;
    return 0;
}

int MPI_Scatterv(const void *sendbuf, const int sendcounts[], const int displs[], MPI_Datatype sendtype,
                 void *recvbuf, int recvcount, MPI_Datatype recvtype, int root, MPI_Comm c) {
    (void)sendcounts; (void)recvtype; (void)root; (void)c;
    if (recvcount <= 0) return 0;
    const size_t es = dt_size(sendtype);
    memmove(recvbuf, (const char *)sendbuf + (size_t)displs[0] * es, (size_t)recvcount * es);
    return 0;
}

/* point-to-point to self: Irecv posts, Isend completes the matching post */
typedef struct { void *buf; size_t bytes; int tag; int done; } shim_recv;
static shim_recv g_recv[16];
static int g_nrecv = 0;

int MPI_Irecv(void *buf, int count, MPI_Datatype dt, int source, int tag, MPI_Comm c, MPI_Request *req) {
    (void)source; (void)c;
    if (g_nrecv >= 16) { fprintf(stderr, "mpi shim: too many receives\n"); abort(); }
    g_recv[g_nrecv].buf = buf;
    g_recv[g_nrecv].bytes = (size_t)count * dt_size(dt);
    g_recv[g_nrecv].tag = tag;
    g_recv[g_nrecv].done = 0;
    *req = g_nrecv++;
    return 0;
}

int MPI_Isend(const void *buf, int count, MPI_Datatype dt, int dest, int tag, MPI_Comm c, MPI_Request *req) {
    (void)dest; (void)c;
    const size_t bytes = (size_t)count * dt_size(dt);
    for (int i = 0; i < g_nrecv; ++i) {
        if (!g_recv[i].done && g_recv[i].tag == tag) {
            memcpy(g_recv[i].buf, buf, bytes < g_recv[i].bytes ? bytes : g_recv[i].bytes);
            g_recv[i].done = 1;
            *req = -1;
            return 0;
        }
    }
    fprintf(stderr, "mpi shim: send to self with no posted receive (tag %d)\n", tag);
    abort();
}

int MPI_Waitall(int count, MPI_Request reqs[], MPI_Status *st) {
    (void)count; (void)reqs; (void)st;
    g_nrecv = 0;
    return 0;
}

struct ifdm_shim_file {
    int fd;
    long long disp;
    long long pos; /* absolute byte offset of the (individual == shared) pointer */
};

int MPI_File_open(MPI_Comm c, const char *filename, int amode, MPI_Info info, MPI_File *fh) {
    (void)c; (void)info;
    int flags = 0;
    if (amode & MPI_MODE_RDONLY) flags = O_RDONLY;
    else if (amode & MPI_MODE_WRONLY) flags = O_WRONLY;
    else flags = O_RDWR;
    if (amode & MPI_MODE_CREATE) flags |= O_CREAT;
    int fd = open(filename, flags, 0644);
    if (fd < 0) return 1;
    struct ifdm_shim_file *f = (struct ifdm_shim_file *)malloc(sizeof(*f));
    f->fd = fd;
    f->disp = 0;
    f->pos = 0;
    if (amode & MPI_MODE_APPEND) {
        struct stat sb;
        fstat(fd, &sb);
        f->pos = (long long)sb.st_size;
    }
    *fh = f;
    return 0;
}

int MPI_File_close(MPI_File *fh) {
    if (fh && *fh) {
        close((*fh)->fd);
        free(*fh);
        *fh = NULL;
    }
    return 0;
}

int MPI_File_set_view(MPI_File fh, MPI_Offset disp, MPI_Datatype etype, MPI_Datatype filetype,
                      const char *datarep, MPI_Info info) {
    (void)etype; (void)filetype; (void)datarep; (void)info;
    fh->disp = disp;
    fh->pos = disp; /* set_view resets the file pointers to the start of the view */
    return 0;
}

static int shim_write(MPI_File fh, const void *buf, size_t bytes) {
    const char *p = (const char *)buf;
    while (bytes) {
        ssize_t w = pwrite(fh->fd, p, bytes, (off_t)fh->pos);
        if (w <= 0) return 1;
        p += w;
        fh->pos += w;
        bytes -= (size_t)w;
    }
    return 0;
}

int MPI_File_write_all(MPI_File fh, const void *buf, int count, MPI_Datatype dt, MPI_Status *st) {
    (void)st;
    return shim_write(fh, buf, (size_t)count * dt_size(dt));
}

int MPI_File_write_ordered(MPI_File fh, const void *buf, int count, MPI_Datatype dt, MPI_Status *st) {
    (void)st;
    return shim_write(fh, buf, (size_t)count * dt_size(dt));
}

int MPI_File_read(MPI_File fh, void *buf, int count, MPI_Datatype dt, MPI_Status *st) {
    (void)st;
    size_t bytes = (size_t)count * dt_size(dt);
    char *p = (char *)buf;
    while (bytes) {
        ssize_t r = pread(fh->fd, p, bytes, (off_t)fh->pos);
        if (r <= 0) return 1;
        p += r;
        fh->pos += r;
        bytes -= (size_t)r;
    }
    return 0;
}

int MPI_File_seek(MPI_File fh, MPI_Offset offset, int whence) {
    if (whence == MPI_SEEK_SET) fh->pos = fh->disp + offset;
    else if (whence == MPI_SEEK_CUR) fh->pos += offset;
    else {
        struct stat sb;
        fstat(fh->fd, &sb);
        fh->pos = (long long)sb.st_size + offset;
    }
    return 0;
}

/* ----------------------------------------------------------------- FFTW -- */

enum { SHIM_C2C = 1, SHIM_R2C = 2, SHIM_C2R = 3, SHIM_UNSUPPORTED = 4 };

struct ifdm_shim_plan {
    int kind;
    int n0, n1, n2;
    void *in, *out;
    int sign;
};

static fftw_plan make_plan(int kind, int n0, int n1, int n2, void *in, void *out, int sign) {
    fftw_plan p = (fftw_plan)malloc(sizeof(*p));
    p->kind = kind;
    p->n0 = n0; p->n1 = n1; p->n2 = n2;
    p->in = in; p->out = out;
    p->sign = sign;
    return p;
}

void fftw_mpi_init(void) {}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int n) { (void)n; }
void fftw_destroy_plan(fftw_plan p) { free(p); }

fftw_plan fftw_mpi_plan_dft_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in, fftw_complex *out,
                               MPI_Comm c, int sign, unsigned flags) {
    (void)c; (void)flags;
    return make_plan(SHIM_C2C, (int)n0, (int)n1, (int)n2, in, out, sign);
}
fftw_plan fftw_mpi_plan_dft_r2c_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, double *in, fftw_complex *out,
                                   MPI_Comm c, unsigned flags) {
    (void)c; (void)flags;
    return make_plan(SHIM_R2C, (int)n0, (int)n1, (int)n2, in, out, -1);
}
fftw_plan fftw_mpi_plan_dft_c2r_3d(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t n2, fftw_complex *in, double *out,
                                   MPI_Comm c, unsigned flags) {
    (void)c; (void)flags;
    return make_plan(SHIM_C2R, (int)n0, (int)n1, (int)n2, in, out, +1);
}
fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags;
    return make_plan(SHIM_C2C, n0, n1, n2, in, out, sign);
}
fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags;
    return make_plan(SHIM_C2C, 1, n0, n1, in, out, sign);
}
fftw_plan fftw_plan_dft_1d(int n, fftw_complex *in, fftw_complex *out, int sign, unsigned flags) {
    (void)flags;
    return make_plan(SHIM_C2C, 1, 1, n, in, out, sign);
}
/* unpadded serial real transforms: only named by dead helpers in src/matlib.h */
fftw_plan fftw_plan_dft_r2c_1d(int n, double *in, fftw_complex *out, unsigned f) {
    (void)f; return make_plan(SHIM_UNSUPPORTED, 1, 1, n, in, out, -1);
}
fftw_plan fftw_plan_dft_c2r_1d(int n, fftw_complex *in, double *out, unsigned f) {
    (void)f; return make_plan(SHIM_UNSUPPORTED, 1, 1, n, in, out, 1);
}
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned f) {
    (void)f; return make_plan(SHIM_UNSUPPORTED, 1, n0, n1, in, out, -1);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned f) {
    (void)f; return make_plan(SHIM_UNSUPPORTED, 1, n0, n1, in, out, 1);
}

void fftw_execute(const fftw_plan p) {
    const size_t n = (size_t)p->n0 * p->n1 * p->n2;
    switch (p->kind) {
        case SHIM_C2C:
            if (p->in != p->out) memcpy(p->out, p->in, n * sizeof(ocplx));
            offt_c2c_3d((ocplx *)p->out, p->n0, p->n1, p->n2, p->sign);
            break;
        case SHIM_R2C:
            offt_r2c_3d((const double *)p->in, (ocplx *)p->out, p->n0, p->n1, p->n2, 2 * (p->n2 / 2 + 1));
            break;
        case SHIM_C2R:
            offt_c2r_3d((ocplx *)p->in, (double *)p->out, p->n0, p->n1, p->n2, 2 * (p->n2 / 2 + 1));
            break;
        default:
            fprintf(stderr, "fftw shim: unpadded serial real transforms are not provided\n");
            abort();
    }
}

/* ------------------------------------------------------------------ GSL -- */

gsl_integration_workspace *gsl_integration_workspace_alloc(size_t n) {
    gsl_integration_workspace *w = (gsl_integration_workspace *)malloc(sizeof(*w));
    w->limit = n;
    return w;
}
void gsl_integration_workspace_free(gsl_integration_workspace *w) { free(w); }

int gsl_integration_qags(const gsl_function *f, double a, double b, double epsabs, double epsrel, size_t limit,
                         gsl_integration_workspace *w, double *result, double *abserr) {
    (void)w;
    return oq_qags((oq_fn)f->function, f->params, a, b, epsabs, epsrel, (int)limit, result, abserr);
}
