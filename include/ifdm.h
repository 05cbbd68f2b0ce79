/*
 * include/ifdm.h -- C ABI of libifdm_b200.so, the B200 (sm_100a) build of
 * IFDM_Code's leap-frog pseudo-spectral Schroedinger-Poisson step.
 *
 * The reference has no library interface: its drop-in surface is the
 * executable (`BECMPI.o mfdm g xmax res t_write t_stop ti opath icpath rerun`,
 * src/CosmoBEC_MPI.cpp:313-379), the Gadget IC chunk files
 * (src/gadget_IC.h:259-353), the snapshot files (src/write3D.h:7-97) and
 * stdout.  Each entry point below names the reference function it replaces.
 * Paths cited are relative to the reference project.
 *
 * Conventions
 *  - Every function returns IFDM_OK (0) or a negative IFDM_ERR_* code and
 *    never exits the process; ifdm_last_error() gives the message.
 *  - Host arrays are caller-owned.  psi is N^3 complex128 as interleaved
 *    (re, im) doubles, x slowest and z fastest (the reference's
 *    opr.wfc[k + N*(j + N*i)], src/CosmoBEC_MPI.cpp:133).
 *  - A context owns its device buffers and CUDA stream; one host thread at a
 *    time may use a context.
 */
#ifndef IFDM_H
#define IFDM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define IFDM_OK 0
#define IFDM_ERR_ARGS (-1)        /* bad argument count / value */
#define IFDM_ERR_CUDA (-2)        /* CUDA runtime error */
#define IFDM_ERR_IO (-3)          /* missing or truncated file */
#define IFDM_ERR_BOXSIZE (-4)     /* IC box differs from 2*xmax (src/gadget_IC.h:309-314) */
#define IFDM_ERR_UNSUPPORTED (-5) /* grid size without a compiled plan */
#define IFDM_ERR_STATE (-6)       /* call out of order (e.g. step before a psi exists) */
#define IFDM_ERR_DEVICE (-7)      /* a device-side check failed (bounded wait, quadrature limit) */

/* FP64: complex128 state, FP64 arithmetic (the drop-in).
 * FP32: complex64 state, FP32 FFTs/kick/drift; FP64 only for the phase
 *       arguments (reduced mod 2 pi), twiddle generation, reductions and the
 *       Poisson mean.
 * MIXED: complex64 state in HBM, FP64 arithmetic inside every pass, FP32
 *       stores rounded stochastically so rounding errors do not repeat
 *       from step to step. */
enum ifdm_precision { IFDM_FP64 = 0, IFDM_FP32 = 1, IFDM_MIXED = 2 };
/* IC deposit: REF1 reproduces the reference run on one MPI rank (particles in
 * the last half cell deposited twice, one zero particle per chunk at the
 * origin: src/gadget_IC.h:431-448,496-510); EXACT deposits each particle once
 * (what the reference does on many ranks, apart from its rank-boundary
 * off-by-one at src/gadget_IC.h:434-435). */
enum ifdm_ic_mode { IFDM_IC_REF1 = 0, IFDM_IC_EXACT = 1 };

/* The reference's 10 run-time parameters (src/CosmoBEC_MPI.cpp:329-339,
 * README.md:8-21) plus B200 options. */
typedef struct ifdm_params {
    double mfdm;       /* particle mass [eV]                      argv[1] */
    double g;          /* self-interaction [eV cm^3]              argv[2] */
    double xmax;       /* half box [Mpc/h]                        argv[3] */
    int res;           /* grid points per axis                    argv[4] */
    int t_write;       /* snapshot period [steps]                 argv[5] */
    int t_stop;        /* last step (exclusive)                   argv[6] */
    int ti;            /* first step / rerun snapshot number      argv[7] */
    const char *opath; /* output prefix (trailing '/')            argv[8] */
    const char *icpath;/* IC prefix, or snapshot dir when rerun   argv[9] */
    int rerun;         /* 1: start from <icpath>output<ti>.dat    argv[10] */
    int precision;     /* enum ifdm_precision; IFDM_FP64 is the drop-in */
    int stan;          /* 1: snapshot state machine of src/CosmoBEC_MPI_stan.cpp */
    int ic_mode;       /* enum ifdm_ic_mode */
    int device;        /* CUDA device ordinal */
    int verbose;       /* 1: print the reference's per-step stdout lines */
} ifdm_params;

/* Scalars of the time integration after the latest step. */
typedef struct ifdm_state {
    double a;          /* scale factor (par.ai) */
    double dt_KE, dt_PE, dt_QI; /* integrated step weights (src/CosmoBEC_MPI.cpp:66-68) */
    double max_phi;    /* max |phi| over the reference's scan window */
    double max_rho;    /* max |psi|^2 */
    double rhoc;       /* mean density subtracted in the Poisson source */
    long long steps;   /* leap-frog steps taken by this context */
    int criterion;     /* 3: kinetic, 2: potential, 4: self-interaction limited */
    int device_error;  /* nonzero when a device-side check failed */
} ifdm_state;

typedef struct ifdm_ctx ifdm_ctx;

/* Fill defaults: FP64, stan 0, IFDM_IC_REF1, device 0, verbose 0. */
void ifdm_params_default(ifdm_params *p);

/* Parse argv exactly as main() does (src/CosmoBEC_MPI.cpp:324-340): argc must
 * be 11; numbers via atof/atoi.  The strings point into argv. */
int ifdm_params_from_argv(int argc, char **argv, ifdm_params *p);

/* Allocate a context on p->device (Params/Operators, src/struct3D.h:17-125). */
int ifdm_create(const ifdm_params *p, ifdm_ctx **out);
void ifdm_destroy(ifdm_ctx *ctx);
const char *ifdm_last_error(const ifdm_ctx *ctx);
/* 1 if `res` has a compiled FFT plan for `precision`: 16, 32, 48, 64, 96,
 * 128, 256, 512 and 1024 (the reference's production grid, job.sh:24) in
 * IFDM_FP64 and IFDM_FP32; IFDM_MIXED up to 512.  ifdm_load_ic deposits at most
 * 2^28 particles (512^3); larger boxes start from ifdm_set_psi or a snapshot. */
int ifdm_supported_res(int res, int precision);

/* Gadget_IC_Generator (src/gadget_IC.h:686-707): read <icpath>.0..3, CIC
 * deposit, velocity-divergence phase, psi = 1.225 sqrt(rho h^2 1e9/m) e^{i..};
 * also writes <opath>voutput.dat (src/write3D.h:24-53). */
int ifdm_load_ic(ifdm_ctx *ctx);
/* read_rerun (src/gadget_IC.h:709-750): psi and a from <icpath>output<t>.dat. */
int ifdm_load_snapshot(ifdm_ctx *ctx, int t);
/* Start from a host psi (complex128, N^3) at scale factor a; rhoc <= 0 means
 * the constant 3.51059e10 that read_rerun uses. */
int ifdm_set_psi(ifdm_ctx *ctx, const double *psi, double a, double rhoc);
/* psi after the latest full step (the pending second half-kick applied). */
int ifdm_get_psi(ifdm_ctx *ctx, double *psi);
/* phi (N^3 doubles) of the current density. */
int ifdm_get_phi(ifdm_ctx *ctx, double *phi);
int ifdm_get_state(ifdm_ctx *ctx, ifdm_state *out);
/* Power spectrum of the density contrast delta = |psi|^2/<|psi|^2> - 1 of the
 * current state, computed on the device (an extension: the reference has no
 * such output).  Bin b holds the modes with edges[b] <= |kappa| < edges[b+1],
 * kappa the integer wave vector (-N/2..N/2-1 per axis); edges = NULL gives
 * nbins log-spaced bins from 1 to N/2.  Outputs (each may be NULL; nbins
 * entries): k = mean 2 pi |kappa| / L of the bin's modes [1/Mpc], pk =
 * <|delta_k|^2> L^3 / N^6 [Mpc^3] with delta_k the unnormalised forward DFT,
 * modes = modes per bin; mean_rho = <|psi|^2>.  L = 2 xmax (Mpc).
 * nbins <= 64.  Every sum has a fixed order: repeated calls agree bit for bit. */
int ifdm_power_spectrum(ifdm_ctx *ctx, int nbins, const double *edges, double *k, double *pk, long long *modes,
                        double *mean_rho);
/* Grid means of the current state for energy bookkeeping, computed on the
 * device (an extension: the reference has no such output), in the natural
 * units of ifdm_get_psi / ifdm_get_phi: the energy densities are
 * hbar^2/(2m) mean_grad2 (kinetic), m mean_phi_rho / 2 (gravitational) and
 * g mean_rho2 / 2 (self-interaction).  Fixed-order sums. */
typedef struct ifdm_energies {
    double mean_rho;     /* <|psi|^2> */
    double mean_grad2;   /* <|grad psi|^2>, spectral derivative, k = pi kappa / xmax [1/Mpc] */
    double mean_phi_rho; /* <phi |psi|^2> */
    double mean_rho2;    /* <|psi|^4> */
} ifdm_energies;
int ifdm_get_energies(ifdm_ctx *ctx, ifdm_energies *out);

/* Simulation (src/CosmoBEC_MPI.cpp:183-310): steps ti..t_stop-1 with the
 * adaptive timestep, the snapshot state machine and its early stops. */
int ifdm_run(ifdm_ctx *ctx);
/* Fixed-step mode: nsteps leap-frog steps, no snapshots or stops, the
 * selected timestep multiplied by dt_scale (1.0 = the reference's rule).
 * Asynchronous on the context's stream. */
int ifdm_step(ifdm_ctx *ctx, int nsteps, double dt_scale);
/* writeall (src/write3D.h:86-97): <opath>output<t>.dat of the current state;
 * the file is complete on return. */
int ifdm_write_snapshot(ifdm_ctx *ctx, int t);
/* Snapshot streaming (an extension; the reference's writeall blocks the
 * loop).  With streaming on (the default) a snapshot costs the compute stream
 * one kernel into a device staging buffer; the copy to pinned host memory runs
 * on a copy stream and a writer thread writes the file while the steps go on.
 * The bytes are those of the synchronous path.  ifdm_run returns only after
 * every file is written.
 *   ifdm_write_snapshot_async  queue <opath>output<t>.dat and return
 *   ifdm_flush_snapshots       wait for queued files; first write error
 *   ifdm_set_snapshot_streaming  0: gather and write inside the call, as
 *                              the reference does (flushes first)
 *   ifdm_snapshots_written     files written by the streaming writer */
int ifdm_write_snapshot_async(ifdm_ctx *ctx, int t);
int ifdm_flush_snapshots(ifdm_ctx *ctx);
int ifdm_set_snapshot_streaming(ifdm_ctx *ctx, int on);
long long ifdm_snapshots_written(const ifdm_ctx *ctx);
int ifdm_synchronize(ifdm_ctx *ctx);
/* The context's cudaStream_t (as void*). */
void *ifdm_stream(ifdm_ctx *ctx);

/* Average device time per leap-frog step of each fused pass over `nsteps`
 * fixed-mode steps (CUDA events on the context's stream).  ms_out receives
 * up to `cap` entries; names_out (optional) gets static pass names.
 * Returns the number of passes. */
int ifdm_profile_passes(ifdm_ctx *ctx, int nsteps, double dt_scale, double *ms_out, const char **names_out,
                        int cap);
/* Algorithmic HBM bytes one step moves, per pass (same order as above). */
int ifdm_pass_bytes(ifdm_ctx *ctx, double *bytes_out, int cap);

/* Adjoint of the split step (no counterpart in the reference, which has no
 * derivatives).  ifdm_record_steps runs nsteps fixed-mode steps like
 * ifdm_step and keeps what the adjoint needs: the coefficients of every step
 * and a checkpoint of (psi, phi) every checkpoint_every steps.
 * ifdm_adjoint then maps g_final = dL/dRe psi_final + i dL/dIm psi_final (psi
 * as ifdm_get_psi returns it) to the same derivative with respect to the psi
 * the recording started from, replaying each segment forward from its
 * checkpoint and sweeping it backwards: g' = U^H g, w = Im(conj(g') K psi),
 * g = exp(i theta) g' + 2 (a phi_s[w] + b w) psi.  The Delta-t schedule is
 * the recorded one.  Both arrays are complex128 N^3, host or device.  The
 * replay overwrites the context's state: set a psi again before stepping. */
int ifdm_record_steps(ifdm_ctx *ctx, int nsteps, double dt_scale, int checkpoint_every);
int ifdm_adjoint(ifdm_ctx *ctx, const double *g_final, double *g0);

/* Batches: many independent boxes advanced together (no counterpart in the
 * reference, which runs one box per MPI job).  A batch groups contexts made
 * by ifdm_create on one device with one precision, res 16, 32, 48, 64, 96 or
 * 128 (sizes may differ), each with a state (ifdm_set_psi, ifdm_load_ic or
 * ifdm_load_snapshot).  ifdm_batch_step advances every box by nsteps
 * fixed-mode steps, box b with step scale dt_scale[b] (as ifdm_step), in one
 * replay of one captured CUDA graph: the boxes of each grid size share one
 * persistent kernel (or, the other schedule, one launch per phase), sizes run
 * side by side, with the same passes and tile shapes as a one-box run of
 * these sizes.  Contexts are read as usual afterwards (ifdm_get_psi,
 * ifdm_get_state) and must outlive the batch.  ifdm_batch_tune times launch
 * shapes on trial_steps steps (saving and restoring every box's state) and
 * keeps the fastest: the schedule, CTAs per SM, the group size of the item
 * order (all boxes in lock step, or a few at a time for L2 reuse) and the
 * radix plan of each grid size. */
typedef struct ifdm_batch ifdm_batch;
typedef struct ifdm_batch_tuning {
    int mode;           /* 0: one persistent kernel per grid size, 1: one launch per phase and size */
    int blocks_per_sm;  /* persistent CTAs per SM */
    int group;          /* boxes per group of the item order, 0 = all boxes */
    int plan[6];        /* radix-plan variant (0, 1) for res 16, 32, 48, 64, 96, 128 */
    double ms_per_step; /* ifdm_batch_tune: measured time of one batch step */
} ifdm_batch_tuning;
int ifdm_batch_create(ifdm_ctx *const *ctxs, int n, ifdm_batch **out);
int ifdm_batch_step(ifdm_batch *b, int nsteps, const double *dt_scale);
int ifdm_batch_tune(ifdm_batch *b, int trial_steps, const double *dt_scale, ifdm_batch_tuning *out);
int ifdm_batch_get_tuning(ifdm_batch *b, ifdm_batch_tuning *out);
int ifdm_batch_set_tuning(ifdm_batch *b, const ifdm_batch_tuning *t);
/* Wait for the batch; IFDM_ERR_DEVICE if a dependency wait gave up. */
int ifdm_batch_synchronize(ifdm_batch *b);
/* Batched adjoint: ifdm_record_steps / ifdm_adjoint of every box, the boxes
 * side by side (one host thread and the box's own stream each, up to 16 at a
 * time), so many small boxes fill the GPU together.  dt_scale, g_final and g0
 * have one entry per box (host or device complex128 N_i^3 arrays).  Results
 * equal the boxes' own ifdm_adjoint calls bit for bit. */
int ifdm_batch_record_steps(ifdm_batch *b, int nsteps, const double *dt_scale, int checkpoint_every);
int ifdm_batch_adjoint(ifdm_batch *b, const double *const *g_final, double *const *g0);
/* Work items of one batch step and the persistent CTAs of all sizes. */
int ifdm_batch_info(ifdm_batch *b, long long *items_per_step, int *grid);
const char *ifdm_batch_last_error(const ifdm_batch *b);
void ifdm_batch_destroy(ifdm_batch *b);

/* Device-pointer transforms on the caller's stream (cudaStream_t as void*).
 * In-place unnormalised 3-D complex FFT of data[n][n][n] (complex128 when
 * precision == IFDM_FP64, complex64 otherwise; IFDM_MIXED computes in FP64);
 * sign -1 forward, +1 backward
 * -- the contract of the reference's fftw_mpi_plan_dft_3d plans
 * (src/CosmoBEC_MPI.cpp:176-177). */
int ifdm_fft3d(void *data, int n, int precision, int sign, void *stream);
/* One axis of the local step of a slab-decomposed 3-D FFT, in place on device
 * data: the reference splits the box into x-slabs of local_n0 = n/P planes per
 * MPI rank (src/struct3D.h:3-15) and its fftw_mpi plans transpose between
 * ranks (src/CosmoBEC_MPI.cpp:174-177).  Here a rank transforms z and y on
 * its x-slab [planes][n][n] (axis 2, axis 1) and x on the transposed y-slab
 * [n][planes][n] (axis 0) that an all-to-all gives it; the transposes are the
 * caller's (NCCL or gloo, ifdm_code_b200.slab).  op 1 (axis 0 only): forward
 * FFT along x, multiply by -1/(kappa^2 n^3) with the slab's global y planes
 * y0 .. y0+planes-1 (0 at kappa = 0), inverse FFT -- the Poisson multiplier of
 * src/CosmoBEC_MPI.cpp:80-119 with the three inverse normalisations folded in;
 * sign is then ignored.  planes * n must be a multiple of 16; bad arguments
 * return IFDM_ERR_ARGS. */
int ifdm_fft_slab(void *data, int n, int planes, int axis, int precision, int sign, int op, int y0, void *stream);

/* Gravitational potential of a wave function without allocating any device
 * memory.  No counterpart in the reference: it exists for callers that cannot
 * call cudaMalloc/cudaFree -- a process whose device memory is owned by
 * another allocator (a framework's caching pool), or a time-critical loop that
 * cannot afford cudaMalloc/cudaFree, which may synchronise the device.
 *   psi: device pointer, res^3 complex128 (interleaved re, im), as for
 *        ifdm_set_psi; phi: device pointer, res^3 doubles, receives the same
 *        potential ifdm_get_phi returns for that psi.  mfdm [eV] and xmax
 *        [Mpc/h, half box] as on the command line.  Runs on `stream`.
 * Scratch lives in one static device array of IFDM_STATIC_SCRATCH_BYTES that
 * every GPU loading the library holds until exit, so res is limited to
 * IFDM_STATIC_MAX_RES (16, 32, 48, 64); larger sizes return
 * IFDM_ERR_UNSUPPORTED.  All calls share that array: calls that overlap on
 * the GPU (other streams, other host threads) race and must be serialised by
 * the caller.  The first call on a device, whatever its res, does that
 * device's one-time set-up: it looks up the array's address
 * (cudaGetSymbolAddress) and sets the kernels' shared-memory attributes for
 * every supported res; make it before any stream capture.  res <= 0 or a null
 * pointer returns IFDM_ERR_ARGS. */
#define IFDM_STATIC_SCRATCH_BYTES (3u << 20)
#define IFDM_STATIC_MAX_RES 64
int ifdm_poisson_static(const double *psi, double *phi, int res, double mfdm, double xmax, void *stream);

#ifdef __cplusplus
}
#endif
#endif
