/*
 * oracle/ifdm_oracle.h -- CPU restatement of IFDM_Code's leap-frog
 * pseudo-spectral Schroedinger-Poisson path, FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  Imported (through ctypes) by tests/, by
 * __graft_entry__.smoke() as the checker, and by bench.py's cpu_baseline /
 * reference legs.  The product (ifdm_code_b200/) never links it.
 *
 * Every function restates the reference lines it cites (paths relative to
 * the reference project).  FFTW and GSL are replaced by oracle/fft64.c and
 * oracle/qags.c.  Two extensions beyond the reference, both off by default:
 *   - fixed-step mode (orc_run_fixed): the step body without the snapshot
 *     state machine, with the timestep multiplied by a constant C;
 *   - ORC_IC_EXACT: CIC deposit with each particle counted once (the
 *     reference, run on one rank, counts the particles of the last half cell
 *     twice and adds one particle at the origin per chunk).
 */
#ifndef IFDM_ORACLE_H
#define IFDM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_IC_REF1 = 0, ORC_IC_EXACT = 1 };

typedef struct {
    double mfdm;    /* eV                     argv[1] */
    double g_in;    /* eV cm^3                argv[2] */
    double xmax_in; /* Mpc/h, half box        argv[3] */
    int res;        /*                        argv[4] */
    int t_write;    /*                        argv[5] */
    int t_stop;     /*                        argv[6] */
    int ti;         /*                        argv[7] */
    const char *opath;  /*                    argv[8] */
    const char *icpath; /*                    argv[9] */
    int rerun;      /*                        argv[10] */
    int stan;       /* 1: state machine of src/CosmoBEC_MPI_stan.cpp */
    int ic_mode;    /* ORC_IC_REF1 / ORC_IC_EXACT */
    int verbose;
} orc_args;

typedef struct orc_sim orc_sim;

orc_sim *orc_create(const orc_args *args);
void orc_destroy(orc_sim *s);

int orc_load_ic(orc_sim *s);              /* Gadget_IC_Generator  src/gadget_IC.h:686-707 */
int orc_read_rerun(orc_sim *s, int t);    /* read_rerun           src/gadget_IC.h:709-750 */
int orc_simulation(orc_sim *s);           /* Simulation           src/CosmoBEC_MPI.cpp:183-310 */
int orc_run_fixed(orc_sim *s, int nsteps, double dt_scale);
void orc_poisson(orc_sim *s);             /* poisson              src/CosmoBEC_MPI.cpp:80-119 */
void orc_timestep(orc_sim *s, double dt_scale); /* Timestep_criteria src/CosmoBEC_MPI.cpp:19-78 */
void orc_split_op(orc_sim *s);            /* Split_op_MPI         src/CosmoBEC_MPI.cpp:121-159 */
int orc_writeall(orc_sim *s, int t);      /* writeall             src/write3D.h:86-97 */

/* state access (psi as interleaved re/im, N^3 complex, z fastest) */
int orc_set_psi(orc_sim *s, const double *psi, double a);
void orc_get_psi(const orc_sim *s, double *psi);
void orc_get_phi(const orc_sim *s, double *phi); /* N^3, unpadded */
void orc_get_vxg(const orc_sim *s, float *vx);   /* IC velocity grid (after mass weighting) */
void orc_get_theta(const orc_sim *s, double *theta); /* IC phase field phik, complex N^3 */
double orc_get_a(const orc_sim *s);
void orc_get_dts(const orc_sim *s, double *dts3); /* dt_KE, dt_PE, dt_QI */
double orc_get_rhoc(const orc_sim *s);
void orc_get_maxes(const orc_sim *s, double *maxphi_maxrho2);
int orc_num_threads(void);

/* physical constants as the reference evaluates them (src/Cosmoinput3D.h:1-22) */
void orc_constants(double *out8); /* H_0, hbar, bigG, c, Omega_m0, h_0, rhoc, cm2Mpc */

#ifdef __cplusplus
}
#endif
#endif
