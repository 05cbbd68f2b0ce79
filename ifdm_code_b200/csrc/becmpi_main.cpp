// becmpi_main.cpp -- drop-in executable for the reference's BECMPI.o
// (main, src/CosmoBEC_MPI.cpp:313-379):
//
//   BECMPI mfdm g xmax res t_write t_stop ti opath icpath rerun
//
// Same argument parsing, unit conversions, stdout lines and exit codes, on one
// GPU instead of mpirun.  Options the reference does not have come from the
// environment so the command line stays identical:
//   IFDM_PRECISION=fp32   FP32-mixed path (default fp64, the drop-in)
//   IFDM_STAN=1           snapshot state machine of src/CosmoBEC_MPI_stan.cpp
//   IFDM_IC_MODE=exact    deposit each IC particle once (default: the
//                         reference's one-rank behaviour)
//   IFDM_DEVICE=<n>       CUDA device
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <vector>

#include "../../include/ifdm.h"

static const char *env(const char *k) {
    const char *v = std::getenv(k);
    return v ? v : "";
}

int main(int argc, char **argv) {
    ifdm_params p;
    if (ifdm_params_from_argv(argc, argv, &p) != IFDM_OK) {
        std::printf("ERROR: Arguments %d!= 11 \n", argc);
        return 0;
    }
    if (!std::strcmp(env("IFDM_PRECISION"), "fp32")) p.precision = IFDM_FP32;
    if (!std::strcmp(env("IFDM_STAN"), "1")) p.stan = 1;
    if (!std::strcmp(env("IFDM_IC_MODE"), "exact")) p.ic_mode = IFDM_IC_EXACT;
    if (*env("IFDM_DEVICE")) p.device = std::atoi(env("IFDM_DEVICE"));
    p.verbose = 1;
    const double h_0 = 0.677;
    std::printf(" Input parameters: \nmfdm=%g\ng=%g\nxmax = %g Mpc \nBoxsize = %g Mpc \nres = %d\ntwrite = %d\n"
                "timestep = %d\nti = %d\nopath = %s\n\n",
                p.mfdm, p.g, p.xmax / h_0, 2 * p.xmax / h_0, p.res, p.t_write, p.t_stop, p.ti, p.opath);
    const time_t tstart = time(nullptr);
    std::printf(" start IFDM... \n running with 1 cores \n\n");
    ifdm_ctx *ctx = nullptr;
    int rc = ifdm_create(&p, &ctx);
    if (rc != IFDM_OK) {
        std::printf("ERROR: %s\n", ifdm_last_error(ctx));
        ifdm_destroy(ctx);
        return 2;
    }
    rc = p.rerun ? ifdm_load_snapshot(ctx, p.ti) : ifdm_load_ic(ctx);
    if (rc != IFDM_OK) {
        std::printf("%s\n", ifdm_last_error(ctx));
        ifdm_destroy(ctx);
        // reference: exit(0) for IC problems (src/gadget_IC.h:313,349),
        // exit(EXIT_FAILURE) for a missing rerun snapshot (src/gadget_IC.h:729)
        if (rc == IFDM_ERR_IO && p.rerun) return EXIT_FAILURE;
        return (rc == IFDM_ERR_IO || rc == IFDM_ERR_BOXSIZE) ? 0 : 2;
    }
    {
        const size_t n3 = size_t(p.res) * p.res * p.res;
        std::vector<std::complex<double>> psi(n3);
        if (ifdm_get_psi(ctx, reinterpret_cast<double *>(psi.data())) == IFDM_OK && n3 >= 3)
            std::printf("in Simulation : (%g,%g) (%g,%g) (%g,%g) from0\n", psi[0].real(), psi[0].imag(),
                        psi[1].real(), psi[1].imag(), psi[2].real(), psi[2].imag());
    }
    rc = ifdm_run(ctx);
    if (rc != IFDM_OK) {
        std::printf("ERROR: %s\n", ifdm_last_error(ctx));
        ifdm_destroy(ctx);
        return 2;
    }
    std::printf("simulation takes:%ld seconds\n", (long)(time(nullptr) - tstart));
    ifdm_destroy(ctx);
    return 0;
}
