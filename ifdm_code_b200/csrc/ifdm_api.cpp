// ifdm_api.cpp -- the C ABI of include/ifdm.h.
#include "../../include/ifdm.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "batch_engine.hpp"
#include "diagnostics.hpp"
#include "ic_pipeline.hpp"
#include "ic_stream.hpp"
#include "io.hpp"
#include "physics.hpp"
#include "snapshot_stream.hpp"
#include "step_engine.hpp"

using namespace ifdm;

struct ifdm_ctx {
    ifdm_params p{};
    std::string opath, icpath, err;
    int N = 0;
    // globals of main() (src/CosmoBEC_MPI.cpp:329-339) and Params (src/struct3D.h:43-87)
    double mfdm = 0, mfdm_solar = 0, g = 0, xmax = 0, dx = 0;
    std::vector<double> x;
    double a0 = 0, rhoc = 0;
    cudaStream_t stream = nullptr;
    StepEngine eng;
    bool have_psi = false;
    double *d_out = nullptr;   // complex128 N^3 device staging for outputs
    double *d_phi = nullptr;   // N^3 doubles of phi for the field means (first use)
    double *h_out = nullptr;   // pinned host staging
    size_t h_out_bytes = 0;
    bool stream_snapshots = true;  // snapshots copied and written beside the steps
    SnapshotStream snap;
};

static int fail(ifdm_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

#define CTX_CUDA(c, expr)                                                                              \
    do {                                                                                               \
        cudaError_t e_ = (expr);                                                                       \
        if (e_ != cudaSuccess) return fail(c, IFDM_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

#define CTX_STR(c, code, expr)                        \
    do {                                              \
        std::string s_ = (expr);                      \
        if (!s_.empty()) return fail(c, code, s_);    \
    } while (0)

extern "C" {

void ifdm_params_default(ifdm_params *p) {
    std::memset(p, 0, sizeof(*p));
    p->precision = IFDM_FP64;
    p->ic_mode = IFDM_IC_REF1;
    p->t_write = 1;
    p->opath = "";
    p->icpath = "";
}

int ifdm_params_from_argv(int argc, char **argv, ifdm_params *p) {
    if (argc != 11) return IFDM_ERR_ARGS;
    ifdm_params_default(p);
    p->mfdm = std::atof(argv[1]);
    p->g = std::atof(argv[2]);
    p->xmax = std::atof(argv[3]);
    p->res = std::atoi(argv[4]);
    p->t_write = (int)std::atof(argv[5]);
    p->t_stop = (int)(unsigned)std::atof(argv[6]);
    p->ti = (int)std::atof(argv[7]);
    p->opath = argv[8];
    p->icpath = argv[9];
    p->rerun = (std::atof(argv[10]) == 1) ? 1 : 0;
    return IFDM_OK;
}

int ifdm_supported_res(int res, int precision) { return supported_n(res, precision) ? 1 : 0; }

int ifdm_create(const ifdm_params *p, ifdm_ctx **out) {
    if (!p || !out) return IFDM_ERR_ARGS;
    *out = nullptr;
    std::unique_ptr<ifdm_ctx> c(new ifdm_ctx);
    c->p = *p;
    c->opath = p->opath ? p->opath : "";
    c->icpath = p->icpath ? p->icpath : "";
    c->p.opath = c->opath.c_str();
    c->p.icpath = c->icpath.c_str();
    if (p->precision != IFDM_FP64 && p->precision != IFDM_FP32 && p->precision != IFDM_MIXED) {
        *out = c.release();
        return fail(*out, IFDM_ERR_ARGS, "precision must be IFDM_FP64, IFDM_FP32 or IFDM_MIXED");
    }
    if (!supported_n(p->res, p->precision)) {
        *out = c.release();
        return fail(*out, IFDM_ERR_UNSUPPORTED,
                    "res " + std::to_string(p->res) + " has no compiled FFT plan in this precision mode");
    }
    using namespace phys;
    c->N = p->res;
    c->mfdm = p->mfdm;
    c->mfdm_solar = p->mfdm * kg2eV / kg2solar;
    c->g = p->g / (pow(cm2Mpc, 3));
    c->xmax = p->xmax / h_0;
    const unsigned res = (unsigned)p->res;
    c->dx = 2.0 * c->xmax / res;
    c->x.resize(res);
    for (size_t i = 0; i < res; ++i) c->x[i] = c->xmax / res - c->xmax + i * (2.0 * c->xmax / res);
    ifdm_ctx *raw = c.release();
    *out = raw;
    CTX_CUDA(raw, cudaSetDevice(p->device));
    CTX_CUDA(raw, cudaStreamCreateWithFlags(&raw->stream, cudaStreamNonBlocking));
    EngineConfig ec;
    ec.N = raw->N;
    ec.precision = p->precision;
    ec.mfdm = raw->mfdm;
    ec.g = raw->g;
    ec.xmax = raw->xmax;
    ec.dx = raw->dx;
    ec.mfdm_solar = raw->mfdm_solar;
    CTX_STR(raw, IFDM_ERR_CUDA, raw->eng.init(ec, raw->stream));
    return IFDM_OK;
}

void ifdm_destroy(ifdm_ctx *c) {
    if (!c) return;
    c->snap.drain();
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_out);
    cudaFree(c->d_phi);
    if (c->h_out) cudaFreeHost(c->h_out);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

const char *ifdm_last_error(const ifdm_ctx *c) { return c ? c->err.c_str() : "null context"; }

void *ifdm_stream(ifdm_ctx *c) { return c ? (void *)c->stream : nullptr; }

int ifdm_synchronize(ifdm_ctx *c) {
    if (!c) return IFDM_ERR_ARGS;
    CTX_CUDA(c, cudaStreamSynchronize(c->stream));
    return IFDM_OK;
}

static int ensure_out(ifdm_ctx *c) {
    if (!c->d_out) CTX_CUDA(c, cudaMalloc(&c->d_out, c->eng.n3() * 2 * sizeof(double)));
    return IFDM_OK;
}

int ifdm_set_psi(ifdm_ctx *c, const double *psi, double a, double rhoc) {
    if (!c || !psi) return IFDM_ERR_ARGS;
    c->a0 = a;
    c->rhoc = rhoc > 0 ? rhoc : phys::rhoc;
    cudaPointerAttributes attr{};
    const bool dev = cudaPointerGetAttributes(&attr, psi) == cudaSuccess && attr.type == cudaMemoryTypeDevice;
    cudaGetLastError();
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.load_psi(psi, dev, a, c->rhoc));
    c->have_psi = true;
    return IFDM_OK;
}

// psi of the current state into a host buffer; which: 1 snapshot kick, 2 pending kick
static bool is_device_ptr(const void *p) {
    cudaPointerAttributes attr{};
    const bool dev = cudaPointerGetAttributes(&attr, p) == cudaSuccess && attr.type == cudaMemoryTypeDevice;
    cudaGetLastError();
    return dev;
}

// psi of the current state into a host or device buffer; which: 1 snapshot kick, 2 pending kick
static int psi_to_host(ifdm_ctx *c, double *host, int which) {
    if (is_device_ptr(host)) {
        CTX_STR(c, IFDM_ERR_CUDA, c->eng.psi_out(host, which));
        CTX_CUDA(c, cudaStreamSynchronize(c->stream));
        return IFDM_OK;
    }
    // host buffer: chunked conversion and copy through the engine's own
    // staging slots (the snapshot staging buffer is not touched)
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.psi_to_host(host, which));
    return IFDM_OK;
}

int ifdm_get_psi(ifdm_ctx *c, double *psi) {
    if (!c || !psi) return IFDM_ERR_ARGS;
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    return psi_to_host(c, psi, 2);
}

int ifdm_get_phi(ifdm_ctx *c, double *phi) {
    if (!c || !phi) return IFDM_ERR_ARGS;
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    if (ensure_out(c)) return IFDM_ERR_CUDA;
    if (c->snap.ready()) CTX_STR(c, IFDM_ERR_CUDA, c->snap.before_stage(c->stream));
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.phi_out(c->d_out));
    CTX_CUDA(c, cudaMemcpyAsync(phi, c->d_out, c->eng.n3() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    CTX_CUDA(c, cudaStreamSynchronize(c->stream));
    return IFDM_OK;
}

int ifdm_power_spectrum(ifdm_ctx *c, int nbins, const double *edges, double *k, double *pk, long long *modes,
                        double *mean_rho) {
    if (!c || nbins < 1 || nbins > kMaxBins) return fail(c, IFDM_ERR_ARGS, "nbins must be 1..64");
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    if (ensure_out(c)) return IFDM_ERR_CUDA;
    if (c->snap.ready()) CTX_STR(c, IFDM_ERR_CUDA, c->snap.before_stage(c->stream));
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.psi_out(c->d_out, 2));
    CTX_STR(c, IFDM_ERR_ARGS, power_spectrum(reinterpret_cast<double2 *>(c->d_out), c->N, 2.0 * c->xmax, nbins, edges,
                                             k, pk, modes, mean_rho, c->stream));
    return IFDM_OK;
}

int ifdm_get_energies(ifdm_ctx *c, ifdm_energies *out) {
    if (!c || !out) return IFDM_ERR_ARGS;
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    if (ensure_out(c)) return IFDM_ERR_CUDA;
    if (!c->d_phi) CTX_CUDA(c, cudaMalloc(&c->d_phi, c->eng.n3() * sizeof(double)));
    if (c->snap.ready()) CTX_STR(c, IFDM_ERR_CUDA, c->snap.before_stage(c->stream));
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.phi_out(c->d_phi));
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.psi_out(c->d_out, 2));
    double m[4];
    CTX_STR(c, IFDM_ERR_CUDA, field_means(reinterpret_cast<double2 *>(c->d_out), c->d_phi, c->N, c->xmax, m, c->stream));
    out->mean_rho = m[0];
    out->mean_grad2 = m[1];
    out->mean_phi_rho = m[2];
    out->mean_rho2 = m[3];
    return IFDM_OK;
}

int ifdm_get_state(ifdm_ctx *c, ifdm_state *out) {
    if (!c || !out) return IFDM_ERR_ARGS;
    TState t{};
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.read_state(t));
    out->a = t.a;
    out->dt_KE = t.dt_KE;
    out->dt_PE = t.dt_PE;
    out->dt_QI = t.dt_QI;
    out->max_phi = t.maxphi;
    out->max_rho = t.maxrho;
    out->rhoc = c->rhoc;
    out->steps = t.steps;
    out->criterion = t.crit;
    out->device_error = t.err;
    return IFDM_OK;
}

static int write_snapshot_which(ifdm_ctx *c, int t, int which, double a) {
    const size_t n3 = c->eng.n3();
    const size_t bytes = n3 * 2 * sizeof(double);
    const double gg = c->g * (pow(phys::cm2Mpc, 3));
    if (c->stream_snapshots) {
        // psi into the device staging buffer on the compute stream; the copy
        // to the host and the file write go on beside the next steps
        if (ensure_out(c)) return IFDM_ERR_CUDA;
        CTX_STR(c, IFDM_ERR_CUDA, c->snap.init(bytes, c->p.device));
        CTX_STR(c, IFDM_ERR_CUDA, c->snap.before_stage(c->stream));
        CTX_STR(c, IFDM_ERR_CUDA, c->eng.psi_out(c->d_out, which));
        CTX_STR(c, IFDM_ERR_IO, c->snap.submit(c->stream, c->d_out, snapshot_path(c->opath, t), c->mfdm, gg, a, c->x));
        return IFDM_OK;
    }
    if (c->h_out_bytes < bytes) {
        if (c->h_out) cudaFreeHost(c->h_out);
        c->h_out = nullptr;
        c->h_out_bytes = 0;
        CTX_CUDA(c, cudaMallocHost(&c->h_out, bytes));
        c->h_out_bytes = bytes;
    }
    int rc = psi_to_host(c, c->h_out, which);
    if (rc) return rc;
    CTX_STR(c, IFDM_ERR_IO, write_snapshot(snapshot_path(c->opath, t), c->mfdm, gg, a, c->x, c->h_out, n3));
    return IFDM_OK;
}

int ifdm_write_snapshot_async(ifdm_ctx *c, int t) {
    if (!c) return IFDM_ERR_ARGS;
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    TState st{};
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.read_state(st));
    return write_snapshot_which(c, t, 2, st.steps ? st.a : c->a0);
}

int ifdm_flush_snapshots(ifdm_ctx *c) {
    if (!c) return IFDM_ERR_ARGS;
    CTX_STR(c, IFDM_ERR_IO, c->snap.drain());
    return IFDM_OK;
}

int ifdm_write_snapshot(ifdm_ctx *c, int t) {
    const int rc = ifdm_write_snapshot_async(c, t);
    return rc ? rc : ifdm_flush_snapshots(c);
}

int ifdm_set_snapshot_streaming(ifdm_ctx *c, int on) {
    if (!c) return IFDM_ERR_ARGS;
    const int rc = ifdm_flush_snapshots(c);
    if (rc) return rc;
    c->stream_snapshots = on != 0;
    return IFDM_OK;
}

long long ifdm_snapshots_written(const ifdm_ctx *c) { return c ? c->snap.written() : -1; }

int ifdm_load_snapshot(ifdm_ctx *c, int t) {
    if (!c) return IFDM_ERR_ARGS;
    const size_t n3 = c->eng.n3();
    std::vector<double> psi(2 * n3);
    double a = 0;
    std::vector<double> x;
    CTX_STR(c, IFDM_ERR_IO, read_snapshot(snapshot_path(c->icpath, t), c->N, &a, &x, psi.data()));
    c->x = x;  // read_rerun overwrites par.x (src/gadget_IC.h:735)
    return ifdm_set_psi(c, psi.data(), a, phys::rhoc);
}

int ifdm_load_ic(ifdm_ctx *c) {
    if (!c) return IFDM_ERR_ARGS;
    using namespace phys;
    const int N = c->N;
    const int tot_chunks = 4;  // src/gadget_IC.h:610
    const bool ref1 = c->p.ic_mode == IFDM_IC_REF1;
    std::vector<IcChunk> chunks;
    long np = 0;
    // headers (and ghost counts) of all chunks; a read problem in chunk k is
    // reported after chunks 0..k-1 passed their checks, as the reference's
    // chunk-by-chunk loop would
    const std::string scan_err = ic_scan_chunks(c->icpath, tot_chunks, N, ref1, &chunks, &np);
    GadgetHeader hd{};
    double rhoc = 0, a = 0;
    for (const IcChunk &ch : chunks) {
        hd = ch.h;
        if (c->p.verbose)
            std::printf("read file from %s\nnpart = %d\nmass = %g\na = %g\nredshift? = %g\nBoxSize = %g\nh = %g \n",
                        ch.path.c_str(), hd.npart[1], hd.mass[1], hd.time, hd.redshift, hd.BoxSize, hd.HubbleParam);
        // src/gadget_IC.h:309-314
        if (!(std::fabs(hd.BoxSize - 2 * c->xmax * 1e3 * h_0) < 0.001)) {
            char msg[256];
            std::snprintf(msg, sizeof msg, "ERROR: Boxsize of IC is different to xmax in Simulation !%g vs %g",
                          2 * c->xmax * 1e3 / h_0, hd.BoxSize);
            return fail(c, IFDM_ERR_BOXSIZE, msg);
        }
        hd.mass[1] *= 1e10;
        a = hd.time;
        rhoc = tot_chunks * hd.npart[1] * hd.mass[1] / pow(hd.BoxSize, 3) * pow(1e3, 3) * pow(h_0, 2);
    }
    if (!scan_err.empty()) return fail(c, IFDM_ERR_IO, scan_err);
    IcInput in;
    in.N = N;
    in.Lg = hd.BoxSize / N;
    in.box = hd.BoxSize;
    in.pmass = hd.mass[1];
    in.L3 = pow(in.Lg, 3);
    in.a = a;
    in.xmax = c->xmax;
    in.dx = c->dx;
    in.mfdm_solar = c->mfdm_solar;
    in.kf = c->mfdm / pow(phys::c, 2) / hbar;
    in.uc_rho = pow(h_0, 2) * pow(1e3, 3);
    in.uc_vel = 1e3 / m2Mpc * s2Myr;
    in.stream = c->stream;
    in.np = np;
    if (ensure_out(c)) return IFDM_ERR_CUDA;
    // particles straight from the files into device memory (ic_stream.hpp)
    float *d_part = nullptr;
    CTX_CUDA(c, cudaMalloc(&d_part, sizeof(float) * 6 * size_t(np > 0 ? np : 1)));
    std::string err = ic_upload(chunks, ref1, d_part, d_part + 3 * np, c->p.device);
    std::vector<float> vx;
    if (err.empty()) {
        in.d_pos = d_part;
        in.d_vel = d_part + 3 * np;
        err = ic_pipeline(in, c->d_out, &vx);
    }
    cudaFree(d_part);
    if (!err.empty()) return fail(c, err.find("Gadget") != std::string::npos ? IFDM_ERR_IO : IFDM_ERR_CUDA, err);
    CTX_STR(c, IFDM_ERR_IO, write_voutput(c->opath + "voutput.dat", vx.data(), vx.size()));
    return ifdm_set_psi(c, c->d_out, a, rhoc);
}

int ifdm_step(ifdm_ctx *c, int nsteps, double dt_scale) {
    if (!c || nsteps < 0) return IFDM_ERR_ARGS;
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.step(nsteps, dt_scale));
    return IFDM_OK;
}

// Simulation (src/CosmoBEC_MPI.cpp:183-310)
static int run_loop(ifdm_ctx *c);
int ifdm_run(ifdm_ctx *c) {
    if (!c) return IFDM_ERR_ARGS;
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    int rc = run_loop(c);
    // every snapshot file is complete when the run returns, as in the reference
    const std::string e = c->snap.drain();
    if (rc == IFDM_OK && !e.empty()) rc = fail(c, IFDM_ERR_IO, e);
    return rc;
}

static int run_loop(ifdm_ctx *c) {
    const bool v = c->p.verbose != 0;
    int write_num = 0;
    int write_sten_counter = 2;
    for (int tn = c->p.ti; tn < c->p.t_stop; ++tn) {
        const double a_prev = [&] {
            TState t{};
            c->eng.read_state(t);
            return t.steps ? t.a : c->a0;
        }();
        CTX_STR(c, IFDM_ERR_CUDA, c->eng.timestep_only(1.0));
        TState st{};
        CTX_STR(c, IFDM_ERR_CUDA, c->eng.read_state(st));
        if (st.err) return fail(c, IFDM_ERR_DEVICE, "device quadrature hit its interval limit");
        const double a = st.a;
        if (v) {
            std::printf(" max dt_KE = %g max dt_PE = %g max dt_QI = %g\n", st.cand_KE, st.cand_PE, st.cand_QI);
            std::printf("ai = %g a_next = %g da = %g n = %d ", a_prev, a, st.da, st.crit);
        }
        int rc = IFDM_OK;
        bool stop = false;
        if (a > 1) {
            rc = write_snapshot_which(c, 999999, 1, a);
            if (v) std::printf("write z = 0 at step%d\n", tn + 1);
            write_num++;
            stop = true;
        } else if (a > 0.714 && write_num == 4) {
            rc = write_snapshot_which(c, 999998, 1, a);
            if (v) std::printf("write z = 0.4 at step%d\n", tn + 1);
            write_num++;
        } else if (a > 0.5 && write_num == (c->p.stan ? 2 : 3)) {
            rc = write_snapshot_which(c, 999997, 1, a);
            if (v) std::printf("write z = 1 at step%d\n", tn + 1);
            write_num++;
            stop = true;
        } else if (!c->p.stan && a > 0.333 && write_num == 2) {
            rc = write_snapshot_which(c, 999996, 1, a);
            if (v) std::printf("write z = 2 at step%d\n", tn + 1);
            write_num++;
        } else if (a > 0.25 && write_num == 2) {
            rc = write_snapshot_which(c, write_sten_counter, 1, a);
            if (v) std::printf("write z < 3  at step%d\n", write_sten_counter);
            write_sten_counter++;
        } else if (a > 0.25 && write_num == 1) {
            rc = write_snapshot_which(c, 999995, 1, a);
            if (v) std::printf("write z = 3 at step%d\n", tn + 1);
            write_num++;
        } else if (a > 0.105 && write_num == 0) {
            rc = write_snapshot_which(c, 999994, 1, a);
            if (v) std::printf("write z = 8.5 at step%d\n", tn + 1);
            write_num++;
        } else if ((tn % c->p.t_write == 0) || tn == c->p.t_stop - 1) {
            rc = write_snapshot_which(c, tn + 1, 1, a);
        }
        if (rc) return rc;
        if (stop) break;
        if (v) std::printf("before write %d %g\n", write_num, 0.01 * write_num + 1);
        if (v) std::printf(" tn = %d\n", tn);
        CTX_STR(c, IFDM_ERR_CUDA, c->eng.passes_only());
        if (v) {
            CTX_CUDA(c, cudaStreamSynchronize(c->stream));
            std::printf("simulation takes:0 seconds\n");
            std::fflush(stdout);
        }
    }
    CTX_CUDA(c, cudaStreamSynchronize(c->stream));
    return IFDM_OK;
}

int ifdm_profile_passes(ifdm_ctx *c, int nsteps, double dt_scale, double *ms_out, const char **names_out, int cap) {
    if (!c || nsteps <= 0) return IFDM_ERR_ARGS;
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    std::vector<double> ms;
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.profile(nsteps, dt_scale, ms));
    for (int i = 0; i < kNumPasses && i < cap; ++i) {
        if (ms_out) ms_out[i] = ms[i];
        if (names_out) names_out[i] = kPassNames[i];
    }
    return kNumPasses;
}

int ifdm_pass_bytes(ifdm_ctx *c, double *bytes_out, int cap) {
    if (!c) return IFDM_ERR_ARGS;
    auto b = c->eng.pass_bytes();
    for (int i = 0; i < (int)b.size() && i < cap; ++i) bytes_out[i] = b[i];
    return (int)b.size();
}

int ifdm_record_steps(ifdm_ctx *c, int nsteps, double dt_scale, int checkpoint_every) {
    if (!c || nsteps <= 0 || checkpoint_every <= 0) return IFDM_ERR_ARGS;
    if (!c->have_psi) return fail(c, IFDM_ERR_STATE, "no wave function loaded");
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.record(nsteps, dt_scale, checkpoint_every));
    return IFDM_OK;
}

int ifdm_adjoint(ifdm_ctx *c, const double *g_final, double *g0) {
    if (!c || !g_final || !g0) return IFDM_ERR_ARGS;
    if (c->eng.recorded_steps() <= 0) return fail(c, IFDM_ERR_STATE, "ifdm_adjoint: no recorded steps");
    const size_t bytes = c->eng.n3() * 2 * sizeof(double);
    const bool din = is_device_ptr(g_final), dout = is_device_ptr(g0);
    // host arrays go through the context's complex128 staging buffer, in and
    // out alike: the sweep reads the cotangent at its start and writes the
    // gradient at its end, so one buffer serves both, and no allocation (which
    // would synchronise the device) happens per call
    if (!din || !dout) {
        if (ensure_out(c)) return IFDM_ERR_CUDA;
        if (c->snap.ready()) CTX_STR(c, IFDM_ERR_CUDA, c->snap.before_stage(c->stream));
    }
    if (!din) CTX_CUDA(c, cudaMemcpyAsync(c->d_out, g_final, bytes, cudaMemcpyHostToDevice, c->stream));
    std::string e = c->eng.adjoint(din ? g_final : c->d_out, dout ? g0 : c->d_out);
    if (e.empty() && !dout) {
        cudaError_t ce = cudaMemcpyAsync(g0, c->d_out, bytes, cudaMemcpyDeviceToHost, c->stream);
        if (ce != cudaSuccess) e = std::string("cudaMemcpyAsync: ") + cudaGetErrorString(ce);
    }
    cudaError_t ce = cudaStreamSynchronize(c->stream);
    if (e.empty() && ce != cudaSuccess) e = std::string("cudaStreamSynchronize: ") + cudaGetErrorString(ce);
    if (!e.empty()) return fail(c, IFDM_ERR_CUDA, e);
    TState t{};
    CTX_STR(c, IFDM_ERR_CUDA, c->eng.read_state(t));
    if (t.err) return fail(c, IFDM_ERR_DEVICE, "a device-side check failed during the adjoint");
    return IFDM_OK;
}

// ------------------------------------------------------------------ batches --
struct ifdm_batch {
    std::vector<ifdm_ctx *> ctx;
    cudaStream_t stream = nullptr;
    BatchEngine eng;
    std::string err;
};

static int bfail(ifdm_batch *b, int code, const std::string &msg) {
    if (b) b->err = msg;
    return code;
}

int ifdm_batch_create(ifdm_ctx *const *ctxs, int n, ifdm_batch **out) {
    if (!out) return IFDM_ERR_ARGS;
    *out = nullptr;
    if (!ctxs || n <= 0) return IFDM_ERR_ARGS;
    for (int i = 0; i < n; ++i)
        if (!ctxs[i]) return IFDM_ERR_ARGS;
    auto b = std::make_unique<ifdm_batch>();
    std::vector<StepEngine *> engines;
    for (int i = 0; i < n; ++i) {
        b->ctx.push_back(ctxs[i]);
        engines.push_back(&ctxs[i]->eng);
    }
    ifdm_batch *raw = b.release();
    *out = raw;
    for (int i = 0; i < n; ++i)
        if (ctxs[i]->p.device != ctxs[0]->p.device) return bfail(raw, IFDM_ERR_ARGS, "batch: contexts on different devices");
    if (cudaSetDevice(ctxs[0]->p.device) != cudaSuccess ||
        cudaStreamCreateWithFlags(&raw->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bfail(raw, IFDM_ERR_CUDA, "batch: stream creation failed");
    std::string e = raw->eng.init(engines, raw->stream);
    if (!e.empty()) {
        const bool shape = e.find("batch size") != std::string::npos || e.find("precision") != std::string::npos;
        return bfail(raw, shape ? IFDM_ERR_UNSUPPORTED : IFDM_ERR_CUDA, e);
    }
    return IFDM_OK;
}

int ifdm_batch_step(ifdm_batch *b, int nsteps, const double *dt_scale) {
    if (!b || nsteps < 0 || !dt_scale) return IFDM_ERR_ARGS;
    for (auto *c : b->ctx)
        if (!c->have_psi) return bfail(b, IFDM_ERR_STATE, "batch: a context has no wave function");
    if (cudaSetDevice(b->ctx[0]->p.device) != cudaSuccess) return bfail(b, IFDM_ERR_CUDA, "cudaSetDevice failed");
    std::string e = b->eng.step(nsteps, dt_scale);
    return e.empty() ? IFDM_OK : bfail(b, IFDM_ERR_CUDA, e);
}

static void knobs_to_tuning(const BatchKnobs &k, ifdm_batch_tuning *t) {
    t->mode = k.mode;
    t->blocks_per_sm = k.blocks_per_sm;
    t->group = k.group;
    for (int i = 0; i < kBatchSizes; ++i) t->plan[i] = k.plan[i];
}

int ifdm_batch_tune(ifdm_batch *b, int trial_steps, const double *dt_scale, ifdm_batch_tuning *out) {
    if (!b || trial_steps <= 0 || !dt_scale) return IFDM_ERR_ARGS;
    for (auto *c : b->ctx)
        if (!c->have_psi) return bfail(b, IFDM_ERR_STATE, "batch: a context has no wave function");
    double ms = 0;
    std::string e = b->eng.tune(trial_steps, dt_scale, &ms);
    if (!e.empty()) return bfail(b, e.find("gave up") != std::string::npos ? IFDM_ERR_DEVICE : IFDM_ERR_CUDA, e);
    if (out) {
        knobs_to_tuning(b->eng.knobs, out);
        out->ms_per_step = ms;
    }
    return IFDM_OK;
}

int ifdm_batch_get_tuning(ifdm_batch *b, ifdm_batch_tuning *out) {
    if (!b || !out) return IFDM_ERR_ARGS;
    knobs_to_tuning(b->eng.knobs, out);
    out->ms_per_step = 0;
    return IFDM_OK;
}

int ifdm_batch_set_tuning(ifdm_batch *b, const ifdm_batch_tuning *t) {
    if (!b || !t || t->blocks_per_sm < 1 || t->group < 0 || (t->mode != 0 && t->mode != 1)) return IFDM_ERR_ARGS;
    for (int i = 0; i < kBatchSizes; ++i)
        if (t->plan[i] != 0 && t->plan[i] != 1) return IFDM_ERR_ARGS;
    b->eng.knobs.mode = t->mode;
    b->eng.knobs.blocks_per_sm = t->blocks_per_sm;
    b->eng.knobs.group = t->group;
    for (int i = 0; i < kBatchSizes; ++i) b->eng.knobs.plan[i] = t->plan[i];
    return IFDM_OK;
}

int ifdm_batch_synchronize(ifdm_batch *b) {
    if (!b) return IFDM_ERR_ARGS;
    int st = 0;
    std::string e = b->eng.check_status(&st);
    if (!e.empty()) return bfail(b, IFDM_ERR_CUDA, e);
    if (st) return bfail(b, IFDM_ERR_DEVICE, "batch: a dependency wait of the batch kernel gave up");
    return IFDM_OK;
}

}  // extern "C"

// fn(i) for every context of the batch, on up to 16 host threads at a time;
// each context works on its own stream, so the boxes' kernels overlap on the
// device.  Returns the first failing context's code (its message copied).
template <class F> static int for_each_box(ifdm_batch *b, F fn) {
    const int n = (int)b->ctx.size();
    std::vector<int> rc(n, IFDM_OK);
    const int width = std::min(n, 16);
    std::vector<std::thread> pool;
    for (int w = 0; w < width; ++w)
        pool.emplace_back([&, w] {
            cudaSetDevice(b->ctx[0]->p.device);
            for (int i = w; i < n; i += width) rc[i] = fn(i);
        });
    for (auto &t : pool) t.join();
    for (int i = 0; i < n; ++i)
        if (rc[i] != IFDM_OK) return bfail(b, rc[i], "box " + std::to_string(i) + ": " + b->ctx[i]->err);
    return IFDM_OK;
}

extern "C" {

int ifdm_batch_record_steps(ifdm_batch *b, int nsteps, const double *dt_scale, int checkpoint_every) {
    if (!b || nsteps <= 0 || !dt_scale || checkpoint_every <= 0) return IFDM_ERR_ARGS;
    return for_each_box(b, [&](int i) {
        const int rc = ifdm_record_steps(b->ctx[i], nsteps, dt_scale[i], checkpoint_every);
        return rc ? rc : ifdm_synchronize(b->ctx[i]);
    });
}

int ifdm_batch_adjoint(ifdm_batch *b, const double *const *g_final, double *const *g0) {
    if (!b || !g_final || !g0) return IFDM_ERR_ARGS;
    return for_each_box(b, [&](int i) { return ifdm_adjoint(b->ctx[i], g_final[i], g0[i]); });
}

int ifdm_batch_info(ifdm_batch *b, long long *items_per_step, int *grid) {
    if (!b) return IFDM_ERR_ARGS;
    if (items_per_step) *items_per_step = b->eng.items_per_step();
    if (grid) *grid = b->eng.grid();
    return IFDM_OK;
}

const char *ifdm_batch_last_error(const ifdm_batch *b) { return b ? b->err.c_str() : "null batch"; }

void ifdm_batch_destroy(ifdm_batch *b) {
    if (!b) return;
    if (b->stream) {
        cudaStreamSynchronize(b->stream);
        cudaStreamDestroy(b->stream);
    }
    delete b;  // the engine's graphs and buffers do not refer to the stream
}

int ifdm_fft_slab(void *data, int n, int planes, int axis, int precision, int sign, int op, int y0, void *stream) {
    if (!data || (sign != 1 && sign != -1) || precision < 0 || precision > 2 || axis < 0 || axis > 2 || planes < 1 ||
        planes > n || op < 0 || op > 1 || (op == 1 && axis != 0) || y0 < 0 || y0 + planes > n)
        return IFDM_ERR_ARGS;
    if (!supported_n(n, precision)) return IFDM_ERR_UNSUPPORTED;
    const std::string e = fft_slab(data, n, planes, axis, precision, sign, op, y0, (cudaStream_t)stream);
    if (e.empty()) return IFDM_OK;
    return e.rfind("planes", 0) == 0 ? IFDM_ERR_ARGS : IFDM_ERR_CUDA;
}

int ifdm_fft3d(void *data, int n, int precision, int sign, void *stream) {
    if (!data || (sign != 1 && sign != -1) || precision < 0 || precision > 2) return IFDM_ERR_ARGS;
    if (!supported_n(n, precision)) return IFDM_ERR_UNSUPPORTED;
    std::string e = fft3d(data, n, precision, sign, (cudaStream_t)stream);
    return e.empty() ? IFDM_OK : IFDM_ERR_CUDA;
}

}  // extern "C"
