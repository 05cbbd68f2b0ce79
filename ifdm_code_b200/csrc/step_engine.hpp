// step_engine.hpp -- device state and pass launcher of one simulation box.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "state_types.hpp"

#include <string>
#include <vector>

namespace ifdm {

struct EngineConfig {
    int N = 0;
    int precision = 0;  // 0 FP64, 1 FP32
    // physics (natural units of the reference)
    double mfdm = 0, g = 0, xmax = 0, dx = 0;
    double mfdm_solar = 0, rhoc = 0;
    double dt_scale = 1.0;
};

// Device buffers and constants of one box (for the batch launcher).
struct EngineView {
    int N, precision;
    void *psi, *phi, *rhok;
    const void *tw, *twh;
    TState *ts;
    double2 *drift64;
    float2 *drift32;
    Phys phys;  // dt_scale 1
    long win_rows;
    int win_tail;
};

// Names of the fused passes in launch order (timestep first).
constexpr int kNumPasses = 10;
extern const char *const kPassNames[kNumPasses];

class StepEngine {
  public:
    StepEngine() = default;
    ~StepEngine();
    StepEngine(const StepEngine &) = delete;
    StepEngine &operator=(const StepEngine &) = delete;

    // Allocates device buffers on the current device; returns "" or an error.
    std::string init(const EngineConfig &cfg, cudaStream_t stream);
    // psi (host or device complex128, N^3) -> scaled state; sets a and rho_c,
    // runs the initial density/Poisson passes.  Asynchronous.
    std::string load_psi(const double *psi_c128, bool on_device, double a, double rhoc);
    // nsteps fixed-mode steps (timestep + 9 passes each).  Asynchronous.
    std::string step(int nsteps, double dt_scale);
    // Per-pass event timing of nsteps steps (synchronous); ms per step.
    std::string profile(int nsteps, double dt_scale, std::vector<double> &ms);
    // Algorithmic HBM bytes per pass per step.
    std::vector<double> pass_bytes() const;
    // psi as complex128 into dev_out (device), which: 0 raw, 1 snapshot kick, 2 pending kick.
    std::string psi_out(double *dev_out, int which);
    // psi as complex128 into a host buffer (pinned for full speed): chunks
    // converted on the compute stream and copied on the copy stream through
    // the two staging slots, each copy overlapping the next conversion.
    // Returns once the host buffer holds the whole field.
    std::string psi_to_host(double *host_out, int which);
    std::string phi_out(double *dev_out);
    // copy the TState to host (synchronous)
    std::string read_state(TState &out);
    // Adjoint support.  record(): nsteps fixed-mode steps that keep a per-step
    // log of the coefficients and a checkpoint of (psi, phi) every ckpt steps.
    std::string record(int nsteps, double dt_scale, int ckpt);
    // gradient of a real loss through the recorded steps: g_final = dL/dpsi_final
    // (complex128, natural units, dL/dRe + i dL/dIm) -> g0 = dL/dpsi_0; both
    // device pointers.  Leaves the context's state at an intermediate step.
    std::string adjoint(const double *g_final_dev, double *g0_dev);
    int recorded_steps() const { return recorded_; }
    // one step split for the native loop: timestep only / passes only
    std::string timestep_only(double dt_scale);
    std::string passes_only();

    int N() const { return cfg_.N; }
    int precision() const { return cfg_.precision; }
    cudaStream_t stream() const { return stream_; }
    double S() const { return S_; }
    double Phi0() const { return Phi0_; }
    size_t n3() const { return size_t(cfg_.N) * cfg_.N * cfg_.N; }
    void *psi_ptr() const { return psi_; }
    EngineView view() const {
        return {cfg_.N, cfg_.precision, psi_, phi_, rhok_, tw_, twh_, ts_, drift64_, drift32_, phys_, win_rows_, win_tail_};
    }

  private:
    std::string launch_timestep(double dt_scale);
    std::string launch_passes(cudaEvent_t *ev);  // ev: optional 10 events (after each pass)
    std::string launch_initial_density();
    std::string set_physics(double a, double rhoc);
    std::string ensure_staging();
    size_t n3_() const;

    // host transfers: two device slots of kStageElems complex128 each, a copy
    // stream, and per slot an event "copy done" and "slot free" (allocated on
    // the first host transfer, kept for the context's lifetime)
    static constexpr size_t kStageElems = size_t(1) << 22;
    double2 *stage_[2] = {nullptr, nullptr};
    cudaStream_t copy_stream_ = nullptr;
    cudaEvent_t ev_copied_[2] = {nullptr, nullptr}, ev_free_[2] = {nullptr, nullptr};

    EngineConfig cfg_{};
    cudaStream_t stream_ = nullptr;
    void *psi_ = nullptr, *phi_ = nullptr, *rhok_ = nullptr;
    void *tw_ = nullptr, *twh_ = nullptr;  // precision-typed twiddle tables (N and N/2)
    double2 *drift64_ = nullptr;
    float2 *drift32_ = nullptr;
    TState *ts_ = nullptr;
    double *part_ = nullptr;  // per-block partial sums of the initial pass
    Phys phys_{};
    double S_ = 1, Phi0_ = 1;
    long win_rows_ = 0;
    // TMA descriptors of the y/x passes (psi and the half spectrum), used for N >= 128
    bool use_tma_ = false;
    CUtensorMap map_psi_y_{}, map_psi_x_{}, map_rho_y_{}, map_rho_x_{};
    int tma_ly_ = 8, tma_lx_ = 8;  // lines per TMA tile of the y and x passes (inner box extent)
    // adjoint buffers
    void *log_ = nullptr;  // StepLog[log_cap_]
    int log_cap_ = 0, recorded_ = 0, ckpt_every_ = 0, nckpt_cap_ = 0, seg_cap_ = 0;
    void *ckpt_psi_ = nullptr, *ckpt_phi_ = nullptr, *seg_psi_ = nullptr, *seg_phi_ = nullptr;
    void *g_ = nullptr, *w_ = nullptr, *pw_ = nullptr;
    TState *ts_adj_ = nullptr;
    unsigned long long *gmax_ = nullptr;  // max |component| of the incoming gradient (ordered bits)
    double2 *drift64_adj_ = nullptr;
    float2 *drift32_adj_ = nullptr;
    CUtensorMap map_g_y_{}, map_g_x_{};
    std::string ensure_adjoint_buffers(int nsteps, int ckpt);
    std::string adjoint_kick(void *psi, void *phi, double a, double aP, double b, double alpha, long long tag);
    int win_tail_ = 0;
};

// Plain in-place 3-D c2c FFT of device data (complex128 if precision 0).
std::string fft3d(void *data, int n, int precision, int sign, cudaStream_t stream);
// One axis of a slab-decomposed 3-D FFT on device data (ifdm_fft_slab).
std::string fft_slab(void *data, int n, int planes, int axis, int precision, int sign, int op, int y0,
                     cudaStream_t stream);
bool supported_n(int n);
// grid sizes with a compiled plan in a precision mode (0 FP64, 1 FP32, 2 mixed)
bool supported_n(int n, int precision);

}  // namespace ifdm
