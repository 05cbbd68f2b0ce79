// batch_engine.hpp -- many independent boxes advanced by one graph launch.
#pragma once

#include "step_engine.hpp"

#include <map>
#include <string>
#include <vector>

namespace ifdm {

constexpr int kBatchSizes = 6;  // 16, 32, 48, 64, 96, 128
int batch_size_index(int n);     // -1 if n is not a batch size

// Launch shape of the batch: the choices the autotuner makes.
struct BatchKnobs {
    int mode = 0;                 // 0: one persistent kernel per box size; 1: one launch per phase and size
    int blocks_per_sm = 2;        // persistent CTAs per SM (clamped to what fits)
    int group = 0;                // boxes per group in the persistent item order (0: all boxes in lock step)
    int plan[kBatchSizes] = {0};  // radix-plan variant per grid size
};

struct BatchKernels;

class BatchEngine {
  public:
    BatchEngine() = default;
    ~BatchEngine();
    BatchEngine(const BatchEngine &) = delete;
    BatchEngine &operator=(const BatchEngine &) = delete;

    // Boxes share the device and the precision; each keeps its own stream,
    // which the batch orders itself against.
    std::string init(const std::vector<StepEngine *> &boxes, cudaStream_t stream);
    // nsteps fixed-mode steps of every box (dt_scale[b] per box), replayed
    // from a captured CUDA graph: boxes of one size share one persistent
    // launch (mode 0) or one launch per phase (mode 1); sizes run side by
    // side.  Asynchronous.
    std::string step(int nsteps, const double *dt_scale);
    // Time candidate knobs on trial_steps steps each (the boxes' states are
    // saved before and restored after), keep the fastest; synchronous.
    std::string tune(int trial_steps, const double *dt_scale, double *best_ms_per_step);
    // nonzero *status if a dependency wait of the last launch gave up (synchronous)
    std::string check_status(int *status);

    BatchKnobs knobs;
    int grid() const;                   // persistent CTAs of all sizes (mode 0)
    long long items_per_step() const;   // work items of one batch step

  private:
    struct Class {                      // the boxes of one grid size
        int N = 0;
        std::vector<int> boxes;         // indices into boxes_
        int items[10] = {0};            // items per phase of one box
        size_t smem = 0;
        int fit = 0, grid = 0, nsegs = 0;
        long long step_items = 0;
        void *d_boxes = nullptr, *d_segs = nullptr;
        unsigned long long *d_ctr = nullptr;  // [0] claim counter, [1..] per-box done counters
        cudaStream_t side = nullptr;
        cudaEvent_t fork = nullptr, join = nullptr;
    };
    std::string prepare(const double *dt_scale);  // box tables + item orders for the current knobs
    std::string graph_for(int nsteps, cudaGraphExec_t *out);
    std::string capture_body(int nsteps);
    std::string order_streams_before();
    std::string order_streams_after();

    const BatchKernels *K_ = nullptr;
    std::vector<StepEngine *> boxes_;
    std::vector<Class> cls_;
    cudaStream_t stream_ = nullptr;
    int precision_ = 0, dev_ = 0, sms_ = 0;
    int *d_status_ = nullptr;
    std::map<int, cudaGraphExec_t> graphs_;  // per step count
    std::vector<cudaEvent_t> ev_;
    cudaEvent_t ev_done_ = nullptr;
    BatchKnobs prepared_{};
    bool have_prepared_ = false;
    std::vector<unsigned char> prepared_boxes_raw_;
};

}  // namespace ifdm
