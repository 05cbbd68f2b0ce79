// batch_engine.cu -- item order, launch shape, CUDA graph and autotuner of the
// batch kernels (batch_kernels.cuh, instantiated per precision through
// batch_launch.cuh).
#include "batch_engine.hpp"
#include "batch_launch.cuh"

#include <algorithm>
#include <cstring>

namespace ifdm {

#define CUDA_TRY(expr)                                                                   \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) return std::string(#expr) + ": " + cudaGetErrorString(e_); \
    } while (0)

const BatchKernels &batch_kernels_fp64();
const BatchKernels &batch_kernels_fp32();
const BatchKernels &batch_kernels_mixed();

const BatchKernels &batch_kernels(int precision) {
    return precision == 0 ? batch_kernels_fp64() : precision == 1 ? batch_kernels_fp32() : batch_kernels_mixed();
}

int batch_size_index(int n) {
    switch (n) {
        case 16: return 0;
        case 32: return 1;
        case 48: return 2;
        case 64: return 3;
        case 96: return 4;
        case 128: return 5;
        default: return -1;
    }
}

BatchEngine::~BatchEngine() {
    for (auto &g : graphs_) cudaGraphExecDestroy(g.second);
    for (auto e : ev_) cudaEventDestroy(e);
    if (ev_done_) cudaEventDestroy(ev_done_);
    for (auto &c : cls_) {
        cudaFree(c.d_boxes);
        cudaFree(c.d_segs);
        cudaFree(c.d_ctr);
        if (c.side) cudaStreamDestroy(c.side);
        if (c.fork) cudaEventDestroy(c.fork);
        if (c.join) cudaEventDestroy(c.join);
    }
    cudaFree(d_status_);
}

int BatchEngine::grid() const {
    int g = 0;
    for (auto &c : cls_) g += c.grid;
    return g;
}

long long BatchEngine::items_per_step() const {
    long long n = 0;
    for (auto &c : cls_) n += c.step_items;
    return n;
}

std::string BatchEngine::init(const std::vector<StepEngine *> &boxes, cudaStream_t stream) {
    if (boxes.empty()) return "batch: no boxes";
    boxes_ = boxes;
    stream_ = stream;
    precision_ = boxes[0]->precision();
    K_ = &batch_kernels(precision_);
    for (size_t b = 0; b < boxes_.size(); ++b) {
        const int N = boxes_[b]->N();
        if (boxes_[b]->precision() != precision_) return "batch: all boxes must use the same precision";
        if (batch_size_index(N) < 0)
            return "batch: res " + std::to_string(N) + " is not a batch size (16, 32, 48, 64, 96, 128)";
        auto it = std::find_if(cls_.begin(), cls_.end(), [&](const Class &c) { return c.N == N; });
        if (it == cls_.end()) {
            cls_.emplace_back();
            cls_.back().N = N;
            it = cls_.end() - 1;
        }
        it->boxes.push_back((int)b);
    }
    std::sort(cls_.begin(), cls_.end(), [](const Class &a, const Class &b) { return a.N < b.N; });
    CUDA_TRY(cudaGetDevice(&dev_));
    CUDA_TRY(cudaDeviceGetAttribute(&sms_, cudaDevAttrMultiProcessorCount, dev_));
    for (auto &c : cls_) {
        if (!K_->items(c.N, c.items, &c.smem)) return "batch: res " + std::to_string(c.N) + " is not a batch size";
        const size_t nb = c.boxes.size();
        CUDA_TRY(cudaMalloc(&c.d_boxes, sizeof(BatchBox) * nb));
        CUDA_TRY(cudaMalloc(&c.d_segs, sizeof(BatchSeg) * nb * kBatchPhases));
        CUDA_TRY(cudaMalloc(&c.d_ctr, sizeof(unsigned long long) * (nb + 1)));
        CUDA_TRY(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
        CUDA_TRY(cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming));
        CUDA_TRY(cudaEventCreateWithFlags(&c.join, cudaEventDisableTiming));
        for (int v = 0; v < 2; ++v) {
            int fit = 0;
            std::string e = K_->setup(c.N, v, c.smem, &fit);
            if (!e.empty()) return e;
        }
    }
    CUDA_TRY(cudaMalloc(&d_status_, sizeof(int)));
    CUDA_TRY(cudaMemset(d_status_, 0, sizeof(int)));
    ev_.resize(boxes_.size(), nullptr);
    for (auto &e : ev_) CUDA_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&ev_done_, cudaEventDisableTiming));
    return "";
}

std::string BatchEngine::prepare(const double *dt_scale) {
    // box tables (the engines' views are read again: a state load may set new constants)
    std::vector<std::vector<BatchBox>> hb(cls_.size());
    std::vector<unsigned char> raw;
    for (size_t ci = 0; ci < cls_.size(); ++ci) {
        Class &c = cls_[ci];
        for (int b : c.boxes) {
            const EngineView v = boxes_[b]->view();
            BatchBox x;
            std::memset(&x, 0, sizeof x);
            x.N = v.N;
            x.win_rows = v.win_rows;
            x.win_tail = v.win_tail;
            x.psi = v.psi;
            x.phi = v.phi;
            x.rhok = v.rhok;
            x.tw = v.tw;
            x.twh = v.twh;
            x.ts = v.ts;
            x.drift64 = v.drift64;
            x.drift32 = v.drift32;
            x.ph = v.phys;
            x.ph.dt_scale = dt_scale[b];
            int acc = 0;
            for (int p = 0; p < kBatchPhases; ++p) {
                x.prefix[p] = acc;
                acc += c.items[p];
            }
            x.prefix[kBatchPhases] = acc;
            x.step_items = acc;
            hb[ci].push_back(x);
            raw.insert(raw.end(), (const unsigned char *)&x, (const unsigned char *)&x + sizeof x);
        }
    }
    if (have_prepared_ && std::memcmp(&prepared_, &knobs, sizeof(BatchKnobs)) == 0 && raw == prepared_boxes_raw_)
        return "";
    // persistent CTAs: the requested number per SM, shared between the sizes by their work
    double work_all = 0;
    for (auto &c : cls_) work_all += double(c.boxes.size()) * c.N * c.N * c.N;
    for (size_t ci = 0; ci < cls_.size(); ++ci) {
        Class &c = cls_[ci];
        const int nb = (int)c.boxes.size();
        const int V = knobs.plan[batch_size_index(c.N)] ? 1 : 0;
        std::string e = K_->setup(c.N, V, c.smem, &c.fit);
        if (!e.empty()) return e;
        if (c.fit < 1) return "batch: the batch kernel does not fit on an SM";
        const double share = double(nb) * c.N * c.N * c.N / work_all;
        const double ctas = double(sms_) * std::max(1, std::min(knobs.blocks_per_sm, c.fit));
        c.grid = std::max(1, (int)(ctas * share + 0.5));
        // item order of one step: groups of boxes, phase by phase within a group
        const int G = (knobs.group <= 0 || knobs.group >= nb) ? nb : knobs.group;
        std::vector<BatchSeg> segs;
        int first = 0;
        for (int g0 = 0; g0 < nb; g0 += G)
            for (int p = 0; p < kBatchPhases; ++p)
                for (int b = g0; b < std::min(nb, g0 + G); ++b) {
                    segs.push_back({b, p, first, c.items[p]});
                    first += c.items[p];
                }
        c.nsegs = (int)segs.size();
        c.step_items = first;
        CUDA_TRY(cudaMemcpy(c.d_boxes, hb[ci].data(), sizeof(BatchBox) * nb, cudaMemcpyHostToDevice));
        CUDA_TRY(cudaMemcpy(c.d_segs, segs.data(), sizeof(BatchSeg) * segs.size(), cudaMemcpyHostToDevice));
    }
    for (auto &g : graphs_) cudaGraphExecDestroy(g.second);
    graphs_.clear();
    prepared_ = knobs;
    prepared_boxes_raw_ = raw;
    have_prepared_ = true;
    return "";
}

// The launches of nsteps batch steps on stream_ (being captured): every size
// on its own forked stream, joined back at the end.
std::string BatchEngine::capture_body(int nsteps) {
    CUDA_TRY(cudaMemsetAsync(d_status_, 0, sizeof(int), stream_));
    for (auto &c : cls_) {
        const int nb = (int)c.boxes.size();
        const int V = knobs.plan[batch_size_index(c.N)] ? 1 : 0;
        CUDA_TRY(cudaEventRecord(c.fork, stream_));
        CUDA_TRY(cudaStreamWaitEvent(c.side, c.fork, 0));
        if (knobs.mode == 0) {
            CUDA_TRY(cudaMemsetAsync(c.d_ctr, 0, sizeof(unsigned long long) * (nb + 1), c.side));
            BatchArgs a{};
            a.boxes = (const BatchBox *)c.d_boxes;
            a.segs = (const BatchSeg *)c.d_segs;
            a.nsegs = c.nsegs;
            a.step_items = c.step_items;
            a.total = c.step_items * (long long)nsteps;
            a.next = c.d_ctr;
            a.done = c.d_ctr + 1;
            a.status = d_status_;
            CUDA_TRY(K_->persistent(c.N, V, c.grid, c.smem, c.side, a));
        } else {
            for (int s = 0; s < nsteps; ++s)
                for (int p = 0; p < kBatchPhases; ++p)
                    CUDA_TRY(K_->phase(c.N, V, p, c.items[p], nb, c.smem, c.side, (const BatchBox *)c.d_boxes));
        }
        CUDA_TRY(cudaEventRecord(c.join, c.side));
        CUDA_TRY(cudaStreamWaitEvent(stream_, c.join, 0));
    }
    return "";
}

std::string BatchEngine::graph_for(int nsteps, cudaGraphExec_t *out) {
    auto it = graphs_.find(nsteps);
    if (it != graphs_.end()) {
        *out = it->second;
        return "";
    }
    cudaGraph_t g = nullptr;
    CUDA_TRY(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
    std::string e = capture_body(nsteps);
    cudaError_t ee = cudaStreamEndCapture(stream_, &g);
    if (!e.empty() || ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return "batch graph capture: " + (e.empty() ? std::string(cudaGetErrorString(ee)) : e);
    }
    cudaGraphExec_t ex = nullptr;
    ee = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ee != cudaSuccess) return std::string("batch graph instantiate: ") + cudaGetErrorString(ee);
    graphs_[nsteps] = ex;
    *out = ex;
    return "";
}

std::string BatchEngine::order_streams_before() {
    for (size_t b = 0; b < boxes_.size(); ++b) {
        if (boxes_[b]->stream() == stream_) continue;
        CUDA_TRY(cudaEventRecord(ev_[b], boxes_[b]->stream()));
        CUDA_TRY(cudaStreamWaitEvent(stream_, ev_[b], 0));
    }
    return "";
}

std::string BatchEngine::order_streams_after() {
    CUDA_TRY(cudaEventRecord(ev_done_, stream_));
    for (auto *b : boxes_)
        if (b->stream() != stream_) CUDA_TRY(cudaStreamWaitEvent(b->stream(), ev_done_, 0));
    return "";
}

std::string BatchEngine::step(int nsteps, const double *dt_scale) {
    if (nsteps <= 0) return "";
    std::string e = prepare(dt_scale);
    if (!e.empty()) return e;
    cudaGraphExec_t ex = nullptr;
    e = graph_for(nsteps, &ex);
    if (!e.empty()) return e;
    e = order_streams_before();
    if (!e.empty()) return e;
    CUDA_TRY(cudaGraphLaunch(ex, stream_));
    return order_streams_after();
}

std::string BatchEngine::check_status(int *status) {
    CUDA_TRY(cudaStreamSynchronize(stream_));
    CUDA_TRY(cudaMemcpy(status, d_status_, sizeof(int), cudaMemcpyDeviceToHost));
    return "";
}

std::string BatchEngine::tune(int trial_steps, const double *dt_scale, double *best_ms_per_step) {
    if (trial_steps <= 0) return "tune: trial_steps must be positive";
    const int n = (int)boxes_.size();
    // save every box's state (psi, phi, TState); the passes rebuild the rest each step
    const size_t rs = precision_ == 0 ? 8 : 4;
    std::vector<size_t> off(n + 1, 0);
    for (int b = 0; b < n; ++b) {
        const size_t n3 = boxes_[b]->n3();
        off[b + 1] = off[b] + n3 * 3 * rs + ((sizeof(TState) + 255) / 256) * 256;
    }
    for (auto *b : boxes_) CUDA_TRY(cudaStreamSynchronize(b->stream()));
    char *save = nullptr;
    CUDA_TRY(cudaMalloc(&save, off[n]));
    auto copy_state = [&](bool to_save) -> std::string {
        for (int b = 0; b < n; ++b) {
            const EngineView v = boxes_[b]->view();
            const size_t n3 = boxes_[b]->n3();
            char *s = save + off[b];
            char *pairs[3][2] = {{s, (char *)v.psi}, {s + 2 * n3 * rs, (char *)v.phi}, {s + 3 * n3 * rs, (char *)v.ts}};
            const size_t sz[3] = {2 * n3 * rs, n3 * rs, sizeof(TState)};
            for (int k = 0; k < 3; ++k) {
                char *dst = to_save ? pairs[k][0] : pairs[k][1];
                char *src = to_save ? pairs[k][1] : pairs[k][0];
                CUDA_TRY(cudaMemcpyAsync(dst, src, sz[k], cudaMemcpyDeviceToDevice, stream_));
            }
        }
        return "";
    };
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    std::string err;
    auto trial = [&](double *ms) -> std::string {
        std::string e = prepare(dt_scale);
        if (!e.empty()) return e;
        cudaGraphExec_t ex = nullptr;
        e = graph_for(trial_steps, &ex);
        if (!e.empty()) return e;
        float best = 1e30f;
        for (int rep = 0; rep < 2; ++rep) {
            e = copy_state(false);
            if (!e.empty()) return e;
            CUDA_TRY(cudaEventRecord(t0, stream_));
            CUDA_TRY(cudaGraphLaunch(ex, stream_));
            CUDA_TRY(cudaEventRecord(t1, stream_));
            CUDA_TRY(cudaEventSynchronize(t1));
            float t = 0.f;
            CUDA_TRY(cudaEventElapsedTime(&t, t0, t1));
            best = std::min(best, t);
        }
        int st = 0;
        CUDA_TRY(cudaMemcpy(&st, d_status_, sizeof(int), cudaMemcpyDeviceToHost));
        if (st) return "tune: a dependency wait of the batch kernel gave up";
        *ms = best;
        return "";
    };
    do {
        if (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess) {
            err = "tune: event creation failed";
            break;
        }
        err = copy_state(true);
        if (!err.empty()) break;
        BatchKnobs best = knobs;
        double best_ms = 0;
        err = trial(&best_ms);
        if (!err.empty()) break;
        auto consider = [&](const BatchKnobs &k) -> std::string {
            knobs = k;
            double ms = 0;
            std::string e = trial(&ms);
            if (!e.empty()) return e;
            if (ms < best_ms) {
                best_ms = ms;
                best = k;
            }
            return "";
        };
        // 1) schedule: persistent kernels, or one launch per phase
        {
            BatchKnobs k = best;
            k.mode = 1 - k.mode;
            err = consider(k);
        }
        // 2) persistent shape: CTAs per SM, then the group size of the item order
        for (int bps = 1; bps <= 4 && err.empty(); ++bps) {
            BatchKnobs k = best;
            k.mode = 0;
            k.blocks_per_sm = bps;
            err = consider(k);
        }
        const int cand[3] = {(n + 1) / 2, (n + 3) / 4, 8};
        for (int ci = 0; ci < 3 && err.empty(); ++ci) {
            if (best.mode != 0 || cand[ci] >= n) continue;
            BatchKnobs k = best;
            k.group = cand[ci];
            err = consider(k);
        }
        // 3) radix plan of each grid size present that has an alternative
        for (auto &c : cls_) {
            if (!err.empty()) break;
            if (c.N == 16 || c.N == 128) continue;
            BatchKnobs k = best;
            const int si = batch_size_index(c.N);
            k.plan[si] = 1 - k.plan[si];
            err = consider(k);
        }
        if (!err.empty()) break;
        knobs = best;
        *best_ms_per_step = best_ms / trial_steps;
        err = copy_state(false);
        if (!err.empty()) break;
        err = prepare(dt_scale);
    } while (false);
    cudaStreamSynchronize(stream_);
    cudaFree(save);
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    return err;
}

}  // namespace ifdm
