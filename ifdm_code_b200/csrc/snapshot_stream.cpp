// snapshot_stream.cpp -- see snapshot_stream.hpp.
#include "snapshot_stream.hpp"

#include "io.hpp"

namespace ifdm {

#define SS_TRY(expr)                                                                     \
    do {                                                                                 \
        cudaError_t e_ = (expr);                                                         \
        if (e_ != cudaSuccess) return std::string(#expr) + ": " + cudaGetErrorString(e_); \
    } while (0)

SnapshotStream::~SnapshotStream() {
    if (writer_.joinable()) {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        writer_.join();
    }
    if (copy_) cudaStreamSynchronize(copy_);
    for (int s = 0; s < 2; ++s) {
        if (host_[s]) cudaFreeHost(host_[s]);
        if (slot_copied_[s]) cudaEventDestroy(slot_copied_[s]);
    }
    if (staged_) cudaEventDestroy(staged_);
    if (copied_) cudaEventDestroy(copied_);
    if (copy_) cudaStreamDestroy(copy_);
}

std::string SnapshotStream::init(size_t bytes, int device) {
    if (copy_) return bytes == bytes_ ? "" : "snapshot stream already set up for another size";
    device_ = device;
    bytes_ = bytes;
    SS_TRY(cudaSetDevice(device));
    SS_TRY(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
    SS_TRY(cudaEventCreateWithFlags(&staged_, cudaEventDisableTiming));
    SS_TRY(cudaEventCreateWithFlags(&copied_, cudaEventDisableTiming));
    for (int s = 0; s < 2; ++s) {
        SS_TRY(cudaEventCreateWithFlags(&slot_copied_[s], cudaEventDisableTiming));
        SS_TRY(cudaMallocHost(&host_[s], bytes));
    }
    writer_ = std::thread([this] { writer_loop(); });
    return "";
}

std::string SnapshotStream::before_stage(cudaStream_t stream) {
    SS_TRY(cudaStreamWaitEvent(stream, copied_, 0));
    return "";
}

std::string SnapshotStream::submit(cudaStream_t stream, const double *staging, const std::string &path, double mfdm,
                                   double g_cm3, double a, const std::vector<double> &x) {
    int slot;
    {
        std::unique_lock<std::mutex> lk(mu_);
        if (!error_.empty()) return error_;
        cv_.wait(lk, [&] { return !slot_busy_[next_slot_] || !error_.empty(); });
        if (!error_.empty()) return error_;
        slot = next_slot_;
        slot_busy_[slot] = true;
        next_slot_ ^= 1;
    }
    SS_TRY(cudaEventRecord(staged_, stream));
    SS_TRY(cudaStreamWaitEvent(copy_, staged_, 0));
    SS_TRY(cudaMemcpyAsync(host_[slot], staging, bytes_, cudaMemcpyDeviceToHost, copy_));
    SS_TRY(cudaEventRecord(slot_copied_[slot], copy_));
    SS_TRY(cudaEventRecord(copied_, copy_));
    {
        std::lock_guard<std::mutex> lk(mu_);
        queue_.push_back(Job{slot, path, mfdm, g_cm3, a, x});
    }
    cv_.notify_all();
    return "";
}

void SnapshotStream::writer_loop() {
    cudaSetDevice(device_);
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !queue_.empty(); });
            if (queue_.empty()) return;  // stop_ with nothing left
            job = queue_.front();
        }
        std::string err;
        const cudaError_t ce = cudaEventSynchronize(slot_copied_[job.slot]);
        if (ce != cudaSuccess) err = std::string("snapshot copy: ") + cudaGetErrorString(ce);
        if (err.empty())
            err = write_snapshot(job.path, job.mfdm, job.g_cm3, job.a, job.x, host_[job.slot], bytes_ / 16);
        {
            std::lock_guard<std::mutex> lk(mu_);
            queue_.pop_front();
            slot_busy_[job.slot] = false;
            if (err.empty()) ++written_;
            else if (error_.empty()) error_ = err;
        }
        cv_.notify_all();
    }
}

std::string SnapshotStream::drain() {
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return queue_.empty(); });
    std::string e;
    e.swap(error_);  // reported once; later snapshots may succeed
    return e;
}

long long SnapshotStream::written() const {
    std::lock_guard<std::mutex> lk(mu_);
    return written_;
}

}  // namespace ifdm
