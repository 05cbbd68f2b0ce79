// snapshot_stream.hpp -- snapshots written while the steps go on.
//
// The reference's writeall (src/write3D.h:86-97) stops the simulation while a
// snapshot is gathered and written.  Here a snapshot costs the compute stream
// only the kernel that puts psi (complex128) into a device staging buffer:
//
//   compute stream   psi_out -> staging      (event `staged`)
//   copy stream      waits `staged`; staging -> pinned host slot  (event `copied`)
//   writer thread    waits `copied`; writes <opath>output<t>.dat from the slot
//
// The compute stream waits for `copied` before it overwrites the staging
// buffer with the next snapshot (a device-side wait; the host does not
// block).  Two pinned slots let one file be written while the next copy
// runs; submit() blocks only when both slots hold files not yet written.
// Each file is one sequential write: buffered writes to one file are
// serialised by the file system anyway, and 8 threads writing disjoint
// ranges of a 2 GiB file measured no faster.
// The files are the same bytes the synchronous path writes.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

namespace ifdm {

class SnapshotStream {
  public:
    SnapshotStream() = default;
    SnapshotStream(const SnapshotStream &) = delete;
    SnapshotStream &operator=(const SnapshotStream &) = delete;
    ~SnapshotStream();

    // bytes: one snapshot's psi (16 N^3); device: the CUDA device of the streams
    std::string init(size_t bytes, int device);
    bool ready() const { return copy_ != nullptr; }

    // Before producing the next snapshot into the staging buffer: make
    // `stream` wait until the previous copy out of it has finished.
    std::string before_stage(cudaStream_t stream);
    // The staging buffer `staging` (filled by work already queued on
    // `stream`) goes to `path` with the snapshot header (mfdm, g, a, x).
    std::string submit(cudaStream_t stream, const double *staging, const std::string &path, double mfdm, double g_cm3,
                       double a, const std::vector<double> &x);
    // Wait until every submitted file is written; returns (and clears) the
    // first error since the last drain.  submit() fails while one is pending.
    std::string drain();
    // Number of files written since init.
    long long written() const;

  private:
    struct Job {
        int slot;
        std::string path;
        double mfdm, g_cm3, a;
        std::vector<double> x;
    };
    void writer_loop();

    int device_ = 0;
    size_t bytes_ = 0;
    cudaStream_t copy_ = nullptr;
    cudaEvent_t staged_ = nullptr, copied_ = nullptr;  // copied_: last copy out of the staging buffer
    cudaEvent_t slot_copied_[2] = {nullptr, nullptr};
    double *host_[2] = {nullptr, nullptr};
    bool slot_busy_[2] = {false, false};
    int next_slot_ = 0;

    mutable std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Job> queue_;
    std::string error_;
    long long written_ = 0;
    bool stop_ = false;
    std::thread writer_;
};

}  // namespace ifdm
