// Asynchronous snapshot files of a context (mhd_snapshot_write of the C ABI).
//
// The reference writes a snapshot synchronously from its host Grid every snapshot_frequency steps
// (integrator_main.cpp:102-109 -> write_data_to_binary_file, diagnostics.hpp:90-131). Here the
// snapshot is packed on the device in stream order (so later steps cannot disturb it), copied to
// pinned host memory on a copy stream of its own, and written to its file by a host thread, while
// the caller keeps stepping. Two slots (device staging + pinned host buffer each) let two
// snapshots be in flight; a third waits for a free slot.
#pragma once

#include <cuda_runtime.h>

#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>

#include "../../include/mhd_b200.h"

namespace mhd_host {

class SnapshotWriter {
public:
    explicit SnapshotWriter(int device) : device_(device) {}
    ~SnapshotWriter();
    SnapshotWriter(const SnapshotWriter&) = delete;
    SnapshotWriter& operator=(const SnapshotWriter&) = delete;

    // A free slot with room for `bytes` (waits while both are in flight); *d receives its device
    // staging buffer, into which the caller packs the snapshot on its stream.
    mhd_status acquire(size_t bytes, int* slot, double** d);
    // The pack into `slot` was enqueued on `stream`: copy it out on the copy stream after it, then
    // write the file `path` from the writer thread.
    mhd_status submit(int slot, cudaStream_t stream, const std::string& path, size_t bytes);
    // Give a slot back unused (the pack could not be enqueued).
    void release(int slot);
    // Wait until every submitted snapshot is written; MHD_ERR_IO (or a CUDA status) if one failed
    // since the last wait.
    mhd_status wait();

private:
    struct Slot {
        double* d = nullptr;
        void* h = nullptr;  // pinned
        size_t cap = 0;
        cudaEvent_t packed = nullptr, copied = nullptr;
        bool busy = false;
    };
    struct Job {
        int slot;
        std::string path;
        size_t bytes;
    };
    void run();
    mhd_status start();

    int device_;
    Slot slots_[2];
    cudaStream_t copy_ = nullptr;
    std::thread thread_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<Job> jobs_;
    bool stop_ = false;
    bool started_ = false;
    mhd_status error_ = MHD_OK;
};

}  // namespace mhd_host
