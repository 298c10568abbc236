// Host side of the asynchronous snapshot writer (see mhd_snapshot.h).
#include "mhd_snapshot.h"

#include <cstdio>

#include "mhd_host_util.h"

namespace mhd_host {

mhd_status SnapshotWriter::start() {
    if (started_) return MHD_OK;
    MHD_TRY(cudaStreamCreateWithFlags(&copy_, cudaStreamNonBlocking));
    for (Slot& s : slots_) {
        MHD_TRY(cudaEventCreateWithFlags(&s.packed, cudaEventDisableTiming));
        MHD_TRY(cudaEventCreateWithFlags(&s.copied, cudaEventDisableTiming));
    }
    thread_ = std::thread([this] { run(); });
    started_ = true;
    return MHD_OK;
}

SnapshotWriter::~SnapshotWriter() {
    if (started_) {
        wait();
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        thread_.join();
    }
    for (Slot& s : slots_) {
        cudaFree(s.d);
        if (s.h) cudaFreeHost(s.h);
        if (s.packed) cudaEventDestroy(s.packed);
        if (s.copied) cudaEventDestroy(s.copied);
    }
    if (copy_) cudaStreamDestroy(copy_);
    cudaGetLastError();
}

mhd_status SnapshotWriter::acquire(size_t bytes, int* slot, double** d) {
    mhd_status st = start();
    if (st != MHD_OK) return st;
    int k = -1;
    {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return !slots_[0].busy || !slots_[1].busy; });
        k = slots_[0].busy ? 1 : 0;
        slots_[k].busy = true;
    }
    Slot& s = slots_[k];
    if (s.cap < bytes) {  // no copy is in flight from a free slot
        cudaFree(s.d);
        if (s.h) cudaFreeHost(s.h);
        s.d = nullptr;
        s.h = nullptr;
        s.cap = 0;
        cudaError_t e = cudaMalloc(&s.d, bytes);
        if (e == cudaSuccess) e = cudaMallocHost(&s.h, bytes);
        if (e != cudaSuccess) {
            cudaGetLastError();
            release(k);
            return cuda_status(e);
        }
        s.cap = bytes;
    }
    *slot = k;
    *d = s.d;
    return MHD_OK;
}

void SnapshotWriter::release(int slot) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        slots_[slot].busy = false;
    }
    cv_.notify_all();
}

mhd_status SnapshotWriter::submit(int slot, cudaStream_t stream, const std::string& path,
                                  size_t bytes) {
    Slot& s = slots_[slot];
    cudaError_t e = cudaEventRecord(s.packed, stream);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(copy_, s.packed, 0);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s.h, s.d, bytes, cudaMemcpyDeviceToHost, copy_);
    if (e == cudaSuccess) e = cudaEventRecord(s.copied, copy_);
    if (e != cudaSuccess) {
        cudaGetLastError();
        release(slot);
        return cuda_status(e);
    }
    {
        std::lock_guard<std::mutex> lk(mu_);
        jobs_.push_back(Job{slot, path, bytes});
    }
    cv_.notify_all();
    return MHD_OK;
}

mhd_status SnapshotWriter::wait() {
    std::unique_lock<std::mutex> lk(mu_);
    cv_.wait(lk, [&] { return jobs_.empty() && !slots_[0].busy && !slots_[1].busy; });
    const mhd_status st = error_;
    error_ = MHD_OK;
    return st;
}

// Writer thread: each job waits for its copy, then writes the whole buffer to its file.
void SnapshotWriter::run() {
    cudaSetDevice(device_);
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> lk(mu_);
            cv_.wait(lk, [&] { return stop_ || !jobs_.empty(); });
            if (jobs_.empty()) return;  // stop_ with nothing left
            job = jobs_.front();
        }
        Slot& s = slots_[job.slot];
        mhd_status st = cuda_status(cudaEventSynchronize(s.copied));
        if (st == MHD_OK) {
            FILE* f = fopen(job.path.c_str(), "wb");
            if (!f) {
                st = MHD_ERR_IO;
            } else {
                if (fwrite(s.h, 1, job.bytes, f) != job.bytes) st = MHD_ERR_IO;
                if (fclose(f) != 0) st = MHD_ERR_IO;
            }
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (st != MHD_OK && error_ == MHD_OK) error_ = st;
            jobs_.pop_front();
            s.busy = false;
        }
        cv_.notify_all();
    }
}

}  // namespace mhd_host
