// Copies of device results into the caller's pageable host arrays. A device-to-host copy into pageable memory runs at
// the driver's single-threaded staging rate (117 MB of path columns: 6.7 ms on a B200 host); into pinned memory it
// runs at the link's rate (2.2 ms), and host threads then spread the bytes into the caller's array in parallel.
// Pinning the caller's array itself costs more than the copy (117 MB: 12.5 ms), so the library keeps its own pinned
// staging, two slots reused from call to call.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <functional>
#include <mutex>
#include <thread>

#include "common.cuh"

namespace ob {

// Two pinned slots of kSlotBytes, allocated at their first use and kept until release() (ob_release_buffers).
// Portable pinned memory: any device's copies may use it. Null where pinned memory cannot be had (the caller then
// copies into its pageable array directly).
class PinnedStage {
  public:
    static constexpr size_t kSlotBytes = size_t(32) << 20;
    static PinnedStage& get() {
        static PinnedStage* s = new PinnedStage();
        return *s;
    }
    double* slot(int k) {
        std::lock_guard<std::mutex> lock(m_);
        if (!base_ && !failed_) {
            if (cudaHostAlloc(&base_, 2 * kSlotBytes, cudaHostAllocPortable) != cudaSuccess) {
                cudaGetLastError();
                base_ = nullptr, failed_ = true;
            }
        }
        return base_ ? reinterpret_cast<double*>(static_cast<char*>(base_) + static_cast<size_t>(k) * kSlotBytes)
                     : nullptr;
    }
    void release() {
        std::lock_guard<std::mutex> lock(m_);
        if (base_) cudaFreeHost(base_);
        cudaGetLastError();
        base_ = nullptr, failed_ = false;
    }

  private:
    std::mutex m_;
    void* base_ = nullptr;
    bool failed_ = false;
};

// Host threads for the copies out of the staging: the hardware threads less one, at most seven, started at the first
// use and kept for the process (never joined: they wait on a condition variable between jobs).
class HostPool {
  public:
    static HostPool& get() {
        static HostPool* p = new HostPool();
        return *p;
    }
    // fn(i) for every i in [0, n), on the pool's threads and the calling one; returns when every call has returned.
    void run(int n, const std::function<void(int)>& fn) {
        if (n <= 0) return;
        std::lock_guard<std::mutex> one(run_m_);
        unsigned long long g;
        {
            std::lock_guard<std::mutex> lock(m_);
            fn_ = &fn, n_ = n, next_ = 0, done_ = 0;
            g = ++gen_;
        }
        cv_.notify_all();
        work(g);
        std::unique_lock<std::mutex> lock(m_);
        done_cv_.wait(lock, [&] { return done_ == n_; });
        fn_ = nullptr;
    }

  private:
    HostPool() {
        const int hw = static_cast<int>(std::thread::hardware_concurrency());
        const int n = std::max(0, std::min(7, hw - 1));
        for (int k = 0; k < n; ++k) std::thread([this] { loop(); }).detach();
    }
    void loop() {
        unsigned long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lock(m_);
                cv_.wait(lock, [&] { return gen_ != seen; });
                seen = gen_;
            }
            work(seen);
        }
    }
    // Items of job g, one at a time under the lock, until none is left (or another job has begun).
    void work(unsigned long long g) {
        for (;;) {
            int i;
            const std::function<void(int)>* fn;
            {
                std::lock_guard<std::mutex> lock(m_);
                if (gen_ != g || next_ >= n_) return;
                i = next_++, fn = fn_;
            }
            (*fn)(i);
            std::lock_guard<std::mutex> lock(m_);
            if (++done_ == n_) done_cv_.notify_all();
        }
    }
    std::mutex run_m_, m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)>* fn_ = nullptr;
    int n_ = 0, next_ = 0, done_ = 0;
    unsigned long long gen_ = 0;
};

}  // namespace ob
