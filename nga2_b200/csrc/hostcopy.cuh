// hostcopy.cuh -- copies between caller host arrays and device memory.
//
// Page-locked host memory is copied by DMA directly.  Pageable memory (the
// usual case for a Fortran or numpy caller) would go through the CUDA driver's
// single bounce buffer at ~11 GB/s; here it goes through a ring of pinned
// staging buffers instead: several host threads fill (or drain) one chunk
// while the copy engine moves the previous one, so the host-side memcpy and
// the PCIe transfer overlap and the host side runs at multi-threaded memcpy
// speed.  The ring and the threads are created on the first pageable copy.
#pragma once
#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

namespace bbmg {

// A fixed set of threads running the parts of one job at a time; the caller
// works on the job too and returns when every part is done.
class CopyPool {
  public:
    explicit CopyPool(int nworkers) {
        for (int t = 0; t < nworkers; t++) workers_.emplace_back([this] { loop(); });
    }
    ~CopyPool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &w : workers_) w.join();
    }
    void run(int nparts, const std::function<void(int)> &f) {
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &f;
            parts_ = nparts;
            next_ = 0;
            done_ = 0;
            gen_++;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(m_);
        done_cv_.wait(lk, [&] { return done_ == parts_; });
        job_ = nullptr;
    }

  private:
    void work() {
        for (;;) {
            int i;
            const std::function<void(int)> *f;
            {
                std::lock_guard<std::mutex> g(m_);
                if (!job_ || next_ >= parts_) return;
                i = next_++;
                f = job_;
            }
            (*f)(i);
            {
                std::lock_guard<std::mutex> g(m_);
                if (++done_ == parts_) done_cv_.notify_all();
            }
        }
    }
    void loop() {
        long long seen = 0;
        for (;;) {
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
                if (stop_) return;
                seen = gen_;
            }
            work();
        }
    }
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_cv_;
    const std::function<void(int)> *job_ = nullptr;
    int parts_ = 0, next_ = 0, done_ = 0;
    long long gen_ = 0;
    bool stop_ = false;
};

class HostCopier {
  public:
    static constexpr size_t kChunk = size_t(32) << 20;
    static constexpr int kSlots = 3;

    ~HostCopier() { release(); }

    void release() {
        for (int i = 0; i < kSlots; i++) {
            if (busy_[i] && ev_[i]) cudaEventSynchronize(ev_[i]);
            busy_[i] = false;
            if (ev_[i]) cudaEventDestroy(ev_[i]);
            if (stage_[i]) cudaFreeHost(stage_[i]);
            ev_[i] = nullptr;
            stage_[i] = nullptr;
        }
        delete pool_;
        pool_ = nullptr;
    }

    static bool pinned(const void *p) {
        cudaPointerAttributes a;
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return a.type == cudaMemoryTypeHost;
    }

    // host src -> device dst, ordered on stream s; src may be reused on return
    // (pageable chunks are in the staging ring by then, and the CUDA driver stages
    // small pageable copies before returning)
    cudaError_t h2d(void *dst, const void *src, size_t bytes, cudaStream_t s) {
        if (bytes < kChunk || pinned(src)) return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
        cudaError_t e = ensure();
        if (e != cudaSuccess) return e;
        size_t c = 0;
        for (size_t off = 0; off < bytes; off += kChunk, c++) {
            const int sl = next_;
            next_ = (next_ + 1) % kSlots;
            const size_t n = std::min(kChunk, bytes - off);
            if ((e = wait_slot(sl)) != cudaSuccess) return e;
            par_copy(stage_[sl], (const char *)src + off, n);
            if ((e = cudaMemcpyAsync((char *)dst + off, stage_[sl], n, cudaMemcpyHostToDevice, s)) != cudaSuccess)
                return e;
            if ((e = cudaEventRecord(ev_[sl], s)) != cudaSuccess) return e;
            busy_[sl] = true;
        }
        return cudaSuccess;
    }

    // device src -> host dst after the work queued on stream s; synchronous
    cudaError_t d2h(void *dst, const void *src, size_t bytes, cudaStream_t s) {
        if (bytes < kChunk || pinned(dst)) {
            cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, s);
            if (e != cudaSuccess) return e;
            return cudaStreamSynchronize(s);
        }
        cudaError_t e = ensure();
        if (e != cudaSuccess) return e;
        for (int sl = 0; sl < kSlots; sl++)
            if ((e = wait_slot(sl)) != cudaSuccess) return e;
        const size_t nch = (bytes + kChunk - 1) / kChunk;
        auto issue = [&](size_t c) -> cudaError_t {
            const int sl = (int)(c % kSlots);
            const size_t off = c * kChunk, n = std::min(kChunk, bytes - off);
            cudaError_t r = cudaMemcpyAsync(stage_[sl], (const char *)src + off, n, cudaMemcpyDeviceToHost, s);
            if (r != cudaSuccess) return r;
            return cudaEventRecord(ev_[sl], s);
        };
        for (size_t c = 0; c < nch && c < (size_t)kSlots; c++)
            if ((e = issue(c)) != cudaSuccess) return e;
        for (size_t c = 0; c < nch; c++) {
            const int sl = (int)(c % kSlots);
            const size_t off = c * kChunk, n = std::min(kChunk, bytes - off);
            if ((e = cudaEventSynchronize(ev_[sl])) != cudaSuccess) return e;
            par_copy((char *)dst + off, stage_[sl], n);
            if (c + kSlots < nch && (e = issue(c + kSlots)) != cudaSuccess) return e;
        }
        return cudaSuccess;
    }

  private:
    // a slot whose last DMA may still be running is waited for before reuse
    cudaError_t wait_slot(int sl) {
        if (!busy_[sl]) return cudaSuccess;
        busy_[sl] = false;
        return cudaEventSynchronize(ev_[sl]);
    }
    cudaError_t ensure() {
        for (int i = 0; i < kSlots; i++) {
            if (!stage_[i]) {
                cudaError_t e = cudaHostAlloc(&stage_[i], kChunk, cudaHostAllocDefault);
                if (e != cudaSuccess) return e;
            }
            if (!ev_[i]) {
                cudaError_t e = cudaEventCreateWithFlags(&ev_[i], cudaEventDisableTiming);
                if (e != cudaSuccess) return e;
            }
        }
        if (!pool_) {
            unsigned hc = std::thread::hardware_concurrency();
            nthreads_ = (int)std::max(1u, std::min(8u, hc ? hc : 1u));
            pool_ = new CopyPool(nthreads_ - 1);
        }
        return cudaSuccess;
    }
    void par_copy(void *dst, const void *src, size_t n) {
        const int parts = nthreads_;
        const size_t piece = (n / parts + 63) & ~size_t(63);
        pool_->run(parts, [&](int i) {
            const size_t o = (size_t)i * piece;
            if (o < n) memcpy((char *)dst + o, (const char *)src + o, std::min(piece, n - o));
        });
    }
    void *stage_[kSlots] = {nullptr, nullptr, nullptr};
    cudaEvent_t ev_[kSlots] = {nullptr, nullptr, nullptr};
    bool busy_[kSlots] = {false, false, false};
    int next_ = 0;
    CopyPool *pool_ = nullptr;
    int nthreads_ = 1;
};

}  // namespace bbmg
