// Host-side range parallelism for the loaders: fn(lo, hi) over [0, n) split
// into one contiguous slice per hardware thread (at most 16), the calling
// thread taking the first slice and any slice no thread could be started
// for.  Returns true when every call returned true.  fn must not throw and
// must only write state private to its slice.
#pragma once

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <exception>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

namespace gs {

template <class F>
bool parallel_ranges(uint64_t n, uint64_t min_per_slice, F&& fn) {
    const unsigned hw = std::thread::hardware_concurrency();
    uint64_t slices = std::min<uint64_t>(hw ? hw : 1u, 16u);
    slices = std::max<uint64_t>(1u, std::min<uint64_t>(slices, n / std::max<uint64_t>(min_per_slice, 1u)));
    if (slices <= 1) return fn(uint64_t(0), n);
    const uint64_t per = (n + slices - 1) / slices;
    std::vector<char> ok((size_t)slices, 1);
    std::vector<std::thread> pool;
    uint64_t started = 1;   // slices [1, started) run on their own threads
    try {
        pool.reserve((size_t)slices - 1);
        for (uint64_t w = 1; w < slices && w * per < n; ++w) {
            const uint64_t lo = w * per, hi = std::min(n, lo + per);
            pool.emplace_back([&ok, &fn, w, lo, hi] { ok[w] = fn(lo, hi) ? 1 : 0; });
            started = w + 1;
        }
    } catch (const std::exception&) {   // no memory or no more threads: the rest runs here
    }
    ok[0] = fn(uint64_t(0), std::min(n, per)) ? 1 : 0;
    for (uint64_t w = started; w < slices && w * per < n; ++w) ok[w] = fn(w * per, std::min(n, w * per + per)) ? 1 : 0;
    for (auto& t : pool) t.join();
    return std::all_of(ok.begin(), ok.end(), [](char c) { return c != 0; });
}

// A fixed set of worker threads for a loader that processes many blocks:
// run(n, fn) calls fn(lo, hi) over [0, n) in one slice per worker plus one
// for the calling thread, and returns when all slices are done.  The threads
// are started once (as many as could be started, at most `workers`) and
// joined by the destructor.  fn must not throw and must only write state
// private to its slice.
class WorkerPool {
  public:
    explicit WorkerPool(unsigned workers) {
        try {
            for (unsigned w = 0; w < workers; ++w) threads_.emplace_back([this, w] { loop(w); });
        } catch (const std::exception&) {   // no memory or no more threads: fewer workers
        }
    }
    ~WorkerPool() {
        {
            std::lock_guard<std::mutex> lk(m_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto& t : threads_) t.join();
    }
    WorkerPool(const WorkerPool&) = delete;
    WorkerPool& operator=(const WorkerPool&) = delete;

    void run(uint64_t n, const std::function<void(uint64_t, uint64_t)>& fn) {
        const uint64_t slices = (uint64_t)threads_.size() + 1;
        const uint64_t per = (n + slices - 1) / slices;
        {
            std::lock_guard<std::mutex> lk(m_);
            fn_ = &fn;
            n_ = n;
            per_ = per;
            pending_ = threads_.size();
            ++generation_;
        }
        cv_.notify_all();
        fn(0, std::min(n, per));   // the calling thread's slice
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return pending_ == 0; });
        fn_ = nullptr;
    }

  private:
    void loop(unsigned w) {
        uint64_t seen = 0;
        for (;;) {
            const std::function<void(uint64_t, uint64_t)>* fn;
            uint64_t lo, hi;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return stop_ || generation_ != seen; });
                if (stop_) return;
                seen = generation_;
                fn = fn_;
                lo = std::min(n_, (uint64_t)(w + 1) * per_);
                hi = std::min(n_, lo + per_);
            }
            if (lo < hi) (*fn)(lo, hi);
            {
                std::lock_guard<std::mutex> lk(m_);
                if (--pending_ == 0) done_.notify_one();
            }
        }
    }

    std::vector<std::thread> threads_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void(uint64_t, uint64_t)>* fn_ = nullptr;
    uint64_t n_ = 0, per_ = 0, generation_ = 0;
    size_t pending_ = 0;
    bool stop_ = false;
};

}  // namespace gs
