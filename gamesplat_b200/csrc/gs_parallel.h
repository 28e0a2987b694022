// Host-side range parallelism for the loaders: fn(lo, hi) over [0, n) split
// into one contiguous slice per hardware thread (at most 16), the calling
// thread taking the first slice and any slice no thread could be started
// for.  Returns true when every call returned true.  fn must not throw and
// must only write state private to its slice.
#pragma once

#include <algorithm>
#include <cstdint>
#include <exception>
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

}  // namespace gs
