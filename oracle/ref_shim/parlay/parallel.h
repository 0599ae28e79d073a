// Stand-in for parlaylib's parlay/parallel.h (an un-vendored git dependency of the
// reference, CMakeLists.txt:330-339), for building the reference's own code here: the
// four calls it makes.  Workers are PARLAY_NUM_THREADS threads (default: the hardware
// threads); worker_id() is 0 on the calling thread and 1..n-1 on the helpers a
// parallel_for starts; a parallel_for inside a worker runs on that worker alone, so
// worker ids stay unique among the threads running at once.  Scheduling only -- results
// do not depend on it.  Test and baseline infrastructure only.
#pragma once

#include <atomic>
#include <cstddef>
#include <cstdlib>
#include <thread>
#include <vector>

namespace parlay {

namespace shim {
inline std::size_t& worker_slot() { thread_local std::size_t id = 0; return id; }
inline bool& in_parallel() { thread_local bool busy = false; return busy; }
}  // namespace shim

inline std::size_t num_workers() {
    static const std::size_t n = [] {
        const char* e = std::getenv("PARLAY_NUM_THREADS");
        const long v = e ? std::atol(e) : 0;
        const std::size_t hw = std::thread::hardware_concurrency();
        return v > 0 ? (std::size_t)v : (hw ? hw : 1);
    }();
    return n;
}

inline std::size_t worker_id() { return shim::worker_slot(); }

template <typename F>
inline void parallel_for(std::size_t lo, std::size_t hi, F&& f, long granularity = 0, bool = false) {
    if (hi <= lo) return;
    const std::size_t n = hi - lo, W = num_workers();
    if (W == 1 || n == 1 || shim::in_parallel()) {
        for (std::size_t i = lo; i < hi; ++i) f(i);
        return;
    }
    const std::size_t chunk = granularity > 0 ? (std::size_t)granularity : (n + 8 * W - 1) / (8 * W);
    std::atomic<std::size_t> next(lo);
    auto body = [&](std::size_t id) {
        const std::size_t saved = shim::worker_slot();
        shim::worker_slot() = id;
        shim::in_parallel() = true;
        for (;;) {
            const std::size_t a = next.fetch_add(chunk);
            if (a >= hi) break;
            const std::size_t b = a + chunk < hi ? a + chunk : hi;
            for (std::size_t i = a; i < b; ++i) f(i);
        }
        shim::in_parallel() = false;
        shim::worker_slot() = saved;
    };
    const std::size_t T = W < (n + chunk - 1) / chunk ? W : (n + chunk - 1) / chunk;
    std::vector<std::thread> helpers;
    for (std::size_t t = 1; t < T; ++t) helpers.emplace_back(body, t);
    body(shim::worker_slot());
    for (auto& h : helpers) h.join();
}

template <typename L, typename R>
inline void par_do(L&& left, R&& right, bool = false) { left(); right(); }

}  // namespace parlay
