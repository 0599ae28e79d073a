// Stand-in for parlaylib's parlay/parallel.h (not in the reference tree; an
// un-vendored git dependency, CMakeLists.txt:330-339) in the drop-in test: the four
// calls the reference's discontinuity-graph phases make, run on one worker.
// Scheduling only -- results do not depend on it.  Test infrastructure only.
#pragma once

#include <cstddef>

namespace parlay {
inline std::size_t num_workers() { return 1; }
inline std::size_t worker_id() { return 0; }
template <typename F>
inline void parallel_for(std::size_t lo, std::size_t hi, F&& f, long = 0, bool = false) {
    for (std::size_t i = lo; i < hi; ++i) f(i);
}
template <typename L, typename R>
inline void par_do(L&& left, R&& right, bool = false) { left(); right(); }
}  // namespace parlay
