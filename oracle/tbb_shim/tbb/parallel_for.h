// TBB stand-in (test infrastructure only): parallel_for over an index interval
// or a range object. Serial unless EPI_TBB_SHIM_OPENMP is defined.
#pragma once
#include "blocked_range.h"
#include "blocked_range3d.h"

namespace tbb {
template <typename Index, typename Func>
void parallel_for(Index first, Index last, const Func& f) {
  const long long n = static_cast<long long>(last) - static_cast<long long>(first);
  EPI_SHIM_PARALLEL_FOR
  for (long long i = 0; i < n; ++i) f(static_cast<Index>(first + static_cast<Index>(i)));
}

template <typename Range, typename Body>
void parallel_for(const Range& range, const Body& body) {
  body(range);
}
}  // namespace tbb
