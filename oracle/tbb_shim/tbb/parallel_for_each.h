// TBB stand-in (test infrastructure only): parallel_for_each over a random
// access iterator pair. The serial back end visits elements in order.
#pragma once
#include "tbb_shim_config.h"

namespace tbb {
template <typename It, typename Func>
void parallel_for_each(It first, It last, const Func& f) {
  const long long n = static_cast<long long>(last - first);
  EPI_SHIM_PARALLEL_FOR
  for (long long i = 0; i < n; ++i) f(first[i]);
}
}  // namespace tbb
