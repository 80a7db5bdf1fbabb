// TBB stand-in (test infrastructure only): three-dimensional iteration range.
#pragma once
#include "blocked_range.h"

namespace tbb {
template <typename T>
class blocked_range3d {
  blocked_range<T> p_, r_, c_;

 public:
  blocked_range3d(T p0, T p1, T r0, T r1, T c0, T c1)
      : p_(p0, p1), r_(r0, r1), c_(c0, c1) {}
  const blocked_range<T>& pages() const { return p_; }
  const blocked_range<T>& rows() const { return r_; }
  const blocked_range<T>& cols() const { return c_; }
};
}  // namespace tbb
