// TBB stand-in (test infrastructure only): one-dimensional iteration range.
#pragma once
#include "tbb_shim_config.h"

namespace tbb {
template <typename T>
class blocked_range {
  T b_, e_;

 public:
  blocked_range(T b, T e, std::size_t = 1) : b_(b), e_(e) {}
  T begin() const { return b_; }
  T end() const { return e_; }
  std::size_t size() const { return static_cast<std::size_t>(e_ - b_); }
  bool empty() const { return !(b_ < e_); }
};
}  // namespace tbb
