// TBB stand-in (test infrastructure only): task_group runs tasks inline.
#pragma once
#include "tbb_shim_config.h"

namespace tbb {
class task_group {
 public:
  template <typename F>
  void run(const F& f) { f(); }
  template <typename F>
  void run_and_wait(const F& f) { f(); }
  void wait() {}
};
}  // namespace tbb
