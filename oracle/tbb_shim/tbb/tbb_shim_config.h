// Minimal stand-in for the parts of Intel TBB that the epi5_MT mechanics
// sources include (TBB is not installed in this image).
//
// TEST INFRASTRUCTURE ONLY: this shim exists so the unmodified reference
// sources can be compiled into the oracle / CPU baseline under oracle/_ref.
// It is never linked into the product library.
//
// Two back ends, chosen at compile time:
//   * serial (default): loops run in index order on one thread. The reference's
//     CAS accumulation then happens in a fixed order, so a serial build is a
//     deterministic FP64 oracle.
//   * EPI_TBB_SHIM_OPENMP: loops become OpenMP parallel loops, which is what
//     the timed CPU baseline uses.
#pragma once
#include <cstddef>
#include <cstdlib>
#include <iterator>
#ifdef EPI_TBB_SHIM_OPENMP
#include <omp.h>
#define EPI_SHIM_PRAGMA(x) _Pragma(#x)
#define EPI_SHIM_PARALLEL_FOR EPI_SHIM_PRAGMA(omp parallel for schedule(dynamic, 256))
#else
#define EPI_SHIM_PARALLEL_FOR
#endif

namespace tbb {
inline int shim_threads() {
#ifdef EPI_TBB_SHIM_OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
}  // namespace tbb
