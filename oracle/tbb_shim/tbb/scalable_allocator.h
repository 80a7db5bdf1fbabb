// TBB stand-in (test infrastructure only): scalable_malloc maps to malloc.
#pragma once
#include "tbb_shim_config.h"

inline void* scalable_malloc(std::size_t n) { return std::malloc(n); }
inline void scalable_free(void* p) { std::free(p); }
