// Device helpers shared by the step and adjoint kernels (internal).
#pragma once
#include "epi_kernels.h"

namespace epi {
namespace {

inline int blocks_for(int64_t n, int b) { return (int)((n + b - 1) / b); }
inline int stride_blocks(int64_t n, int b, const LaunchCfg& lc) {
  const int need = blocks_for(n, b);
  const int cap = lc.num_sms * 8;
  return need < cap ? (need > 0 ? need : 1) : cap;
}

// Programmatic dependent launch. Kernels of the step sequence are launched
// with programmatic stream serialisation, so each may be scheduled while its
// predecessor's last blocks still run. pdl_entry() is the first statement of
// such a kernel: it lets the next kernel be scheduled, then waits until the
// predecessor has completed and its writes are visible (griddepcontrol.wait
// returns at once for a kernel launched without the attribute). Every kernel
// therefore starts its real work only after all earlier work on the stream.
__device__ __forceinline__ void pdl_entry() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

// One count per kernel launch (the first thread of the first block).
__device__ __forceinline__ void count_launch(unsigned long long* launches) {
  if (launches && blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) atomicAdd(launches, 1ull);
}

template <typename... Params, typename... Args>
void launch_pdl(void (*kernel)(Params...), int grid, int block, cudaStream_t s, Args... args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, static_cast<Params>(args)...);
}

#define GRID_STRIDE(i, lo, hi) \
  for (int64_t i = (lo) + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (hi); \
       i += (int64_t)gridDim.x * blockDim.x)

// _memb_bend_diff_factor with NEW_BEND_POT (cell_interaction.cpp:349-360)
template <typename R>
__device__ __forceinline__ R bend_factor(R c) {
  return c >= R(0) ? (R(1) - c) : R(1) / ((R(1) + c) * (R(1) + c));
}

// Separation of a pair as cell_interaction_apply computes it for its c1
// (:56-58), seen from particle i: the reference adds +d to c1, -d to c2.
__device__ __forceinline__ void pair_sep(const double4& p, const double4& pq, bool i_is_c1,
                                         const TissueDev& T, double& dx, double& dy, double& dz) {
  if (i_is_c1) {
    dx = pdiff(p.x, pq.x, T.lx);
    dy = pdiff(p.y, pq.y, T.ly);
    dz = p.z - pq.z;
  } else {
    dx = -pdiff(pq.x, p.x, T.lx);
    dy = -pdiff(pq.y, p.y, T.ly);
    dz = -(pq.z - p.z);
  }
}

// Reciprocal square root and division: correctly rounded in the FP64 path,
// the hardware approximations (about 2 ulp) in the FP32 path.
__device__ __forceinline__ float frsqrt(float v) { return rsqrtf(v); }
__device__ __forceinline__ double frsqrt(double v) { return 1.0 / sqrt(v); }
__device__ __forceinline__ float fdiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double fdiv(double a, double b) { return a / b; }

template <typename R>
struct Vec3 {
  R x, y, z;
};
// Offset of a lattice neighbour from the particle (minimum image).
template <typename R>
__device__ __forceinline__ Vec3<R> offset_of(const double4& q, const double4& p,
                                             const TissueDev& T) {
  return Vec3<R>{R(pdiff_h(q.x, p.x, T.lx, T.hlx)), R(pdiff_h(q.y, p.y, T.ly, T.hly)),
                 R(q.z - p.z)};
}
// Unit vector and length of b - a: the nv / dn (or mv / dm) that
// _memb_bend_calc1 stores for a membrane particle (cell_interaction.cpp:296-309).
template <typename R>
struct Unit {
  R x, y, z, d;
};
template <typename R>
__device__ __forceinline__ Unit<R> unit_of(R x, R y, R z) {
  const R s = x * x + y * y + z * z;
  const R inv = frsqrt(s);
  return Unit<R>{x * inv, y * inv, z * inv, s * inv};
}
template <typename R>
__device__ __forceinline__ Unit<R> unit_ab(const Vec3<R>& a, const Vec3<R>& b) {
  return unit_of(b.x - a.x, b.y - a.y, b.z - a.z);
}
template <typename R>
__device__ __forceinline__ R dotu(const Unit<R>& a, const Unit<R>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename R>
__device__ __forceinline__ R cmp(const Unit<R>& v, int k) {
  return k == 0 ? v.x : (k == 1 ? v.y : v.z);
}

}  // namespace
}  // namespace epi
