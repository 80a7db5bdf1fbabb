// Cell maps and external-stimulus diffusion, FP64: the rest of the
// reference's per-step loop before its chemistry (epi5_MT/proc.cpp:152-157).
//
// Per tissue, on an (nx+1) x (ny+1) x (nz+1) grid (z fastest, the layout of
// FArr3D, define.h:243):
//   k_field_zzmax    calc_zzmax (proc.cpp:34-43): highest DEAD / ALIVE /
//                    MUSUME / FIX cell, and the diffusion's z bound
//   k_field_stamp    setup_map_lat (map.cpp:24-167): every cell marks the
//                    grid points inside its radius in cmap1 and, for ALIVE /
//                    FIX / MUSUME, inside FAC_MAP times its radius in cmap2.
//                    Where spheres overlap the reference (in index order)
//                    keeps the highest-index cell; atomicMax on index + 1
//                    gives the same answer in any order.
//   k_field_copy_*   the periodic plane copies of both routines
//   k_ext_stim       calc_ext_stim (ext_stim.cpp:18-69): 7-point diffusion
//                    with cmap2 as the conductance mask and the cornification
//                    source fB, below the z bound; evaluated with the
//                    reference's operation order and no fused multiply-adds,
//                    so results are bit-identical.
#include "epi_kernels.h"
#include "epi_device.cuh"

namespace epi {
namespace {

constexpr double kRad = 1.4;          // Rad, map.cpp:26
constexpr double kFacMap = 2.0;       // FAC_MAP, define.h:184
constexpr double kRMax = 1.4;         // R_max, define.h:116
constexpr double kDtCa = 0.01;        // DT_Ca, define.h:89
constexpr double kDB = 0.0009;        // DB, ext_stim.cpp:20
constexpr double kKb = 0.025;         // kb, ext_stim.cpp:10
constexpr double kDurAlive = 0.5;     // ext_stim.cpp:11
constexpr double kDurDead = 2.0;      // ext_stim.cpp:12
constexpr double kThreshDead = 22.0;  // THRESH_DEAD, define.h:156

__device__ __forceinline__ int64_t fidx(const FieldDev& F, int32_t a, int32_t b, int32_t c) {
  return F.base + ((int64_t)a * (F.ny + 1) + b) * (F.nz + 1) + c;
}

__device__ __forceinline__ bool afm_state(uint32_t s) {
  return s == ST_ALIVE || s == ST_FIX || s == ST_MUSUME;
}

__global__ void k_field_clear(FieldState FS) {
  GRID_STRIDE(v, 0, FS.nvox) {
    FS.cmap1[v] = 0;
    FS.cmap2[v] = 0;
  }
}

// zzmax of every tissue: the z of its qualifying cells folded in with
// atomicMax on the bit patterns (non-negative doubles order like their
// bits; zzmax starts at 0), so the result does not depend on the order.
// Lanes of a warp holding the same tissue first fold their values with
// shuffles, so one atomic per (warp, tissue) run reaches memory.
__global__ void __launch_bounds__(256) k_field_zzmax(DevState S, FieldState FS) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const int64_t base0 = (int64_t)blockIdx.x * blockDim.x;
  for (int64_t base = base0; base < S.n_total; base += stride) {
    const int64_t i = base + threadIdx.x;
    int32_t t = -1;
    unsigned long long z = 0;
    if (i < S.n_total) {
      const uint32_t a = S.attr[i];
      const uint32_t st = attr_state(a);
      t = attr_tissue(a);
      if (st == ST_DEAD || st == ST_ALIVE || st == ST_MUSUME || st == ST_FIX) {
        const double zd = S.pos_cur[i].z;
        if (zd > 0.0) z = (unsigned long long)__double_as_longlong(zd);
      }
    }
    const int lane = threadIdx.x & 31;
    // same-tissue lanes form contiguous runs (particles are grouped by tissue)
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const unsigned long long zo = __shfl_down_sync(0xffffffffu, z, o);
      const int32_t to = __shfl_down_sync(0xffffffffu, t, o);
      if (lane + o < 32 && to == t && zo > z) z = zo;
    }
    const int32_t tprev = __shfl_up_sync(0xffffffffu, t, 1);
    if (t >= 0 && z > 0 && (lane == 0 || tprev != t))
      atomicMax(reinterpret_cast<unsigned long long*>(&FS.zzmax[t]), z);
  }
}

// The diffusion's z bound per tissue, (int)((zzmax + FAC_MAP R_max) inv_dz)
// (ext_stim.cpp:22).
__global__ void k_field_bound(DevState S, FieldState FS) {
  GRID_STRIDE(t, 0, S.ntissues) {
    const FieldDev& F = FS.fd[t];
    const double zz = FS.zzmax[t];
    const int32_t izb = (int32_t)(__dmul_rn(__dadd_rn(zz, kFacMap * kRMax), F.inv_dz));
    // beyond the grid the reference would read outside its arrays
    if (izb > F.nz) raise_error(S.status, E_UNSUPPORTED, S.tissues[t].pbase, -1, zz);
    FS.izb[t] = izb > F.nz ? F.nz : izb;
  }
}

// One thread per (particle, x offset, y offset) of the widest window (wmax
// x wmax columns per particle), each walking its z column: set_lattice and
// the two branches of setup_map_lat.
template <typename Index>
__global__ void __launch_bounds__(256) k_field_stamp(DevState S, FieldState FS, int32_t wmax) {
  const Index cols = (Index)wmax * (Index)wmax;
  const Index total = (Index)S.n_total * cols;
  for (Index g = (Index)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (Index)gridDim.x * blockDim.x) {
    const Index i = g / cols;
    const int32_t col = (int32_t)(g - i * cols);
    const uint32_t a = S.attr[i];
    const int32_t t = attr_tissue(a);
    const TissueDev& T = S.tissues[t];
    const FieldDev& F = FS.fd[t];
    const double4 p = S.pos_cur[i];
    const int32_t lat0 = ((int32_t)(p.x * F.inv_dx) + F.nx) % F.nx;
    const int32_t lat1 = ((int32_t)(p.y * F.inv_dy) + F.ny) % F.ny;
    const int32_t lat2 = ((int32_t)(p.z * F.inv_dz) + F.nz) % F.nz;
    const bool afm = afm_state(attr_state(a));
    const int32_t rx = afm ? 2 * F.irx : F.irx, ry = afm ? 2 * F.iry : F.iry;
    const int32_t rz = afm ? 2 * F.irz : F.irz;
    const double normal_radSq = __dmul_rn(p.w, p.w);
    const double crad = __dmul_rn(kFacMap, p.w);
    const double cradSq = __dmul_rn(crad, crad);
    const int32_t z_b = lat2 - rz, z_u = lat2 + rz;
    const int32_t zmin = z_b >= 1 ? z_b : 1;
    const int32_t zmax = z_u < F.nz ? z_u : F.nz - 1;
    const int32_t mark = (int32_t)i - T.pbase + 1;
    const int32_t ox = col / wmax, oy = col % wmax;
    if (ox > 2 * rx || oy > 2 * ry) continue;  // outside this particle's window
    {
      const int32_t kx = lat0 - rx + ox;
      const double diffx = pdiff(__dmul_rn((double)kx, F.dx), p.x, T.lx);
      const double diffxSq = __dmul_rn(diffx, diffx);
      const int32_t ipx = (kx + F.nx) % F.nx;
      {
        const int32_t ly = lat1 - ry + oy;
        const double diffy = pdiff(__dmul_rn((double)ly, F.dy), p.y, T.ly);
        const double tmps = __dadd_rn(diffxSq, __dmul_rn(diffy, diffy));
        const int32_t ipy = (ly + F.ny) % F.ny;
        for (int32_t mz = zmin; mz <= zmax; ++mz) {
          const double diffz = __dsub_rn(__dmul_rn((double)mz, F.dz), p.z);
          const double distSq = __dadd_rn(tmps, __dmul_rn(diffz, diffz));
          const int64_t v = fidx(F, ipx, ipy, mz);
          if (afm) {
            if (distSq < cradSq) {
              FS.cmap2[v] = 1;
              if (distSq < normal_radSq) atomicMax(&FS.cmap1[v], mark);
            }
          } else if (distSq < normal_radSq) {
            atomicMax(&FS.cmap1[v], mark);
          }
        }
      }
    }
  }
}

// Periodic plane copies of setup_map_lat (map.cpp:156-166), y plane first.
// blockIdx.y = tissue.
__global__ void k_field_copy_map_y(FieldState FS) {
  const FieldDev& F = FS.fd[blockIdx.y];
  const int64_t m = (int64_t)(F.nx + 1) * F.nz;
  for (int64_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    const int32_t j = (int32_t)(e / F.nz), l = (int32_t)(e % F.nz);
    FS.cmap2[fidx(F, j, F.ny, l)] = FS.cmap2[fidx(F, j, 0, l)];
    FS.cmap1[fidx(F, j, F.ny, l)] = FS.cmap1[fidx(F, j, 0, l)];
  }
}
__global__ void k_field_copy_map_x(FieldState FS) {
  const FieldDev& F = FS.fd[blockIdx.y];
  const int64_t m = (int64_t)(F.ny + 1) * F.nz;
  for (int64_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    const int32_t k = (int32_t)(e / F.nz), l = (int32_t)(e % F.nz);
    FS.cmap2[fidx(F, F.nx, k, l)] = FS.cmap2[fidx(F, 0, k, l)];
    FS.cmap1[fidx(F, F.nx, k, l)] = FS.cmap1[fidx(F, 0, k, l)];
  }
}

// fB, ext_stim.cpp:8-16
__device__ __forceinline__ double source_fB(double age, double B, bool cornif) {
  const bool on = cornif && age > kThreshDead - kDurAlive && age <= kThreshDead + kDurDead;
  return __dsub_rn(on ? 1.0 : 0.0, __dmul_rn(kKb, B));
}

// calc_ext_stim's update, one thread per grid point below the z bound.
// blockIdx.y = tissue.
__global__ void __launch_bounds__(256) k_ext_stim(DevState S, FieldState FS) {
  const int32_t t = blockIdx.y;
  const TissueDev& T = S.tissues[t];
  const FieldDev& F = FS.fd[t];
  const int32_t izb = FS.izb[t];
  const int64_t m = (int64_t)F.nx * F.ny * izb;
  for (int64_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    const int32_t l = (int32_t)(e % izb);
    const int64_t r = e / izb;
    const int32_t k = (int32_t)(r % F.ny), j = (int32_t)(r / F.ny);
    const int32_t px = j == 0 ? F.nx - 1 : j - 1, nx = j + 1 == F.nx ? 0 : j + 1;
    const int32_t py = k == 0 ? F.ny - 1 : k - 1, ny = k + 1 == F.ny ? 0 : k + 1;
    const int32_t pz = l == 0 ? 1 : l - 1, nz = l + 1 == F.nz ? F.nz - 1 : l + 1;
    double age = 0.0;
    bool cornif = false;
    const int32_t cm = FS.cmap1[fidx(F, j, k, l)] - 1;
    if (cm >= 0) {
      const int32_t ci = T.pbase + cm;
      const uint32_t st = attr_state(S.attr[ci]);
      if (st == ST_DEAD || st == ST_ALIVE) {
        age = FS.agek[ci];
        cornif = true;
      }
    }
    const double* c = FS.cur;
    const int64_t v = fidx(F, j, k, l);
    const double cext = c[v];
    auto term = [&](int64_t w) {
      return __dmul_rn((double)FS.cmap2[w], __dsub_rn(c[w], cext));
    };
    double sum = term(fidx(F, px, k, l));
    sum = __dadd_rn(sum, term(fidx(F, j, py, l)));
    sum = __dadd_rn(sum, term(fidx(F, j, k, pz)));
    sum = __dadd_rn(sum, term(fidx(F, j, k, nz)));
    sum = __dadd_rn(sum, term(fidx(F, j, ny, l)));
    sum = __dadd_rn(sum, term(fidx(F, nx, k, l)));
    const double diff = __dmul_rn(__dmul_rn(__dmul_rn(kDB, sum), F.inv_dz), F.inv_dz);
    FS.nxt[v] = __dadd_rn(cext, __dmul_rn(kDtCa, __dadd_rn(diff, source_fB(age, cext, cornif))));
  }
}

// Periodic plane copies of calc_ext_stim (ext_stim.cpp:63-66) below the z
// bound, y plane (j < nx) first. blockIdx.y = tissue.
__global__ void k_ext_copy_y(FieldState FS) {
  const FieldDev& F = FS.fd[blockIdx.y];
  const int32_t izb = FS.izb[blockIdx.y];
  const int64_t m = (int64_t)F.nx * izb;
  for (int64_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    const int32_t j = (int32_t)(e / izb), l = (int32_t)(e % izb);
    FS.nxt[fidx(F, j, F.ny, l)] = FS.nxt[fidx(F, j, 0, l)];
  }
}
__global__ void k_ext_copy_x(FieldState FS) {
  const FieldDev& F = FS.fd[blockIdx.y];
  const int32_t izb = FS.izb[blockIdx.y];
  const int64_t m = (int64_t)(F.ny + 1) * izb;
  for (int64_t e = blockIdx.x * blockDim.x + threadIdx.x; e < m; e += gridDim.x * blockDim.x) {
    const int32_t k = (int32_t)(e / izb), l = (int32_t)(e % izb);
    FS.nxt[fidx(F, F.nx, k, l)] = FS.nxt[fidx(F, 0, k, l)];
  }
}

}  // namespace

void field_params(FieldDev& F, double lx, double ly, double lz, int32_t nx, int32_t ny,
                  int32_t nz) {
  F.nx = nx;
  F.ny = ny;
  F.nz = nz;
  // cdefd dx = LX / NX; inv_dx = NX / LX (define.h:111-113)
  F.dx = lx / (double)nx;
  F.dy = ly / (double)ny;
  F.dz = lz / (double)nz;
  F.inv_dx = (double)nx / lx;
  F.inv_dy = (double)ny / ly;
  F.inv_dz = (double)nz / lz;
  // irx = (int)(Rad * NX / LX), map.cpp:28-30
  F.irx = (int32_t)(kRad * (double)nx / lx);
  F.iry = (int32_t)(kRad * (double)ny / ly);
  F.irz = (int32_t)(kRad * (double)nz / lz);
}

void launch_field_step(const DevState& S, const FieldState& FS, int32_t wmax,
                       const LaunchCfg& lc, cudaStream_t s) {
  const int nt = S.ntissues;
  const int grid = lc.num_sms * 8;
  cudaMemsetAsync(FS.zzmax, 0, sizeof(double) * nt, s);
  if (S.n_total > 0) k_field_zzmax<<<stride_blocks(S.n_total, 256, lc), 256, 0, s>>>(S, FS);
  k_field_bound<<<(nt + 255) / 256, 256, 0, s>>>(S, FS);
  k_field_clear<<<grid, 256, 0, s>>>(FS);
  const int64_t columns = S.n_total * (int64_t)wmax * wmax;
  if (columns > 0) {
    // 32-bit index arithmetic whenever the columns fit
    if (columns + (int64_t)lc.num_sms * 8 * 256 < (int64_t)UINT32_MAX)
      k_field_stamp<uint32_t><<<stride_blocks(columns, 256, lc), 256, 0, s>>>(S, FS, wmax);
    else
      k_field_stamp<uint64_t><<<stride_blocks(columns, 256, lc), 256, 0, s>>>(S, FS, wmax);
  }
  const dim3 g2(64, nt);
  k_field_copy_map_y<<<g2, 256, 0, s>>>(FS);
  k_field_copy_map_x<<<g2, 256, 0, s>>>(FS);
  const dim3 g3(lc.num_sms * 8 / (nt < 8 ? nt : 8) + 1, nt);
  k_ext_stim<<<g3, 256, 0, s>>>(S, FS);
  k_ext_copy_y<<<g2, 256, 0, s>>>(FS);
  k_ext_copy_x<<<g2, 256, 0, s>>>(FS);
}

}  // namespace epi
