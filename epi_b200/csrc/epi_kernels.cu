// Mechanics kernels for sm_100a: binning, neighbour search, force + commit.
//
// One step of the reference (epi5_MT/proc.cpp:22-32 without state renewal) is
//   k_force_commit  cell_interaction + pos_copy + cell_pos_periodic_fix
//   k_bin           grid_init's binning (+ membrane bending scratch)
//   scan            bin offsets (counting sort)
//   k_scatter       particles into bin order
//   k_binsort       deterministic order inside each bin, sorted position copy
//   k_search        connect_proc's neighbour search + find_dermis
// Every kernel covers a particle range and a bin range, so the same code runs
// a whole batch of tissues per launch or one tissue per launch.
//
// Forces are gathered, not scattered: each particle sums every interaction it
// takes part in (the reference adds +d to c1 and -d to c2 with CAS atomics,
// cell_interaction.cpp:48-66). No atomics touch positions, so a step is
// deterministic and repeatable bit for bit.
#include "epi_kernels.h"

#include <cstdio>

namespace epi {

const char* const kKernelClassNames[KC_COUNT] = {"force_commit", "bin", "scan",
                                                  "scatter", "binsort", "search"};

namespace {

constexpr int kBlock = 256;

inline int blocks_for(int64_t n, int b = kBlock) { return (int)((n + b - 1) / b); }

// ---------------------------------------------------------------------------
// Scan (reduce -> top-level scan -> down-sweep). No inter-block waiting.
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 256;
constexpr int kScanItems = kScanTile / kScanThreads;  // 8

__device__ __forceinline__ int32_t warp_incl_scan(int32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int32_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  return v;
}

// Block-wide exclusive scan of one value per thread; returns the prefix and
// writes the block total to *total.
__device__ __forceinline__ int32_t block_excl_scan(int32_t v, int32_t* total) {
  __shared__ int32_t wsum[kScanThreads / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int32_t incl = warp_incl_scan(v);
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int32_t w = lane < kScanThreads / 32 ? wsum[lane] : 0;
    w = warp_incl_scan(w);
    if (lane < kScanThreads / 32) wsum[lane] = w;
  }
  __syncthreads();
  const int32_t before = wid == 0 ? 0 : wsum[wid - 1];
  *total = wsum[kScanThreads / 32 - 1];
  __syncthreads();
  return before + incl - v;
}

__global__ void k_scan_partial(const int32_t* __restrict__ in, int32_t n,
                               int32_t* __restrict__ partial) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  int32_t tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void k_set1(int32_t* out, int32_t v) { *out = v; }

__global__ void k_scan_top(int32_t* partial, int32_t nb) {
  int32_t carry = 0;
  for (int32_t base = 0; base < nb; base += kScanThreads) {
    const int32_t i = base + threadIdx.x;
    const int32_t v = i < nb ? partial[i] : 0;
    int32_t tot;
    const int32_t ex = block_excl_scan(v, &tot);
    if (i < nb) partial[i] = carry + ex;
    carry += tot;
  }
}

__global__ void k_scan_final(const int32_t* __restrict__ in, int32_t* __restrict__ out,
                             int32_t n, const int32_t* __restrict__ partial, int32_t init) {
  const int64_t base = (int64_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int32_t v[kScanItems];
  int32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  int32_t tot;
  int32_t run = block_excl_scan(s, &tot) + partial[blockIdx.x] + init;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = run;
    run += v[k];
  }
  if (blockIdx.x == gridDim.x - 1 && threadIdx.x == kScanThreads - 1) out[n] = run;
}

// ---------------------------------------------------------------------------
// Binning: grid_init (cell_connection.cpp:38-62) plus the range assert of
// connect_proc (:95-99). Membrane particles also compute their bending
// scratch, _memb_bend_calc1 (cell_interaction.cpp:296-324).
// ---------------------------------------------------------------------------
template <typename R>
__global__ void k_bin(DevState S, Range r) {
  const int32_t i = r.p0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.p1) return;
  const uint32_t a = S.attr[i];
  const TissueDev& T = S.tissues[attr_tissue(a)];
  const double4 p = S.pos_cur[i];
  const uint32_t st = attr_state(a);
  if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) {
    raise_error(S.status, E_NONFINITE, i, -1, p.x);
    S.bin[i] = -1;
    return;
  }
  const int32_t aix = (int32_t)((0.5 * T.lx - pdiff(0.5 * T.lx, p.x, T.lx)) / kAreaGrid);
  const int32_t aiy = (int32_t)((0.5 * T.ly - pdiff(0.5 * T.ly, p.y, T.ly)) / kAreaGrid);
  const int32_t aiz = (int32_t)(fmax(p.z, 0.0) / kAreaGrid);  // min0, utils.h:55-57
  bool bad = aix >= T.anx || aiy >= T.any || aiz >= T.anz || aix < 0 || aiy < 0 || aiz < 0;
  if (st != ST_MEMB) {
    const int32_t cx = (int32_t)(p.x / kAreaGrid), cy = (int32_t)(p.y / kAreaGrid),
                  cz = (int32_t)(p.z / kAreaGrid);
    bad |= cx >= T.anx || cy >= T.any || cz >= T.anz || cx < 0 || cy < 0 || cz < 0;
  }
  if (bad) {
    raise_error(S.status, E_BIN_RANGE, i, -1, p.z);
    S.bin[i] = -1;
    return;
  }
  const int32_t b = T.binbase + (aix * T.any + aiy) * T.anz + aiz;
  const int32_t rk = atomicAdd(&S.counts[b], 1);
  if (rk + 1 >= kBinCap) raise_error(S.status, E_BIN_OVERFLOW, i, b, (double)(rk + 1));
  S.bin[i] = b;
  S.rank[i] = rk;
  if (st == ST_MEMB) {
    const int32_t j = i - T.pbase;
    const Lattice L = lattice_of(j, T.nmx, T.nmy);
    const double4 pr = S.pos_cur[T.pbase + L.r];
    const double4 pu = S.pos_cur[T.pbase + L.u];
    const R nx = R(pdiff(pr.x, p.x, T.lx)), ny = R(pdiff(pr.y, p.y, T.ly)), nz = R(pr.z - p.z);
    const R dn = sqrt(nx * nx + ny * ny + nz * nz);
    S.sn[i] = make_double4(nx / dn, ny / dn, nz / dn, dn);
    const R mx = R(pdiff(pu.x, p.x, T.lx)), my = R(pdiff(pu.y, p.y, T.ly)), mz = R(pu.z - p.z);
    const R dm = sqrt(mx * mx + my * my + mz * mz);
    S.sm[i] = make_double4(mx / dm, my / dm, mz / dm, dm);
  }
}

__global__ void k_scatter(DevState S, Range r) {
  const int32_t i = r.p0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.p1) return;
  const int32_t b = S.bin[i];
  if (b < 0) return;
  S.skey[S.starts[b] + S.rank[i]] = (uint32_t)i;
}

// Per-bin insertion sort by particle index (bins hold a few to a few dozen
// particles), then the sorted position copy the search streams through.
__global__ void k_binsort(DevState S, Range r) {
  const int32_t b = r.b0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= r.b1) return;
  const int32_t s0 = S.starts[b], s1 = S.starts[b + 1];
  S.counts[b] = 0;  // ready for the next binning
  for (int32_t s = s0 + 1; s < s1; ++s) {
    const uint32_t v = S.skey[s];
    int32_t k = s - 1;
    while (k >= s0 && S.skey[k] > v) {
      S.skey[k + 1] = S.skey[k];
      --k;
    }
    S.skey[k + 1] = v;
  }
  for (int32_t s = s0; s < s1; ++s) {
    const uint32_t g = S.skey[s];
    const bool memb = attr_state(S.attr[g]) == ST_MEMB;
    S.skey[s] = g | (memb ? 0x80000000u : 0u);
    S.spos[s] = S.pos_cur[g];
  }
}

// Bin ranges (inclusive) of the periodic window [x-R, x+R] along one axis:
// at most two ranges, because the window may wrap once. Bin k holds
// [k*AG, (k+1)*AG) of [0, L) (the last one is shortened; AG*AN > L).
__device__ __forceinline__ int window_ranges(double x, double R, double L, int32_t an,
                                             int32_t lo[2], int32_t hi[2]) {
  if (2.0 * R >= L) {
    lo[0] = 0;
    hi[0] = an - 1;
    return 1;
  }
  auto bin_of = [&](double v) {
    int32_t k = (int32_t)floor(v / kAreaGrid);
    return k < 0 ? 0 : (k > an - 1 ? an - 1 : k);
  };
  const double a = x - R, b = x + R;
  if (a < 0.0) {
    lo[0] = 0; hi[0] = bin_of(b);
    lo[1] = bin_of(a + L); hi[1] = an - 1;
    if (lo[1] <= hi[0]) { hi[0] = an - 1; return 1; }
    return 2;
  }
  if (b >= L) {
    lo[0] = bin_of(a); hi[0] = an - 1;
    lo[1] = 0; hi[1] = bin_of(b - L);
    if (hi[1] >= lo[0]) { lo[0] = 0; return 1; }
    return 2;
  }
  lo[0] = bin_of(a);
  hi[0] = bin_of(b);
  return 1;
}

// ---------------------------------------------------------------------------
// Neighbour search, connect_proc (cell_connection.cpp:70-129) + find_dermis
// (:158-172). Every particle collects all partners within
// LJ_THRESH*(r_i+r_j), except membrane-membrane pairs, which the reference
// never searches (only non-membrane cells iterate, and their partners include
// membranes). The predicate is symmetric and evaluated with the reference's
// exact rounding, so the sets equal the reference's two-sided pushes. The
// window covers every bin that can hold a partner within reach (radius bound
// rmax of the tissue); the reference's fixed 5x5x5 window is a superset for
// every reachable pair (reach <= 1.2 * 2.8 < 2 * AREA_GRID).
// ---------------------------------------------------------------------------
__global__ void k_search(DevState S, Range r) {
  const int32_t i = r.p0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.p1) return;
  const uint32_t a = S.attr[i];
  const TissueDev& T = S.tissues[attr_tissue(a)];
  const uint32_t st = attr_state(a);
  const bool memb_i = st == ST_MEMB;
  const bool wants_dermis = st == ST_FIX || st == ST_MUSUME;
  const double4 p = S.pos_cur[i];
  const double lt = T.P.lj_thresh;
  const double R = lt * (p.w + T.rmax) + 1e-6;
  int32_t xlo[2], xhi[2], ylo[2], yhi[2];
  const int nxr = window_ranges(p.x, R, T.lx, T.anx, xlo, xhi);
  const int nyr = window_ranges(p.y, R, T.ly, T.any, ylo, yhi);
  int32_t z0 = (int32_t)floor((p.z - R) / kAreaGrid);
  int32_t z1 = (int32_t)floor((p.z + R) / kAreaGrid);
  z0 = z0 < 0 ? 0 : (z0 > T.anz - 1 ? T.anz - 1 : z0);
  z1 = z1 < 0 ? 0 : (z1 > T.anz - 1 ? T.anz - 1 : z1);
  const int64_t N = S.n_total;
  const int32_t cap = S.max_conn;
  int32_t count = 0;
  int32_t best = -1;
  double bestd = T.lx * T.lx;  // find_dermis starts from LX*LX
  for (int xr = 0; xr < nxr; ++xr) {
    for (int32_t bx = xlo[xr]; bx <= xhi[xr]; ++bx) {
      for (int yr = 0; yr < nyr; ++yr) {
        for (int32_t by = ylo[yr]; by <= yhi[yr]; ++by) {
          const int32_t col = T.binbase + (bx * T.any + by) * T.anz;
          const int32_t s_lo = S.starts[col + z0], s_hi = S.starts[col + z1 + 1];
          for (int32_t s = s_lo; s < s_hi; ++s) {
            const uint32_t key = S.skey[s];
            const int32_t j = (int32_t)(key & 0x7fffffffu);
            if (j == i || (memb_i && (key >> 31))) continue;
            const double4 q = S.spos[s];
            const double dx = pdiff(p.x, q.x, T.lx);
            const double dy = pdiff(p.y, q.y, T.ly);
            const double dz = p.z - q.z;
            const double d2 = dist_sq_exact(dx, dy, dz);
            if (!connected_pred(d2, lt, p.w, q.w)) continue;
            if (count < cap) S.nbr[(int64_t)count * N + i] = j;
            ++count;
            if (wants_dermis && (key >> 31) && (d2 < bestd || (d2 == bestd && j < best))) {
              bestd = d2;
              best = j;
            }
          }
        }
      }
    }
  }
  if (count > cap) raise_error(S.status, E_LIST_OVERFLOW, i, -1, (double)count);
  S.nn[i] = count < cap ? count : cap;
  S.dermis[i] = wants_dermis ? best : -1;
}

// ---------------------------------------------------------------------------
// Force + commit: cell_interaction (cell_interaction.cpp:648-685) gathered per
// particle, then pos_copy (cellmanager.cpp:19-26) and the single periodic
// wrap of cell_pos_periodic_fix (:395-414). R is the arithmetic type of the
// force laws (double: FP64 path; float: mixed path). Sums stay in double.
// ---------------------------------------------------------------------------
template <typename R>
__device__ __forceinline__ R dot3(const double4& a, const double4& b) {
  return R(a.x) * R(b.x) + R(a.y) * R(b.y) + R(a.z) * R(b.z);
}

// _memb_bend_diff_factor with NEW_BEND_POT (cell_interaction.cpp:349-360)
template <typename R>
__device__ __forceinline__ R bend_factor(R c) {
  return c >= R(0) ? (R(1) - c) : R(1) / ((R(1) + c) * (R(1) + c));
}

template <typename R>
__device__ __forceinline__ R comp(const double4& v, int k) {
  return R(k == 0 ? v.x : (k == 1 ? v.y : v.z));
}

template <typename R>
__global__ void k_force_commit(DevState S, Range r) {
  const int32_t i = r.p0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.p1) return;
  const uint32_t a = S.attr[i];
  const TissueDev& T = S.tissues[attr_tissue(a)];
  const Laws<R> L(T.P);
  const uint32_t st = attr_state(a);
  const double4 p = S.pos_cur[i];
  const double dt = T.P.dt;
  double ax = 0.0, ay = 0.0, az = 0.0;

  if (st == ST_MEMB) {
    const int32_t j = i - T.pbase;
    const Lattice Lt = lattice_of(j, T.nmx, T.nmy);
    const int32_t pb = T.pbase;
    // _memb_bend_calc2 + _memb_bend_calc3 (:326-449) from calc1's scratch.
    {
      const double4 nv = S.sn[i], nvr = S.sn[pb + Lt.r], nvl = S.sn[pb + Lt.l];
      const double4 nvll = S.sn[pb + Lt.ll], nvbb = S.sn[pb + Lt.bb];
      const double4 nvbbr = S.sn[pb + lattice_of(Lt.bb, T.nmx, T.nmy).r];
      const double4 mv = S.sm[i], mvu = S.sm[pb + Lt.u], mvb = S.sm[pb + Lt.b];
      const double4 mvbb = S.sm[pb + Lt.bb];
      const R ipn = dot3<R>(nv, nvr), ipnl = dot3<R>(nvl, nv), ipnll = dot3<R>(nvll, nvl);
      const R ipm = dot3<R>(mv, mvu), ipmb = dot3<R>(mvb, mv);
      const R ipmbb = dot3<R>(nvbb, nvbbr);  // the reference reads memb_bb's ipn (:380)
      const R dn = R(nv.w), dnl = R(nvl.w), dm = R(mv.w), dmb = R(mvb.w);
      const R fn = bend_factor(ipn), fnl = bend_factor(ipnl), fnll = bend_factor(ipnll);
      const R fm = bend_factor(ipm), fmb = bend_factor(ipmb), fmbb = bend_factor(ipmbb);
      R f[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const R n0 = comp<R>(nv, k), nr = comp<R>(nvr, k), nl = comp<R>(nvl, k),
                nll = comp<R>(nvll, k);
        const R m0 = comp<R>(mv, k), mu = comp<R>(mvu, k), mb = comp<R>(mvb, k),
                mbb = comp<R>(mvbb, k);
        f[k] = -fn * (nr - ipn * n0) / dn +
               fnl * ((n0 - ipnl * nl) / dnl - (nl - ipnl * n0) / dn) +
               fnll * (nll - ipnll * nl) / dnl - fm * (mu - ipm * m0) / dm +
               fmb * ((m0 - ipmb * mb) / dmb - (mb - ipmb * m0) / dm) +
               fmbb * (mbb - ipmbb * mb) / dmb;
      }
      const R s = R(dt * T.P.kbend);
      ax += double(s * f[0]);
      ay += double(s * f[1]);
      az += double(s * f[2]);
    }
    // _MEMB_interaction (:529-547): the four lattice links, each applied once
    // by the higher index.
    const int32_t links[4] = {Lt.l, Lt.r, Lt.b, Lt.u};
#pragma unroll
    for (int k = 0; k < kMembAdj; ++k) {
      const int32_t q = pb + links[k];
      const double4 pq = S.pos_cur[q];
      const bool hi = i > q;
      double dx, dy, dz;
      if (hi) {
        dx = pdiff(p.x, pq.x, T.lx); dy = pdiff(p.y, pq.y, T.ly); dz = p.z - pq.z;
      } else {
        dx = -pdiff(pq.x, p.x, T.lx); dy = -pdiff(pq.y, p.y, T.ly); dz = -(pq.z - p.z);
      }
      const R rdx = R(dx), rdy = R(dy), rdz = R(dz);
      const R d2 = rdx * rdx + rdy * rdy + rdz * rdz;
      bool bad;
      const R c = L.memb_memb(d2, R(p.w + pq.w), &bad);
      if (bad) raise_error(S.status, E_MEMB_COEF_RANGE, hi ? i : q, hi ? q : i, double(c));
      const R sdt = R(dt) * c;
      ax += double(sdt * rdx);
      ay += double(sdt * rdy);
      az += double(sdt * rdz);
    }
  }
  // wall_interaction (:287-294) for MEMB and DER below their radius
  if ((st == ST_MEMB || st == ST_DER) && p.z < p.w) {
    const R z = R(p.z), rad = R(p.w);
    const R distlj = R(2) * z;
    const R lj6 = pow6(rad) / pow6(z);
    const R ljm = L.eps4 * lj6 * (lj6 - R(1)) / (distlj * distlj);
    az += double(R(dt) * ljm * R(2) * z);
  }

  int32_t pair_i = -1, dermis_i = -1;
  if (st != ST_MEMB) {
    pair_i = S.pair[i];
    if (st == ST_FIX || st == ST_MUSUME) dermis_i = S.dermis[i];
    // _pair_interaction (:637-641), from whichever side has the higher index
    if (pair_i >= 0) {
      const double4 pq = S.pos_cur[pair_i];
      const bool hi = i > pair_i;
      double dx, dy, dz;
      if (hi) {
        dx = pdiff(p.x, pq.x, T.lx); dy = pdiff(p.y, pq.y, T.ly); dz = p.z - pq.z;
      } else {
        dx = -pdiff(pq.x, p.x, T.lx); dy = -pdiff(pq.y, p.y, T.ly); dz = -(pq.z - p.z);
      }
      const R rdx = R(dx), rdy = R(dy), rdz = R(dz);
      const R d2 = rdx * rdx + rdy * rdy + rdz * rdz;
      const R c = L.pair(d2, R(hi ? S.spr[i] : S.spr[pair_i]));
      if (fabs(c) > R(1000)) raise_error(S.status, E_COEF_RANGE, i, pair_i, double(c));
      const R sdt = R(dt) * c;
      ax += double(sdt * rdx);
      ay += double(sdt * rdy);
      az += double(sdt * rdz);
    }
  }

  // Searched connections: the law i applies while iterating q (if i is not a
  // membrane particle) and the law q applies while iterating i (if q is not).
  const int64_t N = S.n_total;
  const int32_t nn = S.nn[i];
  const bool old_i = attr_old(a);
  for (int32_t k = 0; k < nn; ++k) {
    const int32_t q = S.nbr[(int64_t)k * N + i];
    const uint32_t aq = S.attr[q];
    const uint32_t sq = attr_state(aq);
    const double4 pq = S.pos_cur[q];
    const double dx = pdiff(p.x, pq.x, T.lx), dy = pdiff(p.y, pq.y, T.ly), dz = p.z - pq.z;
    const R rdx = R(dx), rdy = R(dy), rdz = R(dz);
    const R d2 = rdx * rdx + rdy * rdy + rdz * rdz;
    const R rs = R(p.w + pq.w);
    const bool both_old = old_i && attr_old(aq);
    R coef = R(0);
    if (st != ST_MEMB) {
      const int law = law_of(st, i, pair_i, dermis_i, sq, q);
      if (law != L_NONE) {
        const R c = eval_law<R>(law, L, d2, rs, both_old, attr_sfm(a));
        if (fabs(c) > R(1000)) raise_error(S.status, E_COEF_RANGE, i, q, double(c));
        coef += c;
      }
    }
    if (sq != ST_MEMB) {
      int32_t pair_q = -1, dermis_q = -1;
      if (sq == ST_FIX || sq == ST_MUSUME) {
        pair_q = S.pair[q];
        dermis_q = S.dermis[q];
      }
      const int law = law_of(sq, q, pair_q, dermis_q, st, i);
      if (law != L_NONE) {
        const R c = eval_law<R>(law, L, d2, rs, both_old, attr_sfm(aq));
        if (fabs(c) > R(1000)) raise_error(S.status, E_COEF_RANGE, q, i, double(c));
        coef += c;
      }
    }
    const R sdt = R(dt) * coef;
    ax += double(sdt * rdx);
    ay += double(sdt * rdy);
    az += double(sdt * rdz);
  }

  double nx = p.x + ax, ny = p.y + ay;
  const double nz = p.z + az;
  if (nx > T.lx) nx -= T.lx;
  else if (nx < 0) nx += T.lx;
  if (ny > T.ly) ny -= T.ly;
  else if (ny < 0) ny += T.ly;
  if (!isfinite(nx) || !isfinite(ny) || !isfinite(nz))
    raise_error(S.status, E_NONFINITE, i, -1, nz);
  S.pos_nxt[i] = make_double4(nx, ny, nz, p.w);
}

// ---------------------------------------------------------------------------
// Export helpers (not on the per-step path).
// ---------------------------------------------------------------------------
__global__ void k_rowlen(DevState S, int32_t* rowlen, int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  rowlen[i] = S.nn[i] + (attr_state(S.attr[i]) == ST_MEMB ? kMembAdj : 0);
}

__global__ void k_fill_csr(DevState S, const int32_t* rowoff, int32_t* idx, int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t a = S.attr[i];
  const TissueDev& T = S.tissues[attr_tissue(a)];
  int32_t o = rowoff[i];
  const int32_t o0 = o;
  if (attr_state(a) == ST_MEMB) {
    const Lattice Lt = lattice_of(i - T.pbase, T.nmx, T.nmy);
    idx[o++] = Lt.l;  // push order of _memb_init, cellmanager.cpp:160-163
    idx[o++] = Lt.r;
    idx[o++] = Lt.b;
    idx[o++] = Lt.u;
  }
  const int32_t nn = S.nn[i];
  for (int32_t k = 0; k < nn; ++k) idx[o++] = S.nbr[(int64_t)k * S.n_total + i] - T.pbase;
  for (int32_t s = o0 + 1; s < o; ++s) {
    const int32_t v = idx[s];
    int32_t k = s - 1;
    while (k >= o0 && idx[k] > v) {
      idx[k + 1] = idx[k];
      --k;
    }
    idx[k + 1] = v;
  }
}

__global__ void k_dermis_local(DevState S, int32_t* out, int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t a = S.attr[i];
  const int32_t d = S.dermis[i];
  out[i] = d < 0 ? -1 : d - S.tissues[attr_tissue(a)].pbase;
}

__global__ void k_unpack(DevState S, double* x, double* y, double* z, int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double4 p = S.pos_cur[i];
  x[i] = p.x;
  y[i] = p.y;
  z[i] = p.z;
}

__global__ void k_pack(DevState S, const double* x, const double* y, const double* z,
                       int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double r = S.pos_cur[i].w;
  const double4 p = make_double4(x[i], y[i], z[i], r);
  S.pos_cur[i] = p;
  S.pos_nxt[i] = p;
}

}  // namespace

void launch_scan(const int32_t* in, int32_t* out, int32_t n, int32_t init,
                 const ScanScratch& sc, cudaStream_t s) {
  const int32_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 0) {
    k_set1<<<1, 1, 0, s>>>(out, init);
    return;
  }
  k_scan_partial<<<nb, kScanThreads, 0, s>>>(in, n, sc.partial);
  k_scan_top<<<1, kScanThreads, 0, s>>>(sc.partial, nb);
  k_scan_final<<<nb, kScanThreads, 0, s>>>(in, out, n, sc.partial, init);
}

void launch_connect(const DevState& S, const Range& r, int precision, const ScanScratch& sc,
                    cudaStream_t s, Timer* tm) {
  const int32_t np = r.p1 - r.p0, nbins = r.b1 - r.b0;
  if (np <= 0) return;
  timer_begin(tm, KC_BIN, s);
  if (precision == 1)
    k_bin<float><<<blocks_for(np), kBlock, 0, s>>>(S, r);
  else
    k_bin<double><<<blocks_for(np), kBlock, 0, s>>>(S, r);
  timer_end(tm, KC_BIN, s);
  timer_begin(tm, KC_SCAN, s);
  launch_scan(S.counts + r.b0, S.starts + r.b0, nbins, r.p0, sc, s);
  timer_end(tm, KC_SCAN, s);
  timer_begin(tm, KC_SCATTER, s);
  k_scatter<<<blocks_for(np), kBlock, 0, s>>>(S, r);
  timer_end(tm, KC_SCATTER, s);
  timer_begin(tm, KC_BINSORT, s);
  k_binsort<<<blocks_for(nbins), kBlock, 0, s>>>(S, r);
  timer_end(tm, KC_BINSORT, s);
  timer_begin(tm, KC_SEARCH, s);
  k_search<<<blocks_for(np), kBlock, 0, s>>>(S, r);
  timer_end(tm, KC_SEARCH, s);
}

void launch_interact_commit(const DevState& S, const Range& r, int precision, cudaStream_t s,
                            Timer* tm) {
  const int32_t np = r.p1 - r.p0;
  if (np <= 0) return;
  timer_begin(tm, KC_FORCE, s);
  if (precision == 1)
    k_force_commit<float><<<blocks_for(np), kBlock, 0, s>>>(S, r);
  else
    k_force_commit<double><<<blocks_for(np), kBlock, 0, s>>>(S, r);
  timer_end(tm, KC_FORCE, s);
}

void launch_rowlen(const DevState& S, int32_t* rowlen, int32_t n, cudaStream_t s) {
  if (n > 0) k_rowlen<<<blocks_for(n), kBlock, 0, s>>>(S, rowlen, n);
}
void launch_fill_csr(const DevState& S, const int32_t* rowoff, int32_t* idx, int32_t n,
                     cudaStream_t s) {
  if (n > 0) k_fill_csr<<<blocks_for(n), kBlock, 0, s>>>(S, rowoff, idx, n);
}
void launch_dermis_local(const DevState& S, int32_t* out, int32_t n, cudaStream_t s) {
  if (n > 0) k_dermis_local<<<blocks_for(n), kBlock, 0, s>>>(S, out, n);
}
void launch_unpack_positions(const DevState& S, double* x, double* y, double* z, int32_t n,
                             cudaStream_t s) {
  if (n > 0) k_unpack<<<blocks_for(n), kBlock, 0, s>>>(S, x, y, z, n);
}
void launch_pack_positions(const DevState& S, const double* x, const double* y,
                           const double* z, int32_t n, cudaStream_t s) {
  if (n > 0) k_pack<<<blocks_for(n), kBlock, 0, s>>>(S, x, y, z, n);
}

}  // namespace epi
