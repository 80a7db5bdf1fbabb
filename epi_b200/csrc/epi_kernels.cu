// Mechanics kernels for sm_100a.
//
// One step of the reference (epi5_MT/proc.cpp:22-32 without state renewal)
// runs as
//   [rebuild]  Verlet candidate rebuild of the tissues that need one
//              (bin -> scan -> scatter -> per-bin sort -> candidate search);
//              every kernel of it exits at once when no tissue does
//   k_prepass  membrane bending scratch (_memb_bend_calc1) and the dermis of
//              FIX / MUSUME cells (find_dermis)
//   k_step     connect_proc's exact predicate over the candidates, every
//              force of cell_interaction, pos_copy and the periodic wrap,
//              fused; flags tissues whose particles moved more than skin/2
//              since their last rebuild
//
// The reference rebuilds its connection lists from scratch every step
// (connect_cell, cell_connection.cpp:191-203). Here a tissue's candidate list
// holds every partner within LJ_THRESH*(r_i+r_j) + skin at the last rebuild;
// while no particle has moved more than skin/2 since, every pair that can
// satisfy the reference's predicate is a candidate, and k_step evaluates that
// predicate exactly (same rounding as the reference) on the current
// positions. The connection set of every step is therefore the reference's.
//
// Forces are gathered, not scattered: each particle sums every interaction it
// takes part in (the reference adds +d to c1 and -d to c2 with CAS atomics,
// cell_interaction.cpp:48-66). No atomics touch positions, so a step is
// deterministic and repeatable bit for bit.
#include "epi_kernels.h"

#include <type_traits>
#include "epi_device.cuh"

namespace epi {

#ifdef EPI_CHECK
constexpr bool kCheck = true;
#else
constexpr bool kCheck = false;
#endif

const char* const kKernelClassNames[KC_COUNT] = {
    "step", "prepass", "rebuild_bin", "rebuild_scan", "rebuild_sort", "rebuild_search", "gate"};

namespace {

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

// Same for NT threads (a multiple of 32, at most 1024).
template <int NT>
__device__ __forceinline__ int32_t block_excl_scan_n(int32_t v, int32_t* total) {
  __shared__ int32_t wsum[NT / 32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int32_t incl = warp_incl_scan(v);
  if (lane == 31) wsum[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    int32_t w = lane < NT / 32 ? wsum[lane] : 0;
    w = warp_incl_scan(w);
    if (lane < NT / 32) wsum[lane] = w;
  }
  __syncthreads();
  const int32_t before = wid == 0 ? 0 : wsum[wid - 1];
  *total = wsum[NT / 32 - 1];
  __syncthreads();
  return before + incl - v;
}

__device__ __forceinline__ bool closed(const int32_t* gate) { return gate && *gate == 0; }

__global__ void k_scan_partial(const int32_t* __restrict__ in, int32_t n,
                               int32_t* __restrict__ partial, const int32_t* gate) {
  if (closed(gate)) return;
  const int64_t base = (int64_t)blockIdx.x * kScanTile + threadIdx.x * kScanItems;
  int32_t s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  int32_t tot;
  block_excl_scan(s, &tot);
  if (threadIdx.x == 0) partial[blockIdx.x] = tot;
}

__global__ void k_set1(int32_t* out, int32_t v, const int32_t* gate) {
  if (closed(gate)) return;
  *out = v;
}

__global__ void k_scan_top(int32_t* partial, int32_t nb, const int32_t* gate) {
  if (closed(gate)) return;
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
                             int32_t n, const int32_t* __restrict__ partial, int32_t init,
                             const int32_t* gate) {
  if (closed(gate)) return;
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
// Reference grid checks: grid_init's bin (cell_connection.cpp:44-53) and the
// range assert of connect_proc (:95-99). Returns the tissue-local bin or -1.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int32_t ref_bin(const TissueDev& T, double x, double y, double z,
                                           bool memb) {
  const int32_t aix = (int32_t)((0.5 * T.lx - pdiff(0.5 * T.lx, x, T.lx)) / kAreaGrid);
  const int32_t aiy = (int32_t)((0.5 * T.ly - pdiff(0.5 * T.ly, y, T.ly)) / kAreaGrid);
  const int32_t aiz = (int32_t)(fmax(z, 0.0) / kAreaGrid);  // min0, utils.h:55-57
  bool bad = aix >= T.anx || aiy >= T.any || aiz >= T.anz || aix < 0 || aiy < 0 || aiz < 0;
  if (!memb) {
    const int32_t cx = (int32_t)(x / kAreaGrid), cy = (int32_t)(y / kAreaGrid),
                  cz = (int32_t)(z / kAreaGrid);
    bad |= cx >= T.anx || cy >= T.any || cz >= T.anz || cx < 0 || cy < 0 || cz < 0;
  }
  return bad ? -1 : (aix * T.any + aiy) * T.anz + aiz;
}

// ---------------------------------------------------------------------------
// Rebuild work list. k_gate_compact lists the gated tissues of [t0, t1) with
// prefix sums of their particle and bin counts; every other rebuild kernel
// then strides over the gated particles (or bins) only, mapping a running
// index back to (tissue, local index) by binary search in the prefix sums.
// With nothing gated the list is empty and each kernel exits at once.
// ---------------------------------------------------------------------------
// For the whole batch the "some tissue" word is cleared once the list is
// built: the step kernel sets it again for the next step.
__device__ __forceinline__ void gate_compact(const DevState& S, int32_t t0, int32_t t1) {
  const bool whole = t0 == 0 && t1 == S.ntissues;
  if (S.gate[0] == 0) {
    if (threadIdx.x == 0) {
      S.rl_count[0] = 0;
      S.rl_ppre[0] = 0;
      S.rl_bpre[0] = 0;
    }
    return;
  }
  __syncthreads();  // every thread has read gate[0] before it is cleared
  if (whole && threadIdx.x == 0) S.gate[0] = 0;
  int32_t cc = 0, cp = 0, cb = 0;
  for (int32_t base = t0; base < t1; base += kScanThreads) {
    const int32_t t = base + threadIdx.x;
    const bool g = t < t1 && S.gate[1 + t] != 0;
    int32_t np = 0, nb = 0;
    if (g) {
      const TissueDev& T = S.tissues[t];
      np = T.n;
      nb = T.anx * T.any * T.anz;
    }
    int32_t tc, tp, tb;
    const int32_t oc = block_excl_scan(g ? 1 : 0, &tc);
    const int32_t op = block_excl_scan(np, &tp);
    const int32_t ob = block_excl_scan(nb, &tb);
    if (g) {
      S.rl_list[cc + oc] = t;
      S.rl_ppre[cc + oc] = cp + op;
      S.rl_bpre[cc + oc] = cb + ob;
    }
    cc += tc;
    cp += tp;
    cb += tb;
  }
  if (threadIdx.x == 0) {
    S.rl_count[0] = cc;
    S.rl_ppre[cc] = cp;
    S.rl_bpre[cc] = cb;
  }
}

// Once the work list is built nothing of the rebuild reads the flags: clear
// the listed tissues' flags and count the rebuilds. Run by one block of the
// candidate search. (gate_compact cleared the "some tissue" word.)
__device__ __forceinline__ void gate_clear(const DevState& S, int32_t cnt) {
  for (int32_t k = threadIdx.x; k < cnt; k += blockDim.x) S.gate[1 + S.rl_list[k]] = 0;
  if (threadIdx.x == 0 && cnt) atomicAdd(S.rebuilds, (unsigned long long)cnt);
}

__global__ void k_gate_compact(DevState S, int32_t t0, int32_t t1) {
  pdl_entry();
  count_launch(S.launches);
  gate_compact(S, t0, t1);
}

// index k of the last prefix entry <= g (pre[0] = 0, non-decreasing, n+1 entries)
__device__ __forceinline__ int32_t locate(const int32_t* pre, int32_t n, int32_t g) {
  int32_t lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const int32_t mid = (lo + hi) >> 1;
    if (pre[mid] <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Gated particle g -> global particle index (and its tissue).
__device__ __forceinline__ int32_t gated_particle(const DevState& S, int32_t cnt, int32_t g,
                                                  int32_t* tissue) {
  const int32_t k = locate(S.rl_ppre, cnt, g);
  const int32_t t = S.rl_list[k];
  *tissue = t;
  return S.tissues[t].pbase + (g - S.rl_ppre[k]);
}

#define GATED_PARTICLES(g, cnt)                                                        \
  const int32_t cnt = S.rl_count[0];                                                   \
  if (cnt == 0) return;                                                                \
  const int32_t ngated_ = S.rl_ppre[cnt];                                              \
  for (int32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngated_;                 \
       g += gridDim.x * blockDim.x)

// Binning on the reference's 2.0 grid (grid_init, cell_connection.cpp:38-62).
__global__ void k_bin(DevState S) {
  pdl_entry();
  count_launch(S.launches);
  GATED_PARTICLES(g, cnt) {
    int32_t t;
    const int32_t i = gated_particle(S, cnt, g, &t);
    const TissueDev& T = S.tissues[t];
    const double4 p = S.pos_cur[i];
    if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z)) {
      raise_error(S.status, E_NONFINITE, i, -1, p.x);
      S.bin[i] = -1;
      continue;
    }
    const int32_t lb = ref_bin(T, p.x, p.y, p.z, attr_state(S.attr[i]) == ST_MEMB);
    if (lb < 0) {
      raise_error(S.status, E_BIN_RANGE, i, -1, p.z);
      S.bin[i] = -1;
      continue;
    }
    const int32_t b = T.binbase + lb;
    const int32_t rk = atomicAdd(&S.counts[b], 1);
    if (rk + 1 >= kBinCap) raise_error(S.status, E_BIN_OVERFLOW, i, b, (double)(rk + 1));
    S.bin[i] = b;
    S.rank[i] = rk;
  }
}

// Per gated tissue, one block: exclusive scan of its bin counts into
// starts, offset by the tissue's first particle, so each tissue's sorted
// particles occupy its own slots [pbase, pbase + n). Each tissue's bins end
// with a sentinel entry that receives the end offset. 1024 threads scan
// 8192 bins per tile.
constexpr int kTissueScanThreads = 1024;
__global__ void __launch_bounds__(kTissueScanThreads) k_scan_tissue(DevState S) {
  pdl_entry();
  count_launch(S.launches);
  const int32_t cnt = S.rl_count[0];
  for (int32_t k = blockIdx.x; k < cnt; k += gridDim.x) {
    const TissueDev& T = S.tissues[S.rl_list[k]];
    const int32_t nb = T.anx * T.any * T.anz;
    const int32_t* in = S.counts + T.binbase;
    int32_t* out = S.starts + T.binbase;
    int32_t carry = T.pbase;
    constexpr int32_t kTile = kTissueScanThreads * kScanItems;
    for (int32_t base = 0; base < nb; base += kTile) {
      const int32_t b0 = base + threadIdx.x * kScanItems;
      int32_t v[kScanItems];
      int32_t sum = 0;
#pragma unroll
      for (int q = 0; q < kScanItems; ++q) {
        v[q] = b0 + q < nb ? in[b0 + q] : 0;
        sum += v[q];
      }
      int32_t tot;
      int32_t run = carry + block_excl_scan_n<kTissueScanThreads>(sum, &tot);
#pragma unroll
      for (int q = 0; q < kScanItems; ++q) {
        if (b0 + q < nb) out[b0 + q] = run;
        run += v[q];
      }
      carry += tot;
    }
    if (threadIdx.x == 0) out[nb] = carry;
    __syncthreads();
  }
}

__global__ void k_scatter(DevState S) {
  pdl_entry();
  count_launch(S.launches);
  GATED_PARTICLES(g, cnt) {
    int32_t t;
    const int32_t i = gated_particle(S, cnt, g, &t);
    const int32_t b = S.bin[i];
    if (b < 0) continue;
    const int32_t slot = S.starts[b] + S.rank[i];
    if (!EPI_CHECKED(slot >= S.tissues[t].pbase && slot < S.tissues[t].pbase + S.tissues[t].n,
                     S.status, i, slot))
      continue;
    S.skey[slot] = (uint32_t)i;
  }
}

// Sorts the particles of one bin (slots [s0, s1)) by index -- the
// deterministic order the candidate search emits them in -- then tags
// membrane particles and writes the sorted FP32 copy of their positions (x
// and y as grid_init bins them, in [0, L)). Bins hold a few to a few dozen
// particles: up to 24 are sorted in registers.
__device__ __forceinline__ void sort_bin(const DevState& S, const TissueDev& T, int32_t s0,
                                         int32_t s1) {
  constexpr int kLocal = 24;  // a bin holds about 8 particles at unit density
  if (s1 - s0 <= kLocal) {
    uint32_t key[kLocal];
    const int m = s1 - s0;
    for (int k = 0; k < m; ++k) {
      const uint32_t v = S.skey[s0 + k];
      int q = k - 1;
      while (q >= 0 && key[q] > v) {
        key[q + 1] = key[q];
        --q;
      }
      key[q + 1] = v;
    }
    for (int k = 0; k < m; ++k) S.skey[s0 + k] = key[k];
  } else {
    for (int32_t s = s0 + 1; s < s1; ++s) {
      const uint32_t v = S.skey[s];
      int32_t q = s - 1;
      while (q >= s0 && S.skey[q] > v) {
        S.skey[q + 1] = S.skey[q];
        --q;
      }
      S.skey[q + 1] = v;
    }
  }
  for (int32_t s = s0; s < s1; ++s) {
    const uint32_t gi = S.skey[s];
    if (!EPI_CHECKED(gi >= (uint32_t)T.pbase && gi < (uint32_t)(T.pbase + T.n), S.status,
                     (int32_t)gi, s))
      continue;
    const bool memb = attr_state(S.attr[gi]) == ST_MEMB;
    S.skey[s] = gi | (memb ? 0x80000000u : 0u);
    S.rank[gi] = s;  // the particle's slot from here on (the search skips it)
    // x and y as grid_init bins them (ref_bin): in [0, L); w: LJ_THRESH *
    // radius, negative for a membrane particle (the search's reach and its
    // membrane test)
    const double4 pg = S.pos_cur[gi];
    const double xc = 0.5 * T.lx - pdiff(0.5 * T.lx, pg.x, T.lx);
    const double yc = 0.5 * T.ly - pdiff(0.5 * T.ly, pg.y, T.ly);
    const float lw = (float)(T.P.lj_thresh * pg.w);
    S.spos[s] = make_float4((float)xc, (float)yc, (float)pg.z, memb ? -lw : lw);
  }
}

// Per-bin insertion sort by particle index (bins hold a few to a few dozen
// particles), then the sorted position copy the search streams through.
__global__ void k_binsort(DevState S) {
  pdl_entry();
  count_launch(S.launches);
  const int32_t cnt = S.rl_count[0];
  if (cnt == 0) return;
  const int32_t nbg = S.rl_bpre[cnt];
  for (int32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < nbg; g += gridDim.x * blockDim.x) {
    const int32_t k = locate(S.rl_bpre, cnt, g);
    const TissueDev& T = S.tissues[S.rl_list[k]];
    const int32_t b = T.binbase + (g - S.rl_bpre[k]);
    const int32_t s0 = S.starts[b], s1 = S.starts[b + 1];
    if (s1 <= s0) continue;
    S.counts[b] = 0;  // ready for the next binning
    sort_bin(S, T, s0, s1);
  }
}

// Bin ranges (inclusive) of the periodic window [x-R, x+R] along one axis:
// at most two ranges, because the window may wrap once. Bin k holds
// [k*AG, (k+1)*AG) of [0, L) (the last one is shortened; AG*AN > L).
// off[r]: the image of range r's particles nearest to x is their binned
// coordinate + off[r] (0, or +-L for the wrapped part of a split window).
__device__ __forceinline__ int window_ranges(double x, double R, double L, int32_t an,
                                             int32_t lo[2], int32_t hi[2], double off[2]) {
  off[0] = off[1] = 0.0;
  if (2.0 * R >= L) {
    lo[0] = 0;
    hi[0] = an - 1;
    return 1;
  }
  // floor(v / AG) through a multiply; the caller's window already carries a
  // margin far wider than the rounding difference.
  auto bin_of = [&](double v) {
    int32_t k = (int32_t)floor(v * (1.0 / kAreaGrid));
    return k < 0 ? 0 : (k > an - 1 ? an - 1 : k);
  };
  const double a = x - R, b = x + R;
  if (a < 0.0) {
    lo[0] = 0; hi[0] = bin_of(b);
    lo[1] = bin_of(a + L); hi[1] = an - 1;
    off[1] = -L;
    if (lo[1] <= hi[0]) { hi[0] = an - 1; return 1; }
    return 2;
  }
  if (b >= L) {
    lo[0] = bin_of(a); hi[0] = an - 1;
    lo[1] = 0; hi[1] = bin_of(b - L);
    off[1] = L;
    if (hi[1] >= lo[0]) { lo[0] = 0; return 1; }
    return 2;
  }
  lo[0] = bin_of(a);
  hi[0] = bin_of(b);
  return 1;
}

// Candidate search of a gated tissue: every partner within
// LJ_THRESH*(r_i+r_j) + skin (membrane pairs excluded: connect_proc only
// iterates non-membrane cells, cell_connection.cpp:93). The window covers
// every bin that can hold such a partner; the reference's fixed 5x5x5 window
// is a superset for every pair it can connect (reach <= 1.2 * 3.2 < 2 * 2.0).
// Candidates come out in column order (x ranges outer, y ranges inner), slot
// order within a column: deterministic after k_binsort.
// Slot positions are the grid's canonical [0, L) coordinates, so every
// particle of a window's x (or y) range has the same nearest image: the
// range's offset is folded into the particle's own coordinate (pxe, pye)
// and no per-slot wrap is needed. Boxes below 2 (R + AG) keep the per-slot
// minimum image (wrap_x, wrap_y): there an edge bin may hold the other image.
struct SearchWindow {
  int32_t xlo[2], xhi[2], ylo[2], yhi[2];
  int nxr, nyr;
  int32_t z0, z1;
  float pxe[2], pye[2], pz, flx, fly, fhx, fhy;
  float rw;        // LJ_THRESH * r_i + skin + margin: the reach less the partner's share
  float memb_lim;  // slots whose w lies below it are excluded (membrane pairs)
  int32_t s_self;  // the particle's own slot (-1: none)
  bool memb_i, wrap_x, wrap_y;

  __device__ __forceinline__ SearchWindow(const DevState& S, const TissueDev& T, int32_t i) {
    constexpr double kInvAG = 1.0 / kAreaGrid;
    memb_i = attr_state(S.attr[i]) == ST_MEMB;
    const double4 p = S.pos_cur[i];
    const double lt = T.P.lj_thresh;
    const double skin = S.skin;
    // Candidates are compared in float: the margin covers the rounding of
    // float coordinates up to the box size (and the window widens with it).
    const double margin = 1e-4 + 5e-7 * (T.lx > T.ly ? T.lx : T.ly) + 5e-7 * T.lz;
    const double R = lt * (p.w + (memb_i ? T.rmax_nm : T.rmax)) + skin + margin + 1e-6;
    double offx[2], offy[2];
    nxr = window_ranges(p.x, R, T.lx, T.anx, xlo, xhi, offx);
    nyr = window_ranges(p.y, R, T.ly, T.any, ylo, yhi, offy);
    wrap_x = !(T.lx > 2.0 * (R + kAreaGrid));
    wrap_y = !(T.ly > 2.0 * (R + kAreaGrid));
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      pxe[r] = (float)(wrap_x ? p.x : p.x - offx[r]);
      pye[r] = (float)(wrap_y ? p.y : p.y - offy[r]);
    }
    // z bins are floor(max(z, 0) / AG) (ref_bin); the margin in R covers the
    // multiply-for-divide rounding, so [z - R, z + R] needs no extra bins
    z0 = (int32_t)floor((p.z - R) * kInvAG);
    z1 = (int32_t)floor((p.z + R) * kInvAG);
    z0 = z0 < 0 ? 0 : (z0 > T.anz - 1 ? T.anz - 1 : z0);
    z1 = z1 < 0 ? 0 : (z1 > T.anz - 1 ? T.anz - 1 : z1);
    pz = (float)p.z;
    flx = (float)T.lx;
    fly = (float)T.ly;
    fhx = 0.5f * flx;
    fhy = 0.5f * fly;
    rw = (float)(lt * p.w + skin + margin);
    memb_lim = memb_i ? 0.f : -INFINITY;
    s_self = S.bin[i] < 0 ? -1 : S.rank[i];
  }
  // Is the particle in slot s (FP32 copy q) of a column of x range xr and y
  // range yr a candidate of i? (ex, ey: pxe[xr], pye[yr]) The reach
  // rw + |q.w| rounds differently from LJ_THRESH (r_i + r_j) + skin by a few
  // ulps, far inside the margin, so the candidates still hold every pair
  // that can be connected. kWrap = false: only for windows with neither
  // wrap_x nor wrap_y.
  template <bool kWrap>
  __device__ __forceinline__ bool hit_t(int32_t s, const float4& q, float ex, float ey) const {
    if (s == s_self || q.w < memb_lim) return false;
    float dx = ex - q.x, dy = ey - q.y;
    if (kWrap && wrap_x) dx = dx > fhx ? dx - flx : (dx <= -fhx ? dx + flx : dx);
    if (kWrap && wrap_y) dy = dy > fhy ? dy - fly : (dy <= -fhy ? dy + fly : dy);
    const float dz = pz - q.z;
    const float reach = rw + fabsf(q.w);
    return dx * dx + dy * dy + dz * dz <= reach * reach;
  }
  __device__ __forceinline__ bool hit(int32_t s, const float4& q, float ex, float ey) const {
    return hit_t<true>(s, q, ex, ey);
  }
};

__device__ __forceinline__ void finish_search(const DevState& S, int32_t i, int32_t count) {
  const int32_t cap = S.max_cand;
  if (count > cap) raise_error(S.status, E_LIST_OVERFLOW, i, -1, (double)count);
  cand_set(S, i, 0, (uint32_t)(count < cap ? count : cap));
  const double4 p = S.pos_cur[i];
  S.bpos[i] = make_float4((float)p.x, (float)p.y, (float)p.z, 0.f);
}

// Few gated particles (a tissue or two): G = 32 lanes (one warp) per
// particle, so the GPU has work for all its warps. The group's lanes fetch
// the slot ranges of G bin columns at a time; a scan within the group lays
// the ranges end to end, the group sweeps the concatenation G slots at a
// time, and ballots keep the slot order. (Groups of 4 to 16 lanes emit the
// same rows; they measured slower than one thread per particle for large
// rebuilds, whose window set-up they repeat on every lane.)
template <int G>
__device__ __forceinline__ void cand_search_groups(const DevState& S, int32_t cnt,
                                                   int32_t ngated) {
  static_assert(G == 4 || G == 8 || G == 16 || G == 32, "group of 4 to 32 lanes");
  const int lane = threadIdx.x & 31;
  const int gl = lane & (G - 1);          // lane within the group
  const int gbase = lane & ~(G - 1);      // the group's first lane
  const unsigned gmask = G == 32 ? 0xffffffffu : ((0xffffffffu >> (32 - G)) << gbase);
  const unsigned lt_mask = (1u << gl) - 1u;
  const int32_t groups = (gridDim.x * blockDim.x) / G;
  const int32_t cap = S.max_cand;
  for (int32_t g = (blockIdx.x * blockDim.x + threadIdx.x) / G; g < ngated; g += groups) {
    int32_t t;
    const int32_t i = gated_particle(S, cnt, g, &t);
    const TissueDev& T = S.tissues[t];
    const SearchWindow W(S, T, i);
    const int32_t nx0 = W.xhi[0] - W.xlo[0] + 1, ny0 = W.yhi[0] - W.ylo[0] + 1;
    const int32_t ncx = nx0 + (W.nxr > 1 ? W.xhi[1] - W.xlo[1] + 1 : 0);
    const int32_t ncy = ny0 + (W.nyr > 1 ? W.yhi[1] - W.ylo[1] + 1 : 0);
    const int32_t ncol = ncx * ncy;  // column c = cx * ncy + cy
    int32_t count = 0;
    for (int32_t c0 = 0; c0 < ncol; c0 += G) {
      const int32_t c = c0 + gl;
      int32_t lo = 0, len = 0;
      float cex = 0.f, cey = 0.f;
      if (c < ncol) {
        const int32_t cx = c / ncy, cy = c - cx * ncy;
        cex = cx < nx0 ? W.pxe[0] : W.pxe[1];
        cey = cy < ny0 ? W.pye[0] : W.pye[1];
        const int32_t bx = cx < nx0 ? W.xlo[0] + cx : W.xlo[1] + (cx - nx0);
        const int32_t by = cy < ny0 ? W.ylo[0] + cy : W.ylo[1] + (cy - ny0);
        const int32_t col = T.binbase + (bx * T.any + by) * T.anz;
        lo = S.starts[col + W.z0];
        len = S.starts[col + W.z1 + 1] - lo;
      }
      int32_t incl = len;
#pragma unroll
      for (int o = 1; o < G; o <<= 1) {
        const int32_t v = __shfl_up_sync(gmask, incl, o, G);
        if (gl >= o) incl += v;
      }
      const int32_t excl = incl - len;
      const int32_t total = __shfl_sync(gmask, incl, G - 1, G);
      for (int32_t base = 0; base < total; base += G) {
        const int32_t f = base + gl;
        // the last column whose range starts at or before f (k + step <= G - 1)
        int32_t k = 0;
#pragma unroll
        for (int32_t step = G / 2; step > 0; step >>= 1) {
          const int32_t e = __shfl_sync(gmask, excl, k + step, G);
          if (e <= f) k += step;
        }
        const int32_t s = __shfl_sync(gmask, lo, k, G) + (f - __shfl_sync(gmask, excl, k, G));
        const float ex = __shfl_sync(gmask, cex, k, G), ey = __shfl_sync(gmask, cey, k, G);
        bool hit = false;
        uint32_t key = 0;
        if (f < total) {
          key = S.skey[s];
          hit = W.hit(s, S.spos[s], ex, ey);
        }
        const unsigned m = (__ballot_sync(gmask, hit) & gmask) >> gbase;
        if (hit) {
          const int32_t kk = count + __popc(m & lt_mask);
          if (kk < cap) cand_set(S, i, kk + 1, (key & 0x7fffffffu) - (uint32_t)T.pbase);
        }
        count += __popc(m);
      }
    }
    if (gl == 0) finish_search(S, i, count);
  }
}

// A thread's candidate row written a whole 16-byte chunk at a time: entries
// are shifted into a register chunk from the top (the oldest reaches slot 0
// after a chunk's worth of entries) and the chunk is stored when full or at
// the end. Chunk 0 starts with a zero in the count slot; the caller stores
// the count afterwards.
template <bool k16>
struct RowWriter {
  static constexpr int kPer = k16 ? 8 : 4;  // entries per chunk
  uint32_t w0 = 0, w1 = 0, w2 = 0, w3 = 0;
  int32_t e = 1;  // next entry (entry 0 is the count)
  __device__ __forceinline__ void shift_in(uint32_t v) {
    if (k16) {
      w0 = __funnelshift_r(w0, w1, 16);
      w1 = __funnelshift_r(w1, w2, 16);
      w2 = __funnelshift_r(w2, w3, 16);
      w3 = __funnelshift_r(w3, v, 16);
    } else {
      w0 = w1;
      w1 = w2;
      w2 = w3;
      w3 = v;
    }
  }
  __device__ __forceinline__ void put(const DevState& S, int64_t i, uint32_t v) {
    if (!EPI_CHECKED(!k16 || v < 65536u, S.status, (int32_t)i, e)) return;
    shift_in(v);
    ++e;
    if ((e & (kPer - 1)) == 0)
      S.cand[(int64_t)(e / kPer - 1) * S.n_total + i] = make_uint4(w0, w1, w2, w3);
  }
  __device__ __forceinline__ void close(const DevState& S, int64_t i) {
    const int n = e & (kPer - 1);
    if (n == 0) return;
    for (int k = n; k < kPer; ++k) shift_in(0u);
    S.cand[(int64_t)(e / kPer) * S.n_total + i] = make_uint4(w0, w1, w2, w3);
  }
};

// One particle's candidate search by one thread. The window's columns
// (x ranges outer, y ranges inner) are walked as one flat sequence of
// slots, two per iteration: a lane moves on to its next column whenever it
// has used up the current one, so the lanes of a warp stay in step however
// their columns' slot counts differ. Each column's slot range is fetched one
// column ahead, so opening a column waits on no load. kWrap: the box is too
// small for the folded images (per-slot minimum image).
template <bool k16, bool kWrap>
__device__ __forceinline__ void search_particle(const DevState& S, const TissueDev& T,
                                                const SearchWindow& W, int32_t i) {
  const int32_t cap = S.max_cand;
  const int32_t nx0 = W.xhi[0] - W.xlo[0] + 1, ny0 = W.yhi[0] - W.ylo[0] + 1;
  const int32_t ncx = nx0 + (W.nxr > 1 ? W.xhi[1] - W.xlo[1] + 1 : 0);
  const int32_t ncy = ny0 + (W.nyr > 1 ? W.yhi[1] - W.ylo[1] + 1 : 0);
  const int32_t any = T.any, anz = T.anz, binbase = T.binbase;
  const uint32_t pbase = (uint32_t)T.pbase;
  RowWriter<k16> row;
  int32_t count = 0;
  // the column after the current one: its slot range and folded coordinates
  int32_t cx = 0, cy = 0;  // the column to fetch next
  int32_t ns = 0, nhi = 0;
  float nex = 0.f, ney = 0.f;
  bool nvalid = false;
  auto fetch = [&]() {
    nvalid = cx < ncx;
    if (!nvalid) return;
    const int32_t bx = cx < nx0 ? W.xlo[0] + cx : W.xlo[1] + (cx - nx0);
    const int32_t by = cy < ny0 ? W.ylo[0] + cy : W.ylo[1] + (cy - ny0);
    nex = cx < nx0 ? W.pxe[0] : W.pxe[1];
    ney = cy < ny0 ? W.pye[0] : W.pye[1];
    const int32_t col = binbase + (bx * any + by) * anz;
    ns = S.starts[col + W.z0];
    nhi = S.starts[col + W.z1 + 1];
    if (++cy == ncy) {
      cy = 0;
      ++cx;
    }
  };
  fetch();
  int32_t s = 0, s_hi = 0;
  float ex = 0.f, ey = 0.f;
  for (;;) {
    bool live = true;
    while (s >= s_hi) {  // open the next column
      if (!nvalid) {
        live = false;
        break;
      }
      s = ns;
      s_hi = nhi;
      ex = nex;
      ey = ney;
      fetch();
    }
    if (!live) break;
    const bool two = s + 1 < s_hi;
    const uint32_t k0 = S.skey[s];
    const float4 q0 = S.spos[s];
    const uint32_t k1 = two ? S.skey[s + 1] : 0u;
    const float4 q1 = two ? S.spos[s + 1] : make_float4(0.f, 0.f, 0.f, 0.f);
    const bool h0 = W.template hit_t<kWrap>(s, q0, ex, ey);
    const bool h1 = two && W.template hit_t<kWrap>(s + 1, q1, ex, ey);
    if (h0) {
      if (count < cap) row.put(S, i, (k0 & 0x7fffffffu) - pbase);
      ++count;
    }
    if (h1) {
      if (count < cap) row.put(S, i, (k1 & 0x7fffffffu) - pbase);
      ++count;
    }
    s += 2;
  }
  row.close(S, i);
  finish_search(S, i, count);
}

// Many gated particles: one thread per particle (about a hundred slots each:
// bins of 2.0 hold about six particles); a warp keeps 32 particles in flight
// and writes the column-major candidate rows coalesced.
template <bool k16>
__device__ __forceinline__ void cand_search_threads(const DevState& S, int32_t cnt,
                                                    int32_t ngated) {
  for (int32_t g = blockIdx.x * blockDim.x + threadIdx.x; g < ngated;
       g += gridDim.x * blockDim.x) {
    int32_t t;
    const int32_t i = gated_particle(S, cnt, g, &t);
    const TissueDev& T = S.tissues[t];
    const SearchWindow W(S, T, i);
    if (W.wrap_x || W.wrap_y) search_particle<k16, true>(S, T, W, i);
    else search_particle<k16, false>(S, T, W, i);
  }
}

// Below `thread_from` gated particles the warp-per-particle search (which
// keeps the GPU busy with few particles) runs, from there on one thread per
// particle. Both emit every row in the same order.
template <bool k16>
__global__ void __launch_bounds__(256, 4) k_cand_search(DevState S, int32_t thread_from) {
  pdl_entry();
  count_launch(S.launches);
  const int32_t cnt = S.rl_count[0];
  if (blockIdx.x == 0) gate_clear(S, cnt);
  if (cnt == 0) return;
  const int32_t ngated = S.rl_ppre[cnt];
  if (ngated < thread_from) cand_search_groups<32>(S, cnt, ngated);
  else cand_search_threads<k16>(S, cnt, ngated);
}

// Condition of the rebuild node in the captured step graph: builds the work
// list of [t0, t1) (as k_gate_compact) and runs the rebuild kernels only
// when it is not empty.
__global__ void k_rebuild_condition(DevState S, int32_t t0, int32_t t1,
                                    cudaGraphConditionalHandle h) {
  pdl_entry();
  count_launch(S.launches);
  gate_compact(S, t0, t1);
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional(h, S.rl_count[0] > 0 ? 1u : 0u);
}

__global__ void k_gate_set_all(DevState S, int32_t ntissues) {
  GRID_STRIDE(t, 0, ntissues) S.gate[1 + t] = 1;
  if (blockIdx.x == 0 && threadIdx.x == 0) S.gate[0] = 1;
}

// ---------------------------------------------------------------------------
// find_dermis (cell_connection.cpp:158-172) for the FIX / MUSUME cells in
// prep[f0, f1), from the current positions: the nearest connected membrane
// particle, strict <, starting from LX*LX.
// ---------------------------------------------------------------------------
__global__ void k_dermis(DevState S, int32_t f0, int32_t f1) {
  pdl_entry();
  count_launch(S.launches);
  GRID_STRIDE(e, f0, f1) {
    const int32_t i = S.prep[e];
    const TissueDev& T = S.tissues[attr_tissue(S.attr[i])];
    const double4 p = S.pos_cur[i];
    const int32_t nc = cand_count(S, i);
    const double lt = T.P.lj_thresh;
    int32_t best = -1;
    double bestd = T.lx * T.lx;
    for (int32_t k = 0; k < nc; ++k) {
      const int32_t q = T.pbase + (int32_t)cand_entry(S, i, k + 1);
      if (attr_state(S.attr[q]) != ST_MEMB) continue;
      const double4 pq = S.pos_cur[q];
      const double d2 =
          dist_sq_exact(pdiff(p.x, pq.x, T.lx), pdiff(p.y, pq.y, T.ly), p.z - pq.z);
      if (!connected_pred(d2, lt, p.w, pq.w)) continue;
      // on exact ties the lowest index wins (the reference: first in list order)
      if (d2 < bestd || (d2 == bestd && q < best)) {
        bestd = d2;
        best = q;
      }
    }
    S.dermis[i] = best;
  }
}

// ---------------------------------------------------------------------------
// Step: cell_interaction (cell_interaction.cpp:648-685) gathered per
// particle, pos_copy (cellmanager.cpp:19-26), the single periodic wrap of
// cell_pos_periodic_fix (:395-414), and the range checks the next
// connect_cell would make. R is the arithmetic type of the force laws
// (double: FP64 path; float: mixed path). Sums and positions stay double.
// ---------------------------------------------------------------------------

// rintf(v) for |v| <= 2^22 on the FMA pipe: adding and subtracting
// 1.5 * 2^23 rounds v to the nearest integer (ties to even) exactly.
__device__ __forceinline__ float rint_fma(float v) {
  return __fsub_rn(__fadd_rn(v, 12582912.f), 12582912.f);
}

// Offsets of lattice neighbours from membrane particle i (minimum image): from
// the FP64 positions in the FP64 path, from the FP32 copies in the mixed path.
template <typename R>
struct SiteOffsets;
template <>
struct SiteOffsets<double> {
  const DevState& S;
  const double4 p;
  const TissueDev& T;
  __device__ __forceinline__ SiteOffsets(const DevState& S_, int32_t, const double4& p_,
                                         const TissueDev& T_)
      : S(S_), p(p_), T(T_) {}
  __device__ __forceinline__ Vec3<double> operator()(int32_t q) const {
    return offset_of<double>(S.pos_cur[q], p, T);
  }
};
template <>
struct SiteOffsets<float> {
  const DevState& S;
  const float4 pf;
  const TissueDev& T;
  __device__ __forceinline__ SiteOffsets(const DevState& S_, int32_t i, const double4&,
                                         const TissueDev& T_)
      : S(S_), pf(S_.posf_cur[i]), T(T_) {}
  __device__ __forceinline__ Vec3<float> operator()(int32_t q) const {
    const float4 o = S.posf_cur[q];
    // minimum image as d - L rint(d / L): lattice neighbours lie far
    // closer than L/2, where it equals the compare-and-shift form
    const float dx0 = o.x - pf.x, dy0 = o.y - pf.y;
    const float dx = fmaf(-T.lxf, rint_fma(dx0 * T.ilxf), dx0);
    const float dy = fmaf(-T.lyf, rint_fma(dy0 * T.ilyf), dy0);
    return Vec3<float>{dx, dy, o.z - pf.z};
  }
};

template <typename R>
__device__ __forceinline__ Vec3<R> v3_cross(const Vec3<R>& a, const Vec3<R>& b) {
  return Vec3<R>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <typename R>
__device__ __forceinline__ Vec3<R> v3_sub(const Vec3<R>& a, const Vec3<R>& b) {
  return Vec3<R>{a.x - b.x, a.y - b.y, a.z - b.z};
}
template <typename R>
__device__ __forceinline__ Vec3<R> v3_axpy(R s, const Vec3<R>& a, const Vec3<R>& b) {
  return Vec3<R>{s * a.x + b.x, s * a.y + b.y, s * a.z + b.z};
}
template <typename R>
__device__ __forceinline__ R v3_dot(const Vec3<R>& a, const Vec3<R>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename R>
__device__ __forceinline__ Vec3<R> v3_unit(const Vec3<R>& a) {
  const R inv = frsqrt(v3_dot(a, a));
  return Vec3<R>{a.x * inv, a.y * inv, a.z * inv};
}

// Triangular-membrane bending of particle j (tri_memb_bend, tri_bend_1 and
// tri_bend_2, cell_interaction.cpp:451-508) from the offsets of its six
// lattice neighbours n[i] = memb[i] (indices nb[i]) and of the six
// second-ring sites c[i] = memb[(i+1)%6]->memb[i] (indices ring[i]); the
// particle itself is the origin. Returns
// the sum dr before the DT * KBEND factor. The reference divides each term
// by the norm of a normal it has already normalised in place
// (vec3::normalize, vec3.h:40-44), i.e. by 1 up to rounding; that division
// is left out.
template <typename R, typename Off>
__device__ __forceinline__ Vec3<R> tri_bending(const Off& off, const int32_t (&nb)[6],
                                               const int32_t (&ring)[6]) {
  Vec3<R> n[6], c[6];
#pragma unroll
  for (int i = 0; i < 6; ++i) n[i] = off(nb[i]);
#pragma unroll
  for (int i = 0; i < 6; ++i) c[i] = off(ring[i]);
  Vec3<R> dr{R(0), R(0), R(0)};
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    // tri_bend_1(r1 = self, a1 = n[i], b1 = n[i+1], c1 = c[i])
    const Vec3<R>& a = n[i];
    const Vec3<R>& b = n[(i + 1) % 6];
    const Vec3<R> rb{-b.x, -b.y, -b.z};
    const Vec3<R> ab = v3_sub(a, b);
    const Vec3<R> n1 = v3_unit(v3_cross(rb, ab));
    const Vec3<R> n2 = v3_unit(v3_cross(ab, v3_sub(c[i], b)));
    const R d = v3_dot(n1, n2);
    const Vec3<R> t = v3_cross(ab, v3_axpy(-d, n1, n2));  // ab x tri_rho(n1, n2)
    dr = v3_axpy(bend_factor(d), t, dr);
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) {
    // tri_bend_2(r1 = self, a1 = n[i], b1 = n[i+1], c1 = n[i+2])
    const Vec3<R>& a = n[i];
    const Vec3<R>& b = n[(i + 1) % 6];
    const Vec3<R>& cc = n[(i + 2) % 6];
    const Vec3<R> rc{-cc.x, -cc.y, -cc.z};
    const Vec3<R> rb{-b.x, -b.y, -b.z};
    const Vec3<R> bc = v3_sub(b, cc);
    const Vec3<R> ab = v3_sub(a, b);
    const Vec3<R> n1 = v3_unit(v3_cross(rc, bc));
    const Vec3<R> n2 = v3_unit(v3_cross(rb, ab));
    const R d = v3_dot(n1, n2);
    const Vec3<R> t1 = v3_cross(bc, v3_axpy(-d, n1, n2));  // bc x tri_rho(n1, n2)
    const Vec3<R> t2 = v3_cross(ab, v3_axpy(-d, n2, n1));  // ab x tri_rho(n2, n1)
    const R g = bend_factor(d);
    dr = v3_axpy(g, Vec3<R>{t1.x + t2.x, t1.y + t2.y, t1.z + t2.z}, dr);
  }
  return dr;
}

// Membrane particles: bending (square: _memb_bend_calc1..3, :296-449, the
// unit vectors of calc1 recomputed from the eleven lattice positions the
// stencil reaches instead of being stored; triangular: tri_memb_bend,
// :451-508), the lattice springs of _MEMB_interaction (:529-547, each
// applied once by the higher index) and the wall (:287-294), summed for
// membrane particle i.
template <typename R>
__device__ __forceinline__ double3 memb_force(const DevState& S, int32_t i) {
  {
    const TissueDev& T = S.tissues[attr_tissue(S.attr[i])];
    const Laws<R>& L = T.laws<R>();
    const double dt = T.P.dt;
    const int32_t pb = T.pbase, NMX = T.nmx, NMY = T.nmy;
    const int32_t j = i - pb, jj = j % NMX, kk = j / NMX;
    // lattice site at column jj+dj, row kk+dk with periodic wrap; the same
    // wiring as _memb_init (cellmanager.cpp:114-158)
    auto site = [&](int dj, int dk) {
      int32_t c = jj + dj, w = kk + dk;
      c += c < 0 ? NMX : 0;
      c -= c >= NMX ? NMX : 0;
      w += w < 0 ? NMY : 0;
      w -= w >= NMY ? NMY : 0;
      const int32_t q = pb + w * NMX + c;
      return EPI_CHECKED(q >= pb && q < pb + T.nmemb, S.status, i, q) ? q : i;
    };
    const double4 p = S.pos_cur[i];
    const SiteOffsets<R> off(S, i, p, T);
    double ax = 0.0, ay = 0.0, az = 0.0;
    // lattice links in connected_cell's order (square: l, r, b, u)
    int32_t nb[6];
    const bool tri = T.lattice == kLatticeTriangular;
    if (tri) {
      const TriSite s0{jj, kk};
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const TriSite a = tri_step(s0, k, NMX, NMY);
        nb[k] = pb + a.row * NMX + a.col;
      }
    } else {
      nb[0] = site(-1, 0);
      nb[1] = site(1, 0);
      nb[2] = site(0, -1);
      nb[3] = site(0, 1);
      nb[4] = nb[5] = nb[0];
    }
    if (tri) {
      int32_t ring[6];
      const TriSite s0{jj, kk};
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const TriSite a = tri_step(tri_step(s0, (k + 1) % 6, NMX, NMY), k, NMX, NMY);
        ring[k] = pb + a.row * NMX + a.col;
      }
      const Vec3<R> b = tri_bending<R>(off, nb, ring);
      const R s = R(dt * T.P.kbend);
      ax += double(s * b.x);
      ay += double(s * b.y);
      az += double(s * b.z);
    } else {
      const Vec3<R> o_r = off(site(1, 0));
      const Vec3<R> o_rr = off(site(2, 0));
      const Vec3<R> o_l = off(site(-1, 0));
      const Vec3<R> o_ll = off(site(-2, 0));
      const Vec3<R> o_u = off(site(0, 1));
      const Vec3<R> o_uu = off(site(0, 2));
      const Vec3<R> o_b = off(site(0, -1));
      const Vec3<R> o_bb = off(site(0, -2));
      const Vec3<R> o_bbr = off(site(1, -2));
      const Vec3<R> o_bbrr = off(site(2, -2));
      const Vec3<R> o0{R(0), R(0), R(0)};
      const Unit<R> nv = unit_ab(o0, o_r), nvr = unit_ab(o_r, o_rr);
      const Unit<R> nvl = unit_ab(o_l, o0), nvll = unit_ab(o_ll, o_l);
      const Unit<R> nvbb = unit_ab(o_bb, o_bbr), nvbbr = unit_ab(o_bbr, o_bbrr);
      const Unit<R> mv = unit_ab(o0, o_u), mvu = unit_ab(o_u, o_uu);
      const Unit<R> mvb = unit_ab(o_b, o0), mvbb = unit_ab(o_bb, o_b);
      const R ipn = dotu(nv, nvr), ipnl = dotu(nvl, nv), ipnll = dotu(nvll, nvl);
      const R ipm = dotu(mv, mvu), ipmb = dotu(mvb, mv);
      const R ipmbb = dotu(nvbb, nvbbr);  // the reference reads memb_bb's ipn (:380)
      const R fn = bend_factor(ipn), fnl = bend_factor(ipnl), fnll = bend_factor(ipnll);
      const R fm = bend_factor(ipm), fmb = bend_factor(ipmb), fmbb = bend_factor(ipmbb);
      const R s = R(dt * T.P.kbend);
      const R idn = fdiv(R(1), nv.d), idnl = fdiv(R(1), nvl.d);
      const R idm = fdiv(R(1), mv.d), idmb = fdiv(R(1), mvb.d);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const R n0 = cmp(nv, k), nr = cmp(nvr, k), nl = cmp(nvl, k), nll = cmp(nvll, k);
        const R m0 = cmp(mv, k), mu = cmp(mvu, k), mb = cmp(mvb, k), mbb = cmp(mvbb, k);
        const R f = -fn * (nr - ipn * n0) * idn +
                    fnl * ((n0 - ipnl * nl) * idnl - (nl - ipnl * n0) * idn) +
                    fnll * (nll - ipnll * nl) * idnl - fm * (mu - ipm * m0) * idm +
                    fmb * ((m0 - ipmb * mb) * idmb - (mb - ipmb * m0) * idm) +
                    fmbb * (mbb - ipmbb * mb) * idmb;
        const double d = double(s * f);
        if (k == 0) ax += d;
        else if (k == 1) ay += d;
        else az += d;
      }
    }
    for (int k = 0; k < T.nadj; ++k) {
      const int32_t q = nb[k];
      const bool hi = i > q;
      R dx, dy, dz, rs, d2;
      if constexpr (sizeof(R) == 4) {
        // mixed path: the FP32 copies, as for the bending stencil; the
        // minimum-image FP32 difference is antisymmetric, so both ends of a
        // link see opposite forces
        const Vec3<float> o = off(q);
        dx = -o.x;
        dy = -o.y;
        dz = -o.z;
        rs = off.pf.w + S.posf_cur[q].w;
        d2 = dx * dx + dy * dy + dz * dz;
      } else {
        const double4 pq = S.pos_cur[q];
        pair_sep(p, pq, hi, T, dx, dy, dz);
        rs = p.w + pq.w;
        d2 = dist_sq_exact(dx, dy, dz);
      }
      bool bad;
      const R c = L.memb_memb(d2, rs, &bad);
      if (bad) raise_error(S.status, E_MEMB_COEF_RANGE, hi ? i : q, hi ? q : i, double(c));
      const R sdt = R(dt) * c;
      ax += double(sdt * dx);
      ay += double(sdt * dy);
      az += double(sdt * dz);
    }
    if (p.z < p.w) {
      const R z = R(p.z), rad = R(p.w);
      const R distlj = R(2) * z;
      const R lj6 = pow6(rad) / pow6(z);
      const R ljm = L.eps4 * lj6 * (lj6 - R(1)) / (distlj * distlj);
      az += double(R(dt) * ljm * R(2) * z);
    }
    return make_double3(ax, ay, az);
  }
}

// The membrane sum of memb_force for the prep list's membrane particles
// [m0, m1), into S.fmemb for k_step. Computing it inside k_step instead
// spills the step kernel's registers and costs more than this launch. The
// mixed path is held to 64 registers (four blocks per SM; a few bytes spill)
// and runs about a quarter faster than at its natural 80; the FP64 path to
// 128 (two blocks per SM, no spill; 40 % faster than at its natural 138).
template <typename R>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? 4 : 2) k_memb_force(DevState S, int32_t m0, int32_t m1) {
  pdl_entry();
  count_launch(S.launches);
  GRID_STRIDE(e, m0, m1) {
    const int32_t i = S.prep[e];
    const double3 f = memb_force<R>(S, i);
    S.fmemb[i] = make_double4(f.x, f.y, f.z, 0.0);
  }
}

// The step proper. Per particle: connect_proc's exact predicate
// (cell_connection.cpp:115-119) on every candidate, the law(s) the reference
// applies to each connected pair, the particle's own terms, then pos_copy and
// the single wrap of cell_pos_periodic_fix.
//
// kSimple: every cell of the batch is ALIVE, DEAD or AIR (or a membrane
// particle) and none is paired; then each connected pair receives exactly
// one application of CI_al_air_de_to_al_air_de_fix_mu (:141-152): from the
// higher index when both cells are ALIVE/DEAD/AIR (:566-570), from the
// cell's side when the partner is a membrane particle (:573-575). kOld: some
// cell is older than THRESH_SP, so the adhesion constant depends on both
// cells' ages.
template <typename R, bool kSimple, bool kOld>
struct Particle {
  // The mixed path gathers candidates' FP32 copies and forms separations in
  // FP32; the FP64 path gathers the FP64 positions.
  static constexpr bool kFloatPos = sizeof(R) == 4;
  using Pos = typename std::conditional<kFloatPos, float4, double4>::type;
  const DevState& S;
  const int32_t i;
  const uint32_t a;
  const uint32_t t;
  const uint32_t st;
  const TissueDev& T;
  const Laws<R>& L;
  const double4 p;
  const double lt2;  // LJ_THRESH * LJ_THRESH, folded as the reference does
  const R dt;
  int32_t pair_i = -1, dermis_i = -1;
  double ax = 0.0, ay = 0.0, az = 0.0;
  // the first too-strong interaction of this particle (|coef| > 1000): kept
  // in registers and reported by finish(), so the candidate loop stores
  // nothing and the tissue's constants stay in registers across it
  int32_t bad_a = -1, bad_b = -1;
  double bad_v = 0.0;
  __device__ __forceinline__ void note_bad(R c, int32_t x, int32_t y) {
    if (fabs(c) > R(1000) && bad_a < 0) {
      bad_a = x;
      bad_b = y;
      bad_v = double(c);
    }
  }
  // the particle's FP32 copy (mixed path only)
  float4 pf = make_float4(0.f, 0.f, 0.f, 0.f);

  // a_: the particle's attribute word, p_: its current position
  __device__ __forceinline__ Particle(const DevState& S_, int32_t i_, uint32_t a_,
                                     const double4& p_)
      : S(S_), i(i_), a(a_), t(attr_tissue(a)), st(attr_state(a)),
        T(S_.tissues[t]), L(T.laws<R>()), p(p_),
        lt2(T.P.lj_thresh * T.P.lj_thresh), dt(R(T.P.dt)) {
    // the FP32 copy of the particle itself, as every writer of posf forms it
    if (kFloatPos) pf = make_float4((float)p.x, (float)p.y, (float)p.z, (float)p.w);
    if (!kSimple && st != ST_MEMB) {
      pair_i = __ldg(&S.pair[i]);
      if (st == ST_FIX || st == ST_MUSUME) dermis_i = __ldg(&S.dermis[i]);
      if (!EPI_CHECKED(pair_i < T.pbase + T.n && (pair_i >= T.pbase || pair_i == -1), S.status,
                       i, pair_i))
        pair_i = -1;
      if (!EPI_CHECKED(dermis_i < T.pbase + T.n && (dermis_i >= T.pbase || dermis_i == -1),
                       S.status, i, dermis_i))
        dermis_i = -1;
    }
  }

  // Connection test and separation of candidate q. FP64 path: the
  // reference's predicate (connect_proc :115-119) with its rounding. Mixed
  // path: the same test in FP32, decided by the FP64 predicate whenever the
  // FP32 d2 lies within T.ftol of the threshold, so the connection set is
  // the reference's in both.
  __device__ __forceinline__ bool connected(int32_t q, const double4& pq, R& dx, R& dy, R& dz,
                                            R& d2, R& rs) const {
    const double ddx = pdiff_h(p.x, pq.x, T.lx, T.hlx), ddy = pdiff_h(p.y, pq.y, T.ly, T.hly);
    const double ddz = p.z - pq.z;
    const double d2e = dist_sq_exact(ddx, ddy, ddz);
    const double rse = __dadd_rn(p.w, pq.w);
    if (!(d2e <= __dmul_rn(__dmul_rn(lt2, rse), rse))) return false;
    dx = R(ddx);
    dy = R(ddy);
    dz = R(ddz);
    d2 = R(d2e);
    rs = R(rse);
    return true;
  }
  __device__ __forceinline__ bool connected(int32_t q, const float4& qf, R& dx, R& dy, R& dz,
                                            R& d2, R& rs) const {
    // Minimum image as f - L rint(f / L) (positions lie in [0, L], so
    // |f| <= L): the compare-and-shift of p_diff_x for every |f| away from
    // L/2 by more than the rounding of f / L, i.e. for every pair within
    // reach of a connection (LJ_THRESH (r_i + r_j) + skin is far below
    // L/2); a pair near L/2 apart is rejected under either image. The
    // multiply, round and fma take four FMA-pipe instructions, no branch.
    float fx = pf.x - qf.x, fy = pf.y - qf.y;
    fx = fmaf(-T.lxf, rint_fma(fx * T.ilxf), fx);
    fy = fmaf(-T.lyf, rint_fma(fy * T.ilyf), fy);
    const float fz = pf.z - qf.z;
    const float f2 = fx * fx + fy * fy + fz * fz;
    const float frs = pf.w + qf.w;
    const float thr = T.lt2f * frs * frs;
    if (f2 > thr + T.ftol) return false;
    if (f2 >= thr - T.ftol) {
      // too close to the threshold for FP32: the reference's FP64 predicate
      const double4 pq = S.pos_cur[q];
      const double d2e = dist_sq_exact(pdiff_h(p.x, pq.x, T.lx, T.hlx),
                                       pdiff_h(p.y, pq.y, T.ly, T.hly), p.z - pq.z);
      const double rse = __dadd_rn(p.w, pq.w);
      if (!(d2e <= __dmul_rn(__dmul_rn(lt2, rse), rse))) return false;
    }
    dx = R(fx);
    dy = R(fy);
    dz = R(fz);
    d2 = R(f2);
    rs = R(frs);
    return true;
  }

  // Mixed path, simple states: the same test and law as connected() and
  // candidate(), with the law evaluated for every candidate and masked by
  // the test, so the lanes of a warp do not diverge on it; only the rare
  // FP64 decision near the threshold branches. A candidate that is not
  // connected adds +0 or -0 to the sums, which leaves them unchanged: they
  // start at +0 and, rounding to nearest, never become -0.
  __device__ __forceinline__ void candidate_simple(int32_t q, const float4& qf) {
    float fx = pf.x - qf.x, fy = pf.y - qf.y;
    fx = fmaf(-T.lxf, rint_fma(fx * T.ilxf), fx);
    fy = fmaf(-T.lyf, rint_fma(fy * T.ilyf), fy);
    const float fz = pf.z - qf.z;
    const float f2 = fx * fx + fy * fy + fz * fz;
    const float frs = pf.w + qf.w;
    const float thr = T.lt2f * frs * frs;
    bool conn = !(f2 > thr + T.ftol);
    if (conn && f2 >= thr - T.ftol) {
      const double4 pq = S.pos_cur[q];
      const double d2e = dist_sq_exact(pdiff_h(p.x, pq.x, T.lx, T.hlx),
                                       pdiff_h(p.y, pq.y, T.ly, T.hly), p.z - pq.z);
      const double rse = __dadd_rn(p.w, pq.w);
      conn = d2e <= __dmul_rn(__dmul_rn(lt2, rse), rse);
    }
    const bool both_old = kOld && attr_old(a) && attr_old(__ldg(&S.attr[q]));
    float coef = L.aad_fused(f2, frs, both_old);
    coef = conn ? coef : 0.f;
    note_bad(coef, i, q);
    const float sdt = dt * coef;
    ax += double(sdt * fx);
    ay += double(sdt * fy);
    az += double(sdt * fz);
  }

  __device__ __forceinline__ void candidate(int32_t q, const Pos& pq) {
    if constexpr (kFloatPos && kSimple) {
      candidate_simple(q, pq);
      return;
    }
    R dx, dy, dz, d2, rs;
    if (!connected(q, pq, dx, dy, dz, d2, rs)) return;
    R coef;
    if (kSimple) {
      const bool both_old = kOld && attr_old(a) && attr_old(__ldg(&S.attr[q]));
      if constexpr (sizeof(R) == 4) coef = L.aad_fused(d2, rs, both_old);
      else coef = L.aad(d2, rs, both_old);
      note_bad(coef, i, q);
    } else {
      const uint32_t aq = __ldg(&S.attr[q]);
      const uint32_t sq = attr_state(aq);
      const bool both_old = attr_old(a) && attr_old(aq);
      coef = R(0);
      // the law i applies while iterating q (if i is not a membrane particle)
      if (st != ST_MEMB) {
        const int law = law_of(st, i, pair_i, dermis_i, sq, q);
        if (law != L_NONE) {
          const R c = eval_law<R>(law, L, d2, rs, both_old, attr_sfm(a));
          note_bad(c, i, q);
          coef += c;
        }
      }
      // ... and the law q applies while iterating i (if q is not)
      if (sq != ST_MEMB) {
        int32_t pair_q = -1, dermis_q = -1;
        if (sq == ST_FIX || sq == ST_MUSUME) {
          pair_q = __ldg(&S.pair[q]);
          dermis_q = __ldg(&S.dermis[q]);
        }
        const int law = law_of(sq, q, pair_q, dermis_q, st, i);
        if (law != L_NONE) {
          const R c = eval_law<R>(law, L, d2, rs, both_old, attr_sfm(aq));
          note_bad(c, q, i);
          coef += c;
        }
      }
    }
    // DT * coef * separation (cell_interaction_apply, :56-58), summed in FP64
    const R sdt = dt * coef;
    ax += double(sdt * dx);
    ay += double(sdt * dy);
    az += double(sdt * dz);
  }

  // b: the position of the tissue's last candidate rebuild; f: the membrane
  // sums (membrane particles only)
  __device__ __forceinline__ void finish(const float4& b, const double4& f) {
    if (bad_a >= 0) raise_error(S.status, E_COEF_RANGE, bad_a, bad_b, bad_v);
    if (st == ST_MEMB) {
      ax += f.x;
      ay += f.y;
      az += f.z;
    } else if (!kSimple) {
      // wall_interaction (:287-294) for DER below its radius
      if (st == ST_DER && p.z < p.w) {
        const R z = R(p.z), rad = R(p.w);
        const R distlj = R(2) * z;
        const R lj6 = pow6(rad) / pow6(z);
        const R ljm = L.eps4 * lj6 * (lj6 - R(1)) / (distlj * distlj);
        az += double(dt * ljm * R(2) * z);
      }
      // _pair_interaction (:637-641), applied by the higher index of the pair
      if (pair_i >= 0) {
        const double4 pq = S.pos_cur[pair_i];
        const bool hi = i > pair_i;
        double dx, dy, dz;
        pair_sep(p, pq, hi, T, dx, dy, dz);
        const R d2 = R(dist_sq_exact(dx, dy, dz));
        const R c = L.pair(d2, R(hi ? S.spr[i] : S.spr[pair_i]));
        if (fabs(c) > R(1000)) raise_error(S.status, E_COEF_RANGE, i, pair_i, double(c));
        const R sdt = dt * c;
        ax += double(sdt * R(dx));
        ay += double(sdt * R(dy));
        az += double(sdt * R(dz));
      }
    }
    // pos_copy + the single wrap of cell_pos_periodic_fix
    const double lx = T.lx, ly = T.ly, hlx = T.hlx, hly = T.hly;
    double nx = p.x + ax, ny = p.y + ay;
    const double nz = p.z + az;
    if (nx > lx) nx -= lx;
    else if (nx < 0) nx += lx;
    if (ny > ly) ny -= ly;
    else if (ny < 0) ny += ly;
    if (!isfinite(nx) || !isfinite(ny) || !isfinite(nz)) {
      raise_error(S.status, E_NONFINITE, i, -1, nz);
    } else if (!range_ok(T, nx, ny, nz, st == ST_MEMB)) {
      raise_error(S.status, E_BIN_RANGE, i, -1, nz);
    }
    S.pos_nxt[i] = make_double4(nx, ny, nz, p.w);
    if (kFloatPos) S.posf_nxt[i] = make_float4((float)nx, (float)ny, (float)nz, (float)p.w);
    // Candidate validity: rebuild the tissue once a particle moved skin/2.
    double ex = nx - (double)b.x, ey = ny - (double)b.y;
    if (ex > hlx) ex -= lx;
    else if (ex < -hlx) ex += lx;
    if (ey > hly) ey -= ly;
    else if (ey < -hly) ey += ly;
    const double ez = nz - (double)b.z;
    const double lim = 0.5 * S.skin - 1e-3;  // margin covers the float rounding of bpos
    if (!(ex * ex + ey * ey + ez * ez <= lim * lim)) {
      S.gate[1 + t] = 1;
      S.gate[0] = 1;
    }
  }
};

template <typename Pos>
__device__ __forceinline__ const Pos* gather_source(const DevState& S);
template <>
__device__ __forceinline__ const double4* gather_source<double4>(const DevState& S) {
  return S.pos_cur;
}
template <>
__device__ __forceinline__ const float4* gather_source<float4>(const DevState& S) {
  return S.posf_cur;
}

// Entry e of a candidate row from its first chunks held in registers (e a
// constant once the caller's loop is unrolled). 16-bit entries: half e % 2
// of word (e % 8) / 2 of chunk e / 8; 32-bit: word e % 4 of chunk e / 4.
template <bool k16, int NC>
__device__ __forceinline__ uint32_t row_entry(const uint4 (&c)[NC], int e) {
  const uint4& ch = c[k16 ? e / 8 : e / 4];
  const int w = k16 ? (e % 8) / 2 : e % 4;
  const uint32_t word = w == 0 ? ch.x : (w == 1 ? ch.y : (w == 2 ? ch.z : ch.w));
  return k16 ? ((e & 1) ? word >> 16 : word & 0xffffu) : word;
}

// The candidates of particle i, from the first chunks of its row in c (kPre
// entries after the count) and the rest of the row from memory, passed to
// P.candidate with their positions. Positions are gathered kG at a time:
// all kG loads are issued before the first is used.
template <bool k16, int kPre, int kG, typename Part, int NC>
__device__ __forceinline__ void gather_candidates(const DevState& S, Part& P, const uint4 (&c)[NC],
                                                  int64_t i) {
  using Pos = typename Part::Pos;
  const int32_t pbase = P.T.pbase;
  const Pos* src = gather_source<Pos>(S) + pbase;
  const int32_t nc = (int32_t)row_entry<k16>(c, 0);
#pragma unroll
  for (int b = 1; b <= kPre; b += kG) {
    if (b > nc) break;
    int32_t q[kG];
    Pos pq[kG];
#pragma unroll
    for (int u = 0; u < kG; ++u) {
      q[u] = 0;
      if (b + u <= kPre) {
        q[u] = (int32_t)row_entry<k16>(c, b + u);
        if (b + u <= nc && EPI_CHECKED(q[u] < P.T.n, S.status, (int32_t)i, q[u]))
          pq[u] = src[q[u]];
      }
    }
#pragma unroll
    for (int u = 0; u < kG; ++u)
      if (b + u <= kPre && b + u <= nc && (q[u] < P.T.n || !kCheck))
        P.candidate(pbase + q[u], pq[u]);
  }
  for (int32_t e = kPre + 1; e <= nc; ++e) {
    const int32_t q = (int32_t)cand_entry(S, i, e);
    if (!EPI_CHECKED(q < P.T.n, S.status, (int32_t)i, q)) continue;
    P.candidate(pbase + q, src[q]);
  }
}

// One thread per particle. The first chunks of the particle's candidate row
// (15 candidates with 16-bit entries, 15 with 32-bit) are loaded up front,
// independent of each other and of the particle's own data, so the index
// stream costs one memory latency per particle rather than one per
// candidate. The neighbours' positions are then gathered kG at a time (all
// kG loads issued before the first is used). Rows longer than that (rare)
// finish with one load per entry. kMinBlocks bounds the registers so that
// that many 256-thread blocks stay resident per SM.
// One particle of the step.
// Streaming loads that do not allocate in L1 (the particle's own inputs,
// read once), leaving L1 to the neighbours' gathered positions.
__device__ __forceinline__ uint4 ld_na(const uint4* p) {
  uint4 v;
  asm("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
      : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ float4 ld_na(const float4* p) {
  float4 v;
  asm("ld.global.nc.L1::no_allocate.v4.f32 {%0,%1,%2,%3}, [%4];"
      : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "l"(p));
  return v;
}
__device__ __forceinline__ double4 ld_na(const double4* p) {
  double a, b, c, d;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];" : "=d"(a), "=d"(b) : "l"(p));
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0,%1}, [%2];"
      : "=d"(c), "=d"(d) : "l"(reinterpret_cast<const double2*>(p) + 1));
  return make_double4(a, b, c, d);
}
__device__ __forceinline__ uint32_t ld_na(const uint32_t* p) {
  uint32_t v;
  asm("ld.global.nc.L1::no_allocate.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}

template <typename R, bool kSimple, bool kOld, bool k16>
__device__ __forceinline__ void step_particle(const DevState& S, int64_t i) {
  const int64_t N = S.n_total;
  constexpr int kChunks = k16 ? 2 : 4;               // chunks loaded up front
  constexpr int kPre = kChunks * (k16 ? 8 : 4) - 1;  // candidates they hold
  constexpr int kG = sizeof(R) == 4 ? 4 : 2;         // gathers in flight
  uint4 c[kChunks];
#pragma unroll
  for (int k = 0; k < kChunks; ++k) c[k] = ld_na(S.cand + k * N + i);
  const uint32_t a = ld_na(S.attr + i);
  using Part = Particle<R, kSimple, kOld>;
  Part P(S, (int32_t)i, a, ld_na(S.pos_cur + i));
  const float4 bp = ld_na(S.bpos + i);
  const double4 fm = P.st == ST_MEMB ? S.fmemb[i] : make_double4(0.0, 0.0, 0.0, 0.0);
  gather_candidates<k16, kPre, kG>(S, P, c, i);
  P.finish(bp, fm);
}

// The same loop with the gathers copied into shared memory asynchronously
// (cp.async, cached in L1): a thread issues the copies of kS neighbours'
// positions at once -- all 15 candidates its first two chunks hold when
// kS = 15 -- holding no register for data in flight, waits once for its own
// copies, then evaluates the candidates from its own slots (thread t's slot
// k at slots[k * kStepThreads + t]: conflict-free, no barrier needed).
constexpr int kStepThreads = 256;
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
template <typename Pos>
__device__ __forceinline__ void cp_async_pos(Pos* dst, const Pos* src) {
#pragma unroll
  for (int h = 0; h < (int)(sizeof(Pos) / 16); ++h)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16;" ::"r"(smem_u32(
                     reinterpret_cast<char*>(dst) + 16 * h)),
                 "l"(reinterpret_cast<const char*>(src) + 16 * h)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.wait_all;" ::: "memory");
}

template <bool k16, int kPre, int kS, typename Part, int NC>
__device__ __forceinline__ void gather_candidates_async(const DevState& S, Part& P,
                                                        const uint4 (&c)[NC], int64_t i,
                                                        typename Part::Pos* slots) {
  using Pos = typename Part::Pos;
  const int32_t pbase = P.T.pbase;
  const Pos* src = gather_source<Pos>(S) + pbase;
  const int32_t nc = (int32_t)row_entry<k16>(c, 0);
#pragma unroll
  for (int b = 1; b <= kPre; b += kS) {
    if (b > nc) break;
#pragma unroll
    for (int u = 0; u < kS; ++u) {
      const int e = b + u;
      if (e <= kPre && e <= nc) {
        const int32_t q = (int32_t)row_entry<k16>(c, e);
        if (EPI_CHECKED(q < P.T.n, S.status, (int32_t)i, q))
          cp_async_pos(slots + u * kStepThreads, src + q);
      }
    }
    cp_async_wait_all();
#pragma unroll
    for (int u = 0; u < kS; ++u) {
      const int e = b + u;
      if (e <= kPre && e <= nc) {
        const int32_t q = (int32_t)row_entry<k16>(c, e);
        if (q < P.T.n || !kCheck) P.candidate(pbase + q, slots[u * kStepThreads]);
      }
    }
  }
  for (int32_t e = kPre + 1; e <= nc; ++e) {
    const int32_t q = (int32_t)cand_entry(S, i, e);
    if (!EPI_CHECKED(q < P.T.n, S.status, (int32_t)i, q)) continue;
    P.candidate(pbase + q, src[q]);
  }
}

template <typename R, bool kSimple, bool kOld, int kMinBlocks, bool k16, int kS>
__global__ void __launch_bounds__(kStepThreads, kMinBlocks) k_step_async(DevState S, Range r) {
  pdl_entry();
  count_launch(S.launches);
  using Part = Particle<R, kSimple, kOld>;
  using Pos = typename Part::Pos;
  extern __shared__ __align__(16) unsigned char gather_smem[];
  Pos* slots = reinterpret_cast<Pos*>(gather_smem) + threadIdx.x;
  const int64_t i = r.p0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.p1) return;
  const int64_t N = S.n_total;
  constexpr int kChunks = k16 ? 2 : 4;
  constexpr int kPre = kChunks * (k16 ? 8 : 4) - 1;
  uint4 c[kChunks];
#pragma unroll
  for (int k = 0; k < kChunks; ++k) c[k] = ld_na(S.cand + k * N + i);
  Part P(S, (int32_t)i, ld_na(S.attr + i), ld_na(S.pos_cur + i));
  const float4 bp = ld_na(S.bpos + i);
  const double4 fm = P.st == ST_MEMB ? S.fmemb[i] : make_double4(0.0, 0.0, 0.0, 0.0);
  gather_candidates_async<k16, kPre, kS>(S, P, c, i, slots);
  P.finish(bp, fm);
}

template <typename R, bool kSimple, bool kOld, int kMinBlocks, bool k16>
__global__ void __launch_bounds__(256, kMinBlocks) k_step(DevState S, Range r) {
  pdl_entry();
  count_launch(S.launches);
  const int64_t i = r.p0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= r.p1) return;
  step_particle<R, kSimple, kOld, k16>(S, i);
}


// connect_cell's lists (for export): the exact predicate over the candidates.
__global__ void k_exact_lists(DevState S, Range r) {
  GRID_STRIDE(i, r.p0, r.p1) {
    const uint32_t a = S.attr[i];
    const TissueDev& T = S.tissues[attr_tissue(a)];
    const double4 p = S.pos_cur[i];
    const int32_t nc = cand_count(S, i);
    const double lt = T.P.lj_thresh;
    int32_t count = 0;
    for (int32_t k = 0; k < nc; ++k) {
      const int32_t q = T.pbase + (int32_t)cand_entry(S, i, k + 1);
      const double4 pq = S.pos_cur[q];
      const double d2 =
          dist_sq_exact(pdiff(p.x, pq.x, T.lx), pdiff(p.y, pq.y, T.ly), p.z - pq.z);
      if (!connected_pred(d2, lt, p.w, pq.w)) continue;
      if (count < S.max_conn) S.nbr[(int64_t)count * S.n_total + i] = q;
      ++count;
    }
    if (count > S.max_conn) raise_error(S.status, E_LIST_OVERFLOW, (int32_t)i, -1, (double)count);
    S.nn[i] = count < S.max_conn ? count : S.max_conn;
  }
}

// ---------------------------------------------------------------------------
// Export helpers (not on the per-step path).
// ---------------------------------------------------------------------------
__global__ void k_rowlen(DevState S, int32_t* rowlen, int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t a = S.attr[i];
  rowlen[i] = S.nn[i] + (attr_state(a) == ST_MEMB ? S.tissues[attr_tissue(a)].nadj : 0);
}

__global__ void k_fill_csr(DevState S, const int32_t* rowoff, int32_t* idx, int32_t n) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t a = S.attr[i];
  const TissueDev& T = S.tissues[attr_tissue(a)];
  int32_t o = rowoff[i];
  const int32_t o0 = o;
  if (attr_state(a) == ST_MEMB)  // push order of _memb_init, cellmanager.cpp:70-166
    for (int k = 0; k < T.nadj; ++k) idx[o++] = lattice_link(T, i - T.pbase, k);
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
  const uint32_t st = attr_state(a);
  const int32_t d = (st == ST_FIX || st == ST_MUSUME) ? S.dermis[i] : -1;
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
  if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z))
    raise_error(S.status, E_NONFINITE, (int32_t)i, -1, p.z);
  S.pos_cur[i] = p;
  S.pos_nxt[i] = p;
  const float4 f = make_float4((float)p.x, (float)p.y, (float)p.z, (float)r);
  S.posf_cur[i] = f;
  S.posf_nxt[i] = f;
}

// Particles [p0, p1) of a host step: positions from the staged host arrays
// into both buffers and both FP32 copies (as k_pack), and the displacement
// test of the candidate rows (as k_gate_check).
__global__ void k_pack_gate(DevState S, const double* x, const double* y, const double* z,
                            int32_t p0, int32_t p1) {
  GRID_STRIDE(i, p0, p1) {
    const double r = S.pos_cur[i].w;
    const double4 p = make_double4(x[i], y[i], z[i], r);
    if (!isfinite(p.x) || !isfinite(p.y) || !isfinite(p.z))
      raise_error(S.status, E_NONFINITE, (int32_t)i, -1, p.z);
    S.pos_cur[i] = p;
    S.pos_nxt[i] = p;
    const float4 f = make_float4((float)p.x, (float)p.y, (float)p.z, (float)r);
    S.posf_cur[i] = f;
    S.posf_nxt[i] = f;
    const uint32_t t = attr_tissue(S.attr[i]);
    const TissueDev& T = S.tissues[t];
    const float4 b = S.bpos[i];
    double ex = p.x - (double)b.x, ey = p.y - (double)b.y;
    if (ex > T.hlx) ex -= T.lx;
    else if (ex < -T.hlx) ex += T.lx;
    if (ey > T.hly) ey -= T.ly;
    else if (ey < -T.hly) ey += T.ly;
    const double ez = p.z - (double)b.z;
    const double lim = 0.5 * S.skin - 1e-3;
    if (!(ex * ex + ey * ey + ez * ez <= lim * lim)) {
      S.gate[1 + t] = 1;
      S.gate[0] = 1;
    }
  }
}

__global__ void k_unpack_range(DevState S, double* x, double* y, double* z, int32_t p0,
                               int32_t p1) {
  GRID_STRIDE(i, p0, p1) {
    const double4 p = S.pos_cur[i];
    x[i] = p.x;
    y[i] = p.y;
    z[i] = p.z;
  }
}

__global__ void k_posf(DevState S) {
  GRID_STRIDE(i, 0, S.n_total) {
    const double4 p = S.pos_cur[i];
    S.posf_cur[i] = make_float4((float)p.x, (float)p.y, (float)p.z, (float)p.w);
  }
}

}  // namespace

void launch_posf(const DevState& S, const LaunchCfg& lc, cudaStream_t s) {
  if (S.n_total > 0) k_posf<<<stride_blocks(S.n_total, lc.block, lc), lc.block, 0, s>>>(S);
}

void launch_scan(const int32_t* in, int32_t* out, int32_t n, int32_t init,
                 const ScanScratch& sc, const int32_t* gate, const LaunchCfg&,
                 cudaStream_t s) {
  const int32_t nb = (n + kScanTile - 1) / kScanTile;
  if (nb == 0) {
    k_set1<<<1, 1, 0, s>>>(out, init, gate);
    return;
  }
  k_scan_partial<<<nb, kScanThreads, 0, s>>>(in, n, sc.partial, gate);
  k_scan_top<<<1, kScanThreads, 0, s>>>(sc.partial, nb, gate);
  k_scan_final<<<nb, kScanThreads, 0, s>>>(in, out, n, sc.partial, init, gate);
}

void launch_rebuild(const DevState& S, const Range& r, const ScanScratch&,
                    const LaunchCfg& lc, cudaStream_t s, Timer* tm, bool listed) {
  const int B = lc.block;
  const int grid = lc.num_sms * 8;
  if (!listed) {
    timer_begin(tm, KC_GATE, s);
    launch_pdl(k_gate_compact, 1, kScanThreads, s, S, r.t0, r.t1);
    timer_end(tm, KC_GATE, s);
  }
  timer_begin(tm, KC_REBUILD_BIN, s);
  launch_pdl(k_bin, grid, B, s, S);
  timer_end(tm, KC_REBUILD_BIN, s);
  timer_begin(tm, KC_REBUILD_SCAN, s);
  const int nt = r.t1 - r.t0;
  launch_pdl(k_scan_tissue, nt < lc.num_sms * 4 ? (nt > 0 ? nt : 1) : lc.num_sms * 4,
             kTissueScanThreads, s, S);
  timer_end(tm, KC_REBUILD_SCAN, s);
  timer_begin(tm, KC_REBUILD_SORT, s);
  launch_pdl(k_scatter, grid, B, s, S);
  launch_pdl(k_binsort, grid, B, s, S);
  timer_end(tm, KC_REBUILD_SORT, s);
  timer_begin(tm, KC_REBUILD_SEARCH, s);
  if (S.cand16) launch_pdl(k_cand_search<true>, grid, B, s, S, (int32_t)lc.search_switch);
  else launch_pdl(k_cand_search<false>, grid, B, s, S, (int32_t)lc.search_switch);
  timer_end(tm, KC_REBUILD_SEARCH, s);
}

void launch_memb_force(const DevState& S, int32_t m0, int32_t m1, int precision,
                       const LaunchCfg& lc, cudaStream_t s, Timer* tm) {
  if (m1 <= m0) return;
  timer_begin(tm, KC_PREPASS, s);
  const int gm = stride_blocks(m1 - m0, lc.block, lc);
  if (precision == 1)
    launch_pdl(k_memb_force<float>, gm, lc.block, s, S, m0, m1);
  else
    launch_pdl(k_memb_force<double>, gm, lc.block, s, S, m0, m1);
  timer_end(tm, KC_PREPASS, s);
}

void launch_dermis(const DevState& S, int32_t f0, int32_t f1, const LaunchCfg& lc,
                   cudaStream_t s, Timer* tm) {
  if (f1 <= f0) return;
  timer_begin(tm, KC_PREPASS, s);
  launch_pdl(k_dermis, stride_blocks(f1 - f0, lc.block, lc), lc.block, s, S, f0, f1);
  timer_end(tm, KC_PREPASS, s);
}

void launch_prepass(const DevState& S, int32_t m0, int32_t m1, int32_t f0, int32_t f1,
                    int precision, const LaunchCfg& lc, cudaStream_t s, Timer* tm) {
  launch_memb_force(S, m0, m1, precision, lc, s, tm);
  launch_dermis(S, f0, f1, lc, s, tm);
}

// The asynchronous-gather kernel with kS shared-memory slots per thread.
template <typename R, bool kSimple, bool kOld, bool k16, int kS, int kMinBlocks>
void launch_step_async(const DevState& S, const Range& r, cudaStream_t s) {
  using Pos = typename std::conditional<sizeof(R) == 4, float4, double4>::type;
  auto kern = k_step_async<R, kSimple, kOld, kMinBlocks, k16, kS>;
  constexpr int smem = kS * kStepThreads * (int)sizeof(Pos);
  static bool configured = false;
  if (!configured) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    configured = true;
  }
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)blocks_for(r.p1 - r.p0, kStepThreads));
  cfg.blockDim = dim3((unsigned)kStepThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kern, S, r);
}

// Tuning variants: 1 and 2, gathers copied asynchronously into shared
// memory, 8 (FP64: 4) and 15 (FP64: 8) slots per thread; 3 (default) and 4,
// gathers into registers four (FP64: two) at a time, at two register budgets
// (3 and 4 resident 256-thread blocks per SM; FP64: 3 and 2).
template <typename R, bool kSimple, bool kOld, bool k16>
void launch_step_w(const DevState& S, const Range& r, const LaunchCfg& lc, cudaStream_t s) {
  const int grid = blocks_for(r.p1 - r.p0, 256);
  constexpr bool kF = sizeof(R) == 4;
  switch (lc.variant) {
    case 1: launch_step_async<R, kSimple, kOld, k16, kF ? 8 : 4, kF ? 4 : 3>(S, r, s); break;
    case 2: launch_step_async<R, kSimple, kOld, k16, kF ? 15 : 8, 3>(S, r, s); break;
    case 4: launch_pdl(k_step<R, kSimple, kOld, kF ? 4 : 2, k16>, grid, 256, s, S, r); break;
    default: launch_pdl(k_step<R, kSimple, kOld, 3, k16>, grid, 256, s, S, r); break;
  }
}

template <typename R, bool kSimple, bool kOld>
void launch_step_v(const DevState& S, const Range& r, const LaunchCfg& lc, cudaStream_t s) {
  if (S.cand16) launch_step_w<R, kSimple, kOld, true>(S, r, lc, s);
  else launch_step_w<R, kSimple, kOld, false>(S, r, lc, s);
}

template <typename R>
void launch_step_r(const DevState& S, const Range& r, const LaunchCfg& lc, cudaStream_t s) {
  if (lc.simple && lc.any_old)
    launch_step_v<R, true, true>(S, r, lc, s);
  else if (lc.simple)
    launch_step_v<R, true, false>(S, r, lc, s);
  else
    launch_step_v<R, false, true>(S, r, lc, s);
}

void launch_step(const DevState& S, const Range& r, int precision, const LaunchCfg& lc,
                 cudaStream_t s, Timer* tm) {
  const int32_t np = r.p1 - r.p0;
  if (np <= 0) return;
  timer_begin(tm, KC_STEP, s);
  if (precision == 1)
    launch_step_r<float>(S, r, lc, s);
  else
    launch_step_r<double>(S, r, lc, s);
  timer_end(tm, KC_STEP, s);
}

void launch_exact_lists(const DevState& S, const Range& r, const LaunchCfg& lc,
                        cudaStream_t s) {
  const int32_t np = r.p1 - r.p0;
  if (np > 0) k_exact_lists<<<stride_blocks(np, lc.block, lc), lc.block, 0, s>>>(S, r);
}

// Loop counter of the step graph's WHILE node: one pass of the body (two
// steps) done; run another while pairs remain.
__global__ void k_loop_tick(int32_t* remaining, cudaGraphConditionalHandle h,
                            unsigned long long* launches) {
  pdl_entry();
  count_launch(launches);
  const int32_t left = *remaining - 1;
  *remaining = left;
  cudaGraphSetConditional(h, left > 0 ? 1u : 0u);
}

void launch_loop_tick(int32_t* remaining, cudaGraphConditionalHandle h,
                      unsigned long long* launches, cudaStream_t s) {
  launch_pdl(k_loop_tick, 1, 1, s, remaining, h, launches);
}

void launch_set_counter(int32_t* remaining, int32_t value, cudaStream_t s) {
  k_set1<<<1, 1, 0, s>>>(remaining, value, nullptr);
}

void launch_rebuild_condition(const DevState& S, const Range& r, cudaGraphConditionalHandle h,
                              cudaStream_t s) {
  launch_pdl(k_rebuild_condition, 1, kScanThreads, s, S, r.t0, r.t1, h);
}

void launch_set_gates(const DevState& S, int32_t ntissues, cudaStream_t s) {
  k_gate_set_all<<<(ntissues + 255) / 256 + 1, 256, 0, s>>>(S, ntissues);
}

void launch_rowlen(const DevState& S, int32_t* rowlen, int32_t n, cudaStream_t s) {
  if (n > 0) k_rowlen<<<blocks_for(n, 256), 256, 0, s>>>(S, rowlen, n);
}
void launch_fill_csr(const DevState& S, const int32_t* rowoff, int32_t* idx, int32_t n,
                     cudaStream_t s) {
  if (n > 0) k_fill_csr<<<blocks_for(n, 256), 256, 0, s>>>(S, rowoff, idx, n);
}
void launch_dermis_local(const DevState& S, int32_t* out, int32_t n, cudaStream_t s) {
  if (n > 0) k_dermis_local<<<blocks_for(n, 256), 256, 0, s>>>(S, out, n);
}
void launch_unpack_positions(const DevState& S, double* x, double* y, double* z, int32_t n,
                             cudaStream_t s) {
  if (n > 0) k_unpack<<<blocks_for(n, 256), 256, 0, s>>>(S, x, y, z, n);
}
void launch_pack_gate(const DevState& S, const double* x, const double* y, const double* z,
                      int32_t p0, int32_t p1, const LaunchCfg& lc, cudaStream_t s) {
  if (p1 > p0) k_pack_gate<<<stride_blocks(p1 - p0, lc.block, lc), lc.block, 0, s>>>(S, x, y, z, p0, p1);
}
void launch_unpack_range(const DevState& S, double* x, double* y, double* z, int32_t p0,
                         int32_t p1, const LaunchCfg& lc, cudaStream_t s) {
  if (p1 > p0)
    k_unpack_range<<<stride_blocks(p1 - p0, lc.block, lc), lc.block, 0, s>>>(S, x, y, z, p0, p1);
}
void launch_pack_positions(const DevState& S, const double* x, const double* y,
                           const double* z, int32_t n, cudaStream_t s) {
  if (n > 0) k_pack<<<blocks_for(n, 256), 256, 0, s>>>(S, x, y, z, n);
}

}  // namespace epi
