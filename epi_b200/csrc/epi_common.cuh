// Device-side data layout, helpers and force laws of the mechanics step.
//
// Layout in HBM (all tissues of a batch concatenated, particle g is particle
// g - pbase of its tissue):
//   pos[2][N]  double4 (x, y, z, radius), double-buffered (current / next);
//              the reference's dual_double d1 / d2 (epi5_MT/DualValue.h:17-55)
//   attr[N]    u32: bits 0-3 state, bit 4 "agek > THRESH_SP", bits 5-6 the
//              MUSUME membrane spring selector, bits 8-31 tissue id
//   pair[N]    i32 global partner index or -1; spr[N] double spring rest length
//   dermis[N]  i32 global index of the nearest connected MEMB (FIX/MUSUME)
//   cand[K][N] Verlet candidates (all partners within reach + skin at the
//              last rebuild) in 16-byte chunks, chunk k of particle i at
//              cand[k * N + i]: entry 0 is the count, entries 1.. the
//              tissue-local candidate indices, 8 per chunk (16-bit) or 4
//              (32-bit, when a tissue of the batch has 65,536 particles or
//              more). A warp's loads of chunk k of 32 consecutive particles
//              are one coalesced 512-byte request, and two loads give a
//              thread its first 15 candidates without a dependent load.
//   nbr[N][C]  i32 exact connection lists, materialised on request; nn[N].
//              Membrane lattice links are implicit in both.
//   sn/sm[N]   membrane bending scratch (unit vector + length to the right /
//              upper lattice neighbour), the reference's Memb_data
//              (epi5_MT/cell.h:42-69)
//   bins       counting-sort cell list over the reference's 2.0 grid
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace epi {

enum State : uint32_t {
  ST_ALIVE = 0, ST_DEAD = 1, ST_DISA = 2, ST_UNUSED = 3, ST_FIX = 4, ST_BLANK = 5,
  ST_DER = 6, ST_MUSUME = 7, ST_AIR = 8, ST_MEMB = 9
};

enum ErrCode : int32_t {
  E_OK = 0, E_BIN_RANGE = 5, E_BIN_OVERFLOW = 6, E_LIST_OVERFLOW = 7, E_COEF_RANGE = 8,
  E_MEMB_COEF_RANGE = 9, E_NONFINITE = 10, E_TIMEOUT = 11, E_UNSUPPORTED = 13, E_CHECK = 14
};

// The bounds-checked build (-DEPI_CHECK, libepi_mech_check.so): every index a
// kernel derives from stored data (candidate entries, bin slots, lattice
// sites, pair and dermis partners) is checked against the range it must lie
// in before it is used; a failed check records E_CHECK with the particle and
// the index, and the access is skipped. The release build compiles the
// checks away. It stands in for a memory checker, which this build does not
// rely on.
#ifdef EPI_CHECK
#define EPI_CHECKED(ok, status, a, b) \
  ((ok) ? true : (raise_error((status), E_CHECK, (a), (b), 0.0), false))
#else
#define EPI_CHECKED(ok, status, a, b) true
#endif

constexpr double kAreaGrid = 2.0 + 1e-7;  // AREA_GRID, cell_connection.cpp:16-19
constexpr int kBinCap = 200;              // N3, cell_connection.cpp:28
constexpr int kMembAdj = 4;               // MEMB_ADJ_CONN_NUM (square), define.h:147-153
constexpr int kMembAdjTri = 6;            // MEMB_ADJ_CONN_NUM (TRI_MEMB)
constexpr int kLatticeSquare = 0, kLatticeTriangular = 1;

struct Params {
  double dt, eps_m, p_memb, der_der_const, k_total, k_desmosome, kspring, kspring_d, kbend,
      delta_r, para_ljp2, kspring_division, lj_thresh, thresh_sp;
};

struct TissueDev;

struct DevStatus {
  int32_t flags;  // bit per ErrCode
  int32_t code;   // first error recorded
  int32_t a, b;   // particle / partner (global) of the first error
  double v;       // offending value
};

struct DevState {
  const TissueDev* tissues;
  double4* pos_cur;
  double4* pos_nxt;
  // FP32 copies of the positions (x, y, z, radius) for the mixed path's
  // candidate gathers and separations; written by the step with pos_nxt
  float4* posf_cur;
  float4* posf_nxt;
  const uint32_t* attr;
  const int32_t* pair;
  const double* spr;
  int32_t* dermis;
  // Verlet candidates: every partner within LJ_THRESH*(r_i+r_j) + skin at
  // the last rebuild, chunked rows (see the layout above; cand_* below).
  uint4* cand;
  int32_t cand16;   // 1: 16-bit entries, 0: 32-bit entries
  float4* bpos;     // positions at the last rebuild (displacement check)
  int32_t* nbr;     // exact connection lists (materialised on request)
  int32_t* nn;
  double4* fmemb;   // membrane bending + lattice spring + wall displacement
  int32_t* bin;
  int32_t* rank;    // place in its bin while binning; its slot once sorted
  int32_t* counts;
  int32_t* starts;
  uint32_t* skey;   // sorted particles: global index | (is_memb << 31)
  float4* spos;     // sorted copy of the positions at rebuild; w: +-LJ_THRESH * radius
  int32_t* gate;    // [0]: some tissue needs a rebuild, [1 + t]: tissue t does
  int32_t* rl_count;  // rebuild work list: number of gated tissues
  int32_t* rl_list;   // their ids
  int32_t* rl_ppre;   // prefix sums of their particle counts (count + 1 entries)
  int32_t* rl_bpre;   // prefix sums of their bin counts
  int32_t ntissues;
  const int32_t* prep;  // membrane particles, then FIX/MUSUME cells
  int32_t nprep, nprep_memb;
  DevStatus* status;
  unsigned long long* rebuilds;  // tissue candidate rebuilds so far
  unsigned long long* launches;  // kernels of the step sequence executed so far
  int64_t n_total;  // column stride of cand / nbr
  int32_t max_conn, max_cand;
  double skin;
};

__device__ __forceinline__ uint32_t attr_state(uint32_t a) { return a & 15u; }
__device__ __forceinline__ bool attr_old(uint32_t a) { return (a >> 4) & 1u; }
__device__ __forceinline__ uint32_t attr_sfm(uint32_t a) { return (a >> 5) & 3u; }
__device__ __forceinline__ uint32_t attr_tissue(uint32_t a) { return a >> 8; }

__device__ __forceinline__ void raise_error(DevStatus* s, int32_t code, int32_t a, int32_t b,
                                            double v) {
  atomicOr(&s->flags, 1 << code);
  if (atomicCAS(&s->code, 0, code) == 0) {
    s->a = a;
    s->b = b;
    s->v = v;
  }
}

// Candidate rows: entry e of particle i (entry 0: the count; entry k + 1:
// candidate k, tissue-local). 16-bit entries: chunk e / 8, half e % 8;
// 32-bit: chunk e / 4, word e % 4.
__device__ __forceinline__ uint32_t cand_entry(const DevState& S, int64_t i, int32_t e) {
  if (S.cand16) {
    const uint16_t* c = reinterpret_cast<const uint16_t*>(S.cand + (int64_t)(e >> 3) * S.n_total + i);
    return c[e & 7];
  }
  const uint32_t* c = reinterpret_cast<const uint32_t*>(S.cand + (int64_t)(e >> 2) * S.n_total + i);
  return c[e & 3];
}
__device__ __forceinline__ void cand_set(const DevState& S, int64_t i, int32_t e, uint32_t v) {
  if (!EPI_CHECKED(e >= 0 && e <= S.max_cand && (e == 0 || v < 65536u || !S.cand16), S.status,
                   (int32_t)i, e))
    return;
  if (S.cand16) {
    uint16_t* c = reinterpret_cast<uint16_t*>(S.cand + (int64_t)(e >> 3) * S.n_total + i);
    c[e & 7] = (uint16_t)v;
  } else {
    uint32_t* c = reinterpret_cast<uint32_t*>(S.cand + (int64_t)(e >> 2) * S.n_total + i);
    c[e & 3] = v;
  }
}
__device__ __forceinline__ int32_t cand_count(const DevState& S, int64_t i) {
  return (int32_t)cand_entry(S, i, 0);
}

// Minimum-image difference, p_diff_x / p_diff_y (epi5_MT/utils.h:25-41).
// Plain IEEE subtraction and comparison: identical rounding on CPU and GPU.
__device__ __forceinline__ double pdiff(double a, double b, double L) {
  const double d = a - b;
  if (d > 0.5 * L) return d - L;
  if (d <= -0.5 * L) return d + L;
  return d;
}

// |d|^2 exactly as the reference evaluates DIST_SQ / p_dist_sq
// (utils.h:48-53, cell_connection.cpp:115-119): no fused multiply-add.
__device__ __forceinline__ double dist_sq_exact(double dx, double dy, double dz) {
  return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

// Connection predicate of connect_proc (cell_connection.cpp:118-119):
// |d|^2 <= LJ_THRESH*LJ_THRESH*rad_sum*rad_sum, evaluated left to right.
__device__ __forceinline__ bool connected_pred(double d2, double lt, double ri, double rj) {
  const double rs = __dadd_rn(ri, rj);
  return d2 <= __dmul_rn(__dmul_rn(__dmul_rn(lt, lt), rs), rs);
}

// Division and square root of the force laws: IEEE in the FP64 path, the
// hardware approximations (MUFU reciprocal / reciprocal square root, about
// 2 ulp) in the FP32 path.
__device__ __forceinline__ double ldiv(double a, double b) { return a / b; }
__device__ __forceinline__ float ldiv(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double lsqrt(double v) { return sqrt(v); }
__device__ __forceinline__ float lsqrt(float v) { return v * rsqrtf(v); }

template <typename R>
__device__ __forceinline__ R pow6(R v) { return v * v * v * v * v * v; }
template <typename R>
__device__ __forceinline__ R pow3(R v) { return v * v * v; }

// Force laws (epi5_MT/cell_interaction.cpp:77-285). Each takes the squared
// distance d2 and radius sum rs of the pair and returns the coefficient that
// cell_interaction_apply multiplies by DT and the separation (:48-66).
template <typename R>
struct Laws {
  R eps4, p_memb, der_der_const, k_total, k_desmosome, kspring, kspring_d, delta_r, para_ljp2,
      kspring_division, lj_thresh, ljt1sq;

  // ljmain, :103-111
  __device__ __forceinline__ R ljmain(R d2, R rs) const {
    const R lj6 = ldiv(pow6(rs), pow3(d2));
    return ldiv(eps4 * lj6 * (lj6 - R(1)), d2);
  }
  // adhesion, :113-124
  __device__ __forceinline__ R adhesion(R d2, R rs, R k) const {
    const R d = lsqrt(d2);
    const R m1 = ldiv(d, rs) - R(1);
    return (m1 + R(1) > lj_thresh) ? R(0) : -ldiv(k, d) * m1 * (R(1) - ldiv(m1 * m1, ljt1sq));
  }
  // is_near, :90-93
  __device__ __forceinline__ bool near(R d2, R rs) const { return d2 < rs * rs; }
  // CI_der_to_der, :129-139
  __device__ __forceinline__ R der_der(R d2, R rs) const {
    const R d = lsqrt(d2);
    const R dd = d + delta_r;
    if (dd < rs) {
      const R lj6 = ldiv(pow6(rs), pow6(dd));
      return ldiv(eps4 * lj6 * (lj6 - R(1)), d * dd) + para_ljp2;
    }
    if (near(d2, rs)) return para_ljp2;
    const R lj6 = ldiv(pow6(rs), pow6(dd));
    return ldiv(eps4 * lj6 * (lj6 - R(1)), d * d) + para_ljp2;
  }
  // CI_al_air_de_to_al_air_de_fix_mu, :141-152
  __device__ __forceinline__ R aad(R d2, R rs, bool both_old) const {
    if (near(d2, rs)) return ljmain(d2, rs);
    return adhesion(d2, rs, both_old ? k_total : k_desmosome);
  }
  // The same law in FP32 without a branch: both sides from one reciprocal
  // square root, then a select, so lanes of a warp on either side of
  // is_near do not run both paths one after the other.
  __device__ __forceinline__ float aad_fused(float d2, float rs, bool both_old) const {
    const float inv_d = rsqrtf(d2);
    const float inv_d2 = inv_d * inv_d;
    const float r2 = rs * rs;
    const float s = r2 * inv_d2;
    const float lj6 = s * s * s;
    const float c_lj = eps4 * lj6 * (lj6 - 1.f) * inv_d2;
    const float m1 = __fdividef(d2 * inv_d, rs) - 1.f;
    const float k = both_old ? k_total : k_desmosome;
    const float c_ad =
        (m1 + 1.f > lj_thresh) ? 0.f : -k * inv_d * m1 * (1.f - __fdividef(m1 * m1, ljt1sq));
    return d2 < r2 ? c_lj : c_ad;
  }
  // CI_fix_mu_to_fix_mu, :154-162
  __device__ __forceinline__ R fixmu(R d2, R rs) const {
    if (near(d2, rs)) return ljmain(d2, rs);
    return adhesion(d2, rs, k_desmosome);
  }
  // CI_mu_to_memb, :164-172 (spring = the MUSUME's spring_force_to_memb)
  __device__ __forceinline__ R mu_memb(R d2, R rs, R spring) const {
    if (near(d2, rs)) return ljmain(d2, rs);
    return adhesion(d2, rs, spring);
  }
  // CI_fix_to_memb, :174-183
  __device__ __forceinline__ R fix_memb(R d2, R rs) const {
    if (near(d2, rs)) return ljmain(d2, rs);
    const R d = lsqrt(d2);
    return -ldiv(kspring, d) * (ldiv(d, rs) - R(1));
  }
  // CI_memb_to_memb, :185-234; *bad set when |coef| > 100 (the reference aborts)
  __device__ __forceinline__ R memb_memb(R d2, R rs, bool* bad) const {
    const R rs2 = rs * rs;
    const R cr2 = rs2 * p_memb * p_memb;
    R tmp;
    if (d2 < cr2) {
      const R lj6 = ldiv(pow3(cr2), pow3(d2));
      tmp = ldiv(eps4 * lj6 * (lj6 - R(1)), d2);
    } else if (d2 < rs2) {
      const R d = lsqrt(d2);
      tmp = -ldiv(der_der_const, d) * (ldiv(d, rs * p_memb) - R(1));
    } else {
      const R d = lsqrt(d2);
      const R lam = (R(1) + p_memb) * rs;
      const R lj6 = ldiv(pow6(rs * p_memb), pow6(lam - d));
      tmp = -ldiv(der_der_const, rs) * ldiv(R(1) - p_memb, p_memb) -
            ldiv(eps4 * (lj6 * (lj6 - R(1))), (lam - d) * d);
    }
    *bad = fabs(tmp) > R(100);
    return tmp;
  }
  // CI_pair, :281-285 (rest = the first cell's spr_nat_len)
  __device__ __forceinline__ R pair(R d2, R rest) const {
    const R d = lsqrt(d2);
    return ldiv(-(kspring_division * (d - rest)), d);
  }
};

// Constants of the laws in arithmetic type R, precomputed once per tissue.
template <typename R>
__host__ __device__ inline Laws<R> make_laws(const Params& P) {
  Laws<R> L;
  L.eps4 = R(4.0 * P.eps_m);
  L.p_memb = R(P.p_memb);
  L.der_der_const = R(P.der_der_const);
  L.k_total = R(P.k_total);
  L.k_desmosome = R(P.k_desmosome);
  L.kspring = R(P.kspring);
  L.kspring_d = R(P.kspring_d);
  L.delta_r = R(P.delta_r);
  L.para_ljp2 = R(P.para_ljp2);
  L.kspring_division = R(P.kspring_division);
  L.lj_thresh = R(P.lj_thresh);
  L.ljt1sq = R((P.lj_thresh - 1.0) * (P.lj_thresh - 1.0));
  return L;
}

// Law selected when cell c iterates its connection o (the per-state bodies
// of cell_interaction.cpp:549-634). Index order decides double counting
// (no_double_count, cell.h:293-295).
enum Law : int { L_NONE = 0, L_OTHER, L_DER_DER, L_AAD, L_FIXMU, L_FIX_MEMB, L_MU_MEMB };

__device__ __forceinline__ bool is_aad_state(uint32_t s) {
  return s == ST_ALIVE || s == ST_AIR || s == ST_DEAD;
}

__device__ __forceinline__ int law_of(uint32_t sc, int32_t c, int32_t c_pair, int32_t c_dermis,
                                      uint32_t so, int32_t o) {
  switch (sc) {
    case ST_DER:  // _DER_interaction, :549-561
      return (so == ST_DER && c > o) ? L_DER_DER : L_OTHER;
    case ST_ALIVE:
    case ST_AIR:
    case ST_DEAD:  // _AL_AIR_DE_interaction, :563-579
      if (is_aad_state(so)) return c > o ? L_AAD : L_NONE;
      return so == ST_DER ? L_NONE : L_AAD;
    case ST_FIX:  // _FIX_interaction, :581-604
      if (so == ST_FIX) return (c_pair != o && c > o) ? L_FIXMU : L_NONE;
      if (so == ST_MUSUME) return c_pair != o ? L_FIXMU : L_NONE;
      if (so == ST_MEMB) return c_dermis == o ? L_FIX_MEMB : L_OTHER;
      return L_NONE;
    case ST_MUSUME:  // _MUSUME_interaction, :613-634
      if (so == ST_MEMB) return c_dermis == o ? L_MU_MEMB : L_OTHER;
      if (so == ST_MUSUME && c_pair != o && c > o) return L_FIXMU;
      return L_NONE;
    default:
      return L_NONE;
  }
}

// spring_force_to_memb of a MUSUME (cell_interaction.cpp:614-620), selected
// on the host at upload: 0 -> 0, 1 -> Kspring, 2 -> Kspring_d.
template <typename R>
__device__ __forceinline__ R sfm_value(uint32_t code, const Laws<R>& L) {
  return code == 1 ? L.kspring : (code == 2 ? L.kspring_d : R(0));
}

template <typename R>
__device__ __forceinline__ R eval_law(int law, const Laws<R>& L, R d2, R rs, bool both_old,
                                      uint32_t c_sfm) {
  switch (law) {
    case L_OTHER: return L.ljmain(d2, rs);
    case L_DER_DER: return L.der_der(d2, rs);
    case L_AAD: return L.aad(d2, rs, both_old);
    case L_FIXMU: return L.fixmu(d2, rs);
    case L_FIX_MEMB: return L.fix_memb(d2, rs);
    case L_MU_MEMB: return L.mu_memb(d2, rs, sfm_value(c_sfm, L));
    default: return R(0);
  }
}

struct TissueDev {
  int32_t pbase, n, nmemb, nder, nmx, nmy;
  int32_t anx, any, anz;  // reference grid (cell_connection.cpp:22-26)
  int32_t binbase;        // first bin; a tissue owns anx*any*anz bins + 1 sentinel
  int32_t lattice;        // kLatticeSquare / kLatticeTriangular
  int32_t nadj;           // lattice links per membrane particle (4 / 6)
  int32_t mbase;          // index in prep of the tissue's first membrane particle
  double lx, ly, lz, hlx, hly;     // box and half box
  double rmax;     // largest radius in the tissue
  double rmax_nm;  // largest non-membrane radius (membranes only pair with those)
  // Range asserts of grid_init / connect_proc (cell_connection.cpp:48-53,
  // :99) as thresholds on a wrapped position, found on the host with the
  // same IEEE arithmetic: grid_init fails for gx_hi <= x < lx (x == lx wraps
  // to bin 0), gy_hi likewise, z >= gz_hi; connect_proc (non-membrane cells)
  // fails for x >= cx_hi, y >= cy_hi, z >= cz_hi or z <= cz_lo.
  double gx_hi, gy_hi, gz_hi, cx_hi, cy_hi, cz_hi, cz_lo;
  // Mixed path: the box and its inverse in FP32, LJ_THRESH^2 in FP32, and
  // ftol, a bound on |d2_f32 - d2_exact| + |thr_f32 - thr_exact| for any
  // pair that can be connected (positions rounded to FP32 once, separations
  // and the threshold evaluated in FP32). A candidate whose FP32 d2 lies
  // within ftol of the FP32 threshold is decided by the exact FP64 predicate.
  float lxf, lyf, lt2f, ftol;
  float ilxf, ilyf;  // 1 / L in FP32 (minimum image as f - L rint(f / L))
  Params P;
  Laws<float> lawf;
  Laws<double> lawd;
  template <typename R>
  __device__ __forceinline__ const Laws<R>& laws() const;
};
template <>
__device__ __forceinline__ const Laws<float>& TissueDev::laws<float>() const { return lawf; }
template <>
__device__ __forceinline__ const Laws<double>& TissueDev::laws<double>() const { return lawd; }

// The reference's range asserts for a wrapped position (see TissueDev).
__device__ __forceinline__ bool range_ok(const TissueDev& T, double x, double y, double z,
                                         bool memb) {
  bool ok = (x < T.gx_hi || x >= T.lx) && (y < T.gy_hi || y >= T.ly) && z < T.gz_hi;
  if (!memb) ok = ok && x < T.cx_hi && y < T.cy_hi && z < T.cz_hi && z > T.cz_lo;
  return ok;
}

// Minimum-image difference with a precomputed half box (same result as pdiff).
__device__ __forceinline__ double pdiff_h(double a, double b, double L, double h) {
  const double d = a - b;
  if (d > h) return d - L;
  if (d <= -h) return d + L;
  return d;
}

// Square membrane lattice neighbours of membrane particle j (tissue-local),
// _memb_init square branch (epi5_MT/cellmanager.cpp:114-158).
struct Lattice {
  int32_t l, ll, r, b, bb, u;
};
__device__ __forceinline__ Lattice lattice_of(int32_t j, int32_t NMX, int32_t NMY) {
  const int32_t jj = j % NMX, kk = j / NMX;
  Lattice L;
  L.l = jj == 0 ? j + NMX - 1 : j - 1;
  L.ll = jj <= 1 ? j + NMX - 2 : j - 2;
  L.r = jj == NMX - 1 ? j - (NMX - 1) : j + 1;
  L.b = kk == 0 ? j + NMX * NMY - NMX : j - NMX;
  L.bb = kk <= 1 ? j + NMX * NMY - 2 * NMX : j - 2 * NMX;
  L.u = kk == NMY - 1 ? j - (NMX * NMY - NMX) : j + NMX;
  return L;
}

// Triangular lattice: Memb_data::memb[k] of membrane particle j (tissue-local)
// as _memb_init's TRI_MEMB branch wires it (epi5_MT/cellmanager.cpp:70-111):
// 0 right, 3 left; 1, 2 in the row above (j - NMX) and 4, 5 in the row
// below (j + NMX), which of the two columns depending on the row's parity.
__host__ __device__ __forceinline__ int32_t tri_link(int32_t j, int k, int32_t NMX, int32_t nm) {
  auto left = [NMX](int32_t v) { return v % NMX == 0 ? v + NMX - 1 : v - 1; };
  auto right = [NMX](int32_t v) { return v % NMX == NMX - 1 ? v - (NMX - 1) : v + 1; };
  const bool even = (j / NMX) % 2 == 0;
  const int32_t top = (j - NMX + nm) % nm, bot = (j + NMX) % nm;
  switch (k) {
    case 0: return right(j);
    case 1: return even ? top : right(top);
    case 2: return even ? left(top) : top;
    case 3: return left(j);
    case 4: return even ? left(bot) : bot;
    default: return even ? bot : right(bot);
  }
}

// tri_link as a step from (column, row): the same wiring with conditional
// wraps instead of integer divisions (rows alternate their offset; NMY is
// even, so the row wrap keeps the alternation).
struct TriSite {
  int32_t col, row;
};
__device__ __forceinline__ TriSite tri_step(TriSite s, int k, int32_t NMX, int32_t NMY) {
  const bool even = (s.row & 1) == 0;
  int32_t c = s.col, r = s.row;
  switch (k) {
    case 0: c += 1; break;
    case 1: r -= 1; c += even ? 0 : 1; break;
    case 2: r -= 1; c -= even ? 1 : 0; break;
    case 3: c -= 1; break;
    case 4: r += 1; c -= even ? 1 : 0; break;
    default: r += 1; c += even ? 0 : 1; break;
  }
  c += c < 0 ? NMX : 0;
  c -= c >= NMX ? NMX : 0;
  r += r < 0 ? NMY : 0;
  r -= r >= NMY ? NMY : 0;
  return TriSite{c, r};
}

// The k-th lattice link of membrane particle j in connected_cell's push
// order: square l, r, b, u (cellmanager.cpp:160-163), triangular memb[0..5].
__device__ __forceinline__ int32_t lattice_link(const TissueDev& T, int32_t j, int k) {
  if (T.lattice == kLatticeTriangular) return tri_link(j, k, T.nmx, T.nmemb);
  const Lattice L = lattice_of(j, T.nmx, T.nmy);
  return k == 0 ? L.l : (k == 1 ? L.r : (k == 2 ? L.b : L.u));
}

}  // namespace epi
