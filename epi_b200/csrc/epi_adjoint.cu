// Reverse-mode adjoint of the mechanics step, FP64.
//
// The step maps positions X_t to X_{t+1} = wrap(X_t + D(X_t; s)), where D is
// the displacement cell_interaction accumulates (epi5_MT/cell_interaction.cpp
// :648-685) and s = (s_spring, s_eps, s_bend) multiplies every spring
// constant, eps_m and KBEND. The wrap is a translation by a box length, so
// its derivative is the identity. Given lambda = dL/dX_{t+1}, one backward
// step returns
//   dL/dX_t = lambda + (dD/dX_t)^T lambda     and adds   (dD/ds)^T lambda
// to the parameter gradient. The connection set of step t is the exact
// predicate of connect_proc at X_t (piecewise constant in X), evaluated on
// the Verlet candidates like the forward step.
//
// Terms of D, for every cell state of the path:
//   pairs     D_i += DT c(r2) d_ij, c the sum of the laws the reference
//             applies to the pair from either side (law_of: ljmain, adhesion,
//             CI_der_to_der, the FIX / MUSUME dermis springs, :103-183,
//             549-634); J = c I + 2 c'(r2) d d^T and D_j gets -DT c d_ij, so
//             (dD/dX)^T lambda at i is DT sum_j J (lambda_i - lambda_j): a
//             gather over the same lists. The pair springs of dividing cells
//             (CI_pair, :281-285, 637-641) add the same form for the partner.
//   lattice   the four lattice springs of _MEMB_interaction (CI_memb_to_memb,
//             :185-234), the same gather over fixed partners.
//   wall      z += DT W(z) for z < r, membrane and DER (:287-294, 549-561).
//   bending   D_k += DT KBEND B_k(stencil sites): square, eleven lattice
//             sites (_memb_bend_calc1..3, :296-449); triangular, the six
//             neighbours and six second-ring sites of the twelve dihedral
//             terms of tri_memb_bend (:451-508). Their vector-Jacobian
//             products are derived by hand below; each membrane particle
//             writes the products for the sites of its stencil and every
//             site gathers the entries that name it, so no atomics are
//             needed and results are deterministic.
#include "epi_kernels.h"
#include "epi_device.cuh"

namespace epi {
namespace {

struct D3 {
  double x, y, z;
};
__device__ __forceinline__ D3 d3(double x, double y, double z) { return D3{x, y, z}; }
__device__ __forceinline__ D3 operator+(D3 a, D3 b) { return D3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ D3 operator-(D3 a, D3 b) { return D3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ D3 operator*(double s, D3 a) { return D3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ D3& operator+=(D3& a, D3 b) { return a = a + b; }
__device__ __forceinline__ D3& operator-=(D3& a, D3 b) { return a = a - b; }
__device__ __forceinline__ double dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ D3 xyz(double4 v) { return D3{v.x, v.y, v.z}; }
__device__ __forceinline__ D3 cross(D3 a, D3 b) {
  return D3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// A pair coefficient with its derivatives: c, dc/d(r2), and the parts of c
// that scale with s_spring and with s_eps (each law is linear in them).
struct LawD {
  double c, dc_dr2, c_spring, c_eps;
};
__device__ __forceinline__ LawD operator+(const LawD& a, const LawD& b) {
  return LawD{a.c + b.c, a.dc_dr2 + b.dc_dr2, a.c_spring + b.c_spring, a.c_eps + b.c_eps};
}

// ljmain (:103-111): c = eps4 u (u - 1) / r2 with u = rs^6 / r2^3.
__device__ __forceinline__ LawD ljmain_d(const Laws<double>& L, double r2, double rs) {
  const double rs2 = rs * rs;
  const double u = rs2 * rs2 * rs2 / (r2 * r2 * r2);
  const double c = L.eps4 * u * (u - 1.0) / r2;
  const double dc = -L.eps4 * u * (7.0 * u - 4.0) / (r2 * r2);
  return LawD{c, dc, 0.0, c};
}

// adhesion (:113-124) with spring constant k.
__device__ __forceinline__ LawD adhesion_d(const Laws<double>& L, double r2, double rs,
                                           double k) {
  const double r = sqrt(r2);
  const double y = r / rs - 1.0;
  if (y + 1.0 > L.lj_thresh) return LawD{0.0, 0.0, 0.0, 0.0};
  const double h = 1.0 - y * y / L.ljt1sq;
  const double c = -(k / r) * y * h;
  // dc/dr = k y h / r^2 - (k / r) (1 - 3 y^2 / a^2) / rs
  const double dcdr = k * y * h / r2 - (k / r) * (1.0 - 3.0 * y * y / L.ljt1sq) / rs;
  return LawD{c, dcdr / (2.0 * r), c, 0.0};
}

// CI_al_air_de_to_al_air_de_fix_mu (:141-152).
__device__ __forceinline__ LawD aad_d(const Laws<double>& L, double r2, double rs,
                                      bool both_old) {
  if (r2 < rs * rs) return ljmain_d(L, r2, rs);
  return adhesion_d(L, r2, rs, both_old ? L.k_total : L.k_desmosome);
}

// CI_fix_mu_to_fix_mu (:154-162).
__device__ __forceinline__ LawD fixmu_d(const Laws<double>& L, double r2, double rs) {
  if (r2 < rs * rs) return ljmain_d(L, r2, rs);
  return adhesion_d(L, r2, rs, L.k_desmosome);
}

// CI_mu_to_memb (:164-172) with the MUSUME's spring_force_to_memb.
__device__ __forceinline__ LawD mu_memb_d(const Laws<double>& L, double r2, double rs,
                                          uint32_t sfm) {
  if (r2 < rs * rs) return ljmain_d(L, r2, rs);
  return adhesion_d(L, r2, rs, sfm_value(sfm, L));
}

// CI_fix_to_memb (:174-183): c = -(kspring / r) (r / rs - 1) = kspring (1/r - 1/rs).
__device__ __forceinline__ LawD fix_memb_d(const Laws<double>& L, double r2, double rs) {
  if (r2 < rs * rs) return ljmain_d(L, r2, rs);
  const double r = sqrt(r2);
  const double c = -(L.kspring / r) * (r / rs - 1.0);
  return LawD{c, -L.kspring / (2.0 * r2 * r), c, 0.0};
}

// CI_der_to_der (:129-139), dd = r + delta_R, u = (rs / dd)^6, h = u (u - 1):
// eps4 h / (r dd) + para_ljp2 while dd < rs, para_ljp2 inside the radius
// sum, eps4 h / r^2 + para_ljp2 beyond; dh/dr = -6 u (2 u - 1) / dd.
__device__ __forceinline__ LawD der_der_d(const Laws<double>& L, double r2, double rs) {
  const double r = sqrt(r2);
  const double dd = r + L.delta_r;
  if (!(dd < rs) && r2 < rs * rs) return LawD{L.para_ljp2, 0.0, 0.0, 0.0};
  const double rs2 = rs * rs, dd2 = dd * dd;
  const double u = rs2 * rs2 * rs2 / (dd2 * dd2 * dd2);
  const double h = u * (u - 1.0);
  const double dh = -6.0 * u * (2.0 * u - 1.0) / dd;
  double ce, dce;
  if (dd < rs) {
    const double q = r * dd;
    ce = L.eps4 * h / q;
    dce = L.eps4 * (dh / q - h * (dd + r) / (q * q));
  } else {
    ce = L.eps4 * h / r2;
    dce = L.eps4 * (dh / r2 - 2.0 * h / (r2 * r));
  }
  return LawD{ce + L.para_ljp2, dce / (2.0 * r), 0.0, ce};
}

// CI_pair (:281-285): c = -Kdiv (r - rest) / r, rest the higher index's
// spr_nat_len.
__device__ __forceinline__ LawD pair_d(const Laws<double>& L, double r2, double rest) {
  const double r = sqrt(r2);
  const double c = -(L.kspring_division * (r - rest)) / r;
  return LawD{c, -L.kspring_division * rest / (2.0 * r2 * r), c, 0.0};
}

// The law `law` (law_of) as a LawD.
__device__ __forceinline__ LawD law_d(int law, const Laws<double>& L, double r2, double rs,
                                      bool both_old, uint32_t sfm) {
  switch (law) {
    case L_OTHER: return ljmain_d(L, r2, rs);
    case L_DER_DER: return der_der_d(L, r2, rs);
    case L_AAD: return aad_d(L, r2, rs, both_old);
    case L_FIXMU: return fixmu_d(L, r2, rs);
    case L_FIX_MEMB: return fix_memb_d(L, r2, rs);
    case L_MU_MEMB: return mu_memb_d(L, r2, rs, sfm);
    default: return LawD{0.0, 0.0, 0.0, 0.0};
  }
}

// wall_interaction (:287-294): dz = dt eps4 u (u - 1) / (2 z), u = (r / z)^6;
// adds its adjoint to mu.z and its eps part to g_eps.
__device__ __forceinline__ void wall_back(const Laws<double>& L, double dt, double z, double rad,
                                          double lz, D3& mu, double& g_eps) {
  const double rz = rad / z;
  const double rz2 = rz * rz;
  const double u = rz2 * rz2 * rz2;
  const double W = dt * L.eps4 * u * (u - 1.0) / (2.0 * z);
  const double dW = -dt * L.eps4 * u * (13.0 * u - 7.0) / (2.0 * z * z);
  mu.z += dW * lz;
  g_eps += W * lz;
}

// CI_memb_to_memb (:185-234), three branches.
__device__ __forceinline__ LawD memb_memb_d(const Laws<double>& L, double r2, double rs) {
  const double P = L.p_memb;
  const double rs2 = rs * rs;
  const double cr2 = rs2 * P * P;
  if (r2 < cr2) {
    const double u = cr2 * cr2 * cr2 / (r2 * r2 * r2);
    const double c = L.eps4 * u * (u - 1.0) / r2;
    return LawD{c, -L.eps4 * u * (7.0 * u - 4.0) / (r2 * r2), 0.0, c};
  }
  const double r = sqrt(r2);
  if (r2 < rs2) {
    const double c = -(L.der_der_const / r) * (r / (rs * P) - 1.0);
    return LawD{c, -L.der_der_const / (2.0 * r2 * r), c, 0.0};
  }
  const double lam = (1.0 + P) * rs;
  const double v = lam - r;
  const double cr = rs * P;
  const double cr2v = cr * cr / (v * v);
  const double u = cr2v * cr2v * cr2v;
  const double c_spring = -(L.der_der_const / rs) * ((1.0 - P) / P);
  const double vr = v * r;
  const double c_eps = -L.eps4 * u * (u - 1.0) / vr;
  // d/dr of u (u - 1) / (v r), with du/dr = 6 u / v and d(v r)/dr = v - r
  const double dh = 6.0 * u * (2.0 * u - 1.0) / (v * vr) - u * (u - 1.0) * (v - r) / (vr * vr);
  return LawD{c_spring + c_eps, -L.eps4 * dh / (2.0 * r), c_spring, c_eps};
}

// _memb_bend_diff_factor (:349-360) and its derivative.
__device__ __forceinline__ double bf(double c) {
  return c >= 0.0 ? 1.0 - c : 1.0 / ((1.0 + c) * (1.0 + c));
}
__device__ __forceinline__ double bf_d(double c) {
  if (c >= 0.0) return -1.0;
  const double e = 1.0 + c;
  return -2.0 / (e * e * e);
}

// Unit vector of b - a with its length.
struct U3 {
  D3 v;
  double len;
};
__device__ __forceinline__ U3 unit3(D3 a, D3 b) {
  const D3 w = b - a;
  const double len = sqrt(dot(w, w));
  return U3{(1.0 / len) * w, len};
}
// Adjoint of w = b - a from the adjoints of the unit vector (ub) and of the
// length (lb): w_bar = (ub - (ub . u) u) / len + lb u; b += w_bar, a -= w_bar.
__device__ __forceinline__ void unit3_back(const U3& u, D3 ub, double lb, D3& abar, D3& bbar) {
  const D3 w = (1.0 / u.len) * (ub - dot(ub, u.v) * u.v) + lb * u.v;
  bbar += w;
  abar -= w;
}

// Stencil slots of the bending term of particle k, as lattice offsets:
// k, r, rr, l, ll, u, uu, b, bb, r of bb, rr of bb.
constexpr int kSlots = 11;
// Triangular lattice: k, its neighbour in direction i (slot 1 + i), and the
// second-ring site c_i = memb[(i+1)%6]->memb[i] (slot 7 + i).
constexpr int kTriSlots = 13;
// Entries per membrane particle in the bending-product buffer.
constexpr int kBendStride = 13;
__constant__ int kSlotDj[kSlots] = {0, 1, 2, -1, -2, 0, 0, 0, 0, 1, 2};
__constant__ int kSlotDk[kSlots] = {0, 0, 0, 0, 0, 1, 2, -1, -2, -2, -2};

// One half of BCALC (:396-404) and its adjoint. With n, a (the right /
// upper neighbour's vector), l, m (the left / lower ones), the lengths D, E
// and the cosines p = n.a, q = l.n, w:
//   T = -g(p) (a - p n) / D + g(q) ((n - q l) / E - (l - q n) / D)
//       + g(w) (m - w l) / E.
// Given ybar, returns y . T and accumulates the adjoints of n, a, l, m, D, E
// and w (w's inputs differ between the two halves).
struct HalfBar {
  D3 n, a, l, m;
  double D, E, w;
};
__device__ __forceinline__ double half_back(D3 yb, D3 n, D3 a, D3 l, D3 m, double D, double E,
                                            double w, HalfBar& hb) {
  const double p = dot(n, a), q = dot(l, n);
  const double gp = bf(p), gq = bf(q), gw = bf(w);
  const double yn = dot(yb, n), ya = dot(yb, a), yl = dot(yb, l), ym = dot(yb, m);
  const double iD = 1.0 / D, iE = 1.0 / E;
  const double val = -gp * (ya - p * yn) * iD + gq * ((yn - q * yl) * iE - (yl - q * yn) * iD) +
                     gw * (ym - w * yl) * iE;
  const double pb = (-bf_d(p) * (ya - p * yn) + gp * yn) * iD;
  const double qb = bf_d(q) * ((yn - q * yl) * iE - (yl - q * yn) * iD) + gq * (yn * iD - yl * iE);
  hb.w = bf_d(w) * (ym - w * yl) * iE - gw * yl * iE;
  hb.a = (-gp * iD) * yb + pb * n;
  hb.n = (gp * p * iD + gq * iE + gq * q * iD) * yb + pb * a + qb * l;
  hb.l = (-gq * q * iE - gq * iD - gw * w * iE) * yb + qb * n;
  hb.m = (gw * iE) * yb;
  hb.D = (gp * (ya - p * yn) + gq * (yl - q * yn)) * iD * iD;
  hb.E = -(gq * (yn - q * yl) + gw * (ym - w * yl)) * iE * iE;
  return val;
}

// tri_bend_1 (:475-481) of particle k with offsets a = n_i, b = n_{i+1},
// c = c_i (k at the origin): term = g(d) ab x (n2 - d n1), n1 = unit(rb x
// ab), n2 = unit(ab x cb), d = n1 . n2, rb = -b, ab = a - b, cb = c - b (the
// reference's division by the norm of an already normalised normal is 1 up
// to rounding and is left out, as in the forward step). Returns y . term and
// accumulates the adjoints of a, b, c. For p x q the adjoints are q x ybar
// and ybar x p; for n = N / |N|, Nbar = (nbar - (nbar . n) n) / |N|.
__device__ __forceinline__ double tri1_back(D3 y, D3 a, D3 b, D3 c, D3& abar, D3& bbar,
                                            D3& cbar) {
  const D3 rb = d3(-b.x, -b.y, -b.z), ab = a - b, cb = c - b;
  const D3 N1 = cross(rb, ab), N2 = cross(ab, cb);
  const double l1 = sqrt(dot(N1, N1)), l2 = sqrt(dot(N2, N2));
  const D3 n1 = (1.0 / l1) * N1, n2 = (1.0 / l2) * N2;
  const double d = dot(n1, n2);
  const D3 v = n2 - d * n1;
  const D3 t = cross(ab, v);
  const double g = bf(d), yt = dot(y, t);
  double dbar = bf_d(d) * yt;
  const D3 tbar = g * y;
  D3 abbar = cross(v, tbar);
  const D3 vbar = cross(tbar, ab);
  D3 n2bar = vbar, n1bar = (-d) * vbar;
  dbar -= dot(vbar, n1);
  n1bar += dbar * n2;
  n2bar += dbar * n1;
  const D3 N1bar = (1.0 / l1) * (n1bar - dot(n1bar, n1) * n1);
  const D3 N2bar = (1.0 / l2) * (n2bar - dot(n2bar, n2) * n2);
  const D3 rbbar = cross(ab, N1bar);
  abbar += cross(N1bar, rb);
  abbar += cross(cb, N2bar);
  const D3 cbbar = cross(N2bar, ab);
  abar += abbar;
  bbar -= abbar;
  bbar -= rbbar;
  bbar -= cbbar;
  cbar += cbbar;
  return g * yt;
}

// tri_bend_2 (:483-495) with a = n_i, b = n_{i+1}, cc = n_{i+2}: term =
// g(d) [bc x (n2 - d n1) + ab x (n1 - d n2)], n1 = unit(rc x bc), n2 =
// unit(rb x ab), rc = -cc, rb = -b, bc = b - cc, ab = a - b.
__device__ __forceinline__ double tri2_back(D3 y, D3 a, D3 b, D3 cc, D3& abar, D3& bbar,
                                            D3& ccbar) {
  const D3 rc = d3(-cc.x, -cc.y, -cc.z), rb = d3(-b.x, -b.y, -b.z);
  const D3 bc = b - cc, ab = a - b;
  const D3 N1 = cross(rc, bc), N2 = cross(rb, ab);
  const double l1 = sqrt(dot(N1, N1)), l2 = sqrt(dot(N2, N2));
  const D3 n1 = (1.0 / l1) * N1, n2 = (1.0 / l2) * N2;
  const double d = dot(n1, n2);
  const D3 v1 = n2 - d * n1, v2 = n1 - d * n2;
  const D3 t = cross(bc, v1) + cross(ab, v2);
  const double g = bf(d), yt = dot(y, t);
  double dbar = bf_d(d) * yt;
  const D3 tbar = g * y;
  D3 bcbar = cross(v1, tbar);
  const D3 v1bar = cross(tbar, bc);
  D3 abbar = cross(v2, tbar);
  const D3 v2bar = cross(tbar, ab);
  D3 n2bar = v1bar - d * v2bar, n1bar = v2bar - d * v1bar;
  dbar -= dot(v1bar, n1) + dot(v2bar, n2);
  n1bar += dbar * n2;
  n2bar += dbar * n1;
  const D3 N1bar = (1.0 / l1) * (n1bar - dot(n1bar, n1) * n1);
  const D3 N2bar = (1.0 / l2) * (n2bar - dot(n2bar, n2) * n2);
  const D3 rcbar = cross(bc, N1bar);
  bcbar += cross(N1bar, rc);
  const D3 rbbar = cross(ab, N2bar);
  abbar += cross(N2bar, rb);
  ccbar -= rcbar;
  ccbar -= bcbar;
  bbar -= rbbar;
  bbar += bcbar;
  bbar -= abbar;
  abar += abbar;
  return g * yt;
}

// Membrane particles: bending, lattice-spring and wall adjoints. Writes the
// bending products for the stencil sites to bend[e * kBendStride + slot],
// the lattice + wall product at the particle itself to madj[e], and the
// parameter partials to gmemb[e].
__global__ void __launch_bounds__(256) k_adj_memb(DevState S, const double4* __restrict__ lam,
                                                  double4* __restrict__ bend,
                                                  double4* __restrict__ madj,
                                                  double4* __restrict__ gmemb) {
  GRID_STRIDE(e, 0, S.nprep_memb) {
    const int32_t i = S.prep[e];
    const TissueDev& T = S.tissues[attr_tissue(S.attr[i])];
    const Laws<double>& L = T.lawd;
    const double dt = T.P.dt;
    const int32_t pb = T.pbase, NMX = T.nmx, NMY = T.nmy;
    const int32_t j = i - pb, jj = j % NMX, kk = j / NMX;
    auto site = [&](int dj, int dk) {
      int32_t c = jj + dj, w = kk + dk;
      c += c < 0 ? NMX : 0;
      c -= c >= NMX ? NMX : 0;
      w += w < 0 ? NMY : 0;
      w -= w >= NMY ? NMY : 0;
      return pb + w * NMX + c;
    };
    const double4 p = S.pos_cur[i];
    const D3 li = xyz(lam[i]);
    double g_spring = 0.0, g_eps = 0.0, g_bend = 0.0;
    // --- bending: forward recompute of the stencil, then its adjoint
    const double sb = dt * T.P.kbend;
    const D3 yb = sb * li;
    if (T.lattice == kLatticeTriangular) {
      const int32_t nm = T.nmemb;
      D3 o[kTriSlots], ob[kTriSlots];
      o[0] = d3(0.0, 0.0, 0.0);
#pragma unroll
      for (int k = 0; k < 6; ++k) {
        const Vec3<double> v = offset_of<double>(S.pos_cur[pb + tri_link(j, k, NMX, nm)], p, T);
        o[1 + k] = d3(v.x, v.y, v.z);
        const int32_t c2 = tri_link(tri_link(j, (k + 1) % 6, NMX, nm), k, NMX, nm);
        const Vec3<double> w = offset_of<double>(S.pos_cur[pb + c2], p, T);
        o[7 + k] = d3(w.x, w.y, w.z);
      }
#pragma unroll
      for (int s = 0; s < kTriSlots; ++s) ob[s] = d3(0.0, 0.0, 0.0);
      for (int k = 0; k < 6; ++k) {
        const int b = 1 + (k + 1) % 6;
        g_bend += tri1_back(yb, o[1 + k], o[b], o[7 + k], ob[1 + k], ob[b], ob[7 + k]);
      }
      for (int k = 0; k < 6; ++k) {
        const int b = 1 + (k + 1) % 6, c = 1 + (k + 2) % 6;
        g_bend += tri2_back(yb, o[1 + k], o[b], o[c], ob[1 + k], ob[b], ob[c]);
      }
      D3 self = d3(0.0, 0.0, 0.0);
#pragma unroll
      for (int s = 1; s < kTriSlots; ++s) {
        self -= ob[s];
        bend[(int64_t)e * kBendStride + s] = make_double4(ob[s].x, ob[s].y, ob[s].z, 0.0);
      }
      bend[(int64_t)e * kBendStride] = make_double4(self.x, self.y, self.z, 0.0);
    } else {
      D3 o[kSlots];
      o[0] = d3(0.0, 0.0, 0.0);
#pragma unroll
      for (int s = 1; s < kSlots; ++s) {
        const Vec3<double> v = offset_of<double>(S.pos_cur[site(kSlotDj[s], kSlotDk[s])], p, T);
        o[s] = d3(v.x, v.y, v.z);
      }
      const U3 nv = unit3(o[0], o[1]), nvr = unit3(o[1], o[2]);
      const U3 nvl = unit3(o[3], o[0]), nvll = unit3(o[4], o[3]);
      const U3 mv = unit3(o[0], o[5]), mvu = unit3(o[5], o[6]);
      const U3 mvb = unit3(o[7], o[0]), mvbb = unit3(o[8], o[7]);
      const U3 nvbb = unit3(o[8], o[9]), nvbbr = unit3(o[9], o[10]);
      HalfBar hn, hm;
      const double ipnll = dot(nvll.v, nvl.v);
      const double ipmbb = dot(nvbb.v, nvbbr.v);  // memb_bb's ipn (:380)
      const double fn = half_back(yb, nv.v, nvr.v, nvl.v, nvll.v, nv.len, nvl.len, ipnll, hn);
      const double fm = half_back(yb, mv.v, mvu.v, mvb.v, mvbb.v, mv.len, mvb.len, ipmbb, hm);
      g_bend = fn + fm;  // lambda . (dt kbend BCALC): d/ds_bend of the bending term
      D3 ob[kSlots];
#pragma unroll
      for (int s = 0; s < kSlots; ++s) ob[s] = d3(0.0, 0.0, 0.0);
      // ipnll = nvll . nvl
      hn.m += hn.w * nvl.v;
      hn.l += hn.w * nvll.v;
      unit3_back(nv, hn.n, hn.D, ob[0], ob[1]);
      unit3_back(nvr, hn.a, 0.0, ob[1], ob[2]);
      unit3_back(nvl, hn.l, hn.E, ob[3], ob[0]);
      unit3_back(nvll, hn.m, 0.0, ob[4], ob[3]);
      unit3_back(mv, hm.n, hm.D, ob[0], ob[5]);
      unit3_back(mvu, hm.a, 0.0, ob[5], ob[6]);
      unit3_back(mvb, hm.l, hm.E, ob[7], ob[0]);
      unit3_back(mvbb, hm.m, 0.0, ob[8], ob[7]);
      // ipmbb = nvbb . nvbbr
      unit3_back(nvbb, hm.w * nvbbr.v, 0.0, ob[8], ob[9]);
      unit3_back(nvbbr, hm.w * nvbb.v, 0.0, ob[9], ob[10]);
      // o[s] = x_site - x_k: the particle itself receives minus every offset's
      // adjoint (o[0] is the constant zero)
      D3 self = d3(0.0, 0.0, 0.0);
#pragma unroll
      for (int s = 1; s < kSlots; ++s) {
        self -= ob[s];
        bend[(int64_t)e * kBendStride + s] = make_double4(ob[s].x, ob[s].y, ob[s].z, 0.0);
      }
      bend[(int64_t)e * kBendStride] = make_double4(self.x, self.y, self.z, 0.0);
    }
    // --- lattice springs (each pair from both sides: gather)
    D3 mu = d3(0.0, 0.0, 0.0);
    for (int k = 0; k < T.nadj; ++k) {
      const int32_t q = pb + lattice_link(T, j, k);
      const double4 pq = S.pos_cur[q];
      double dx, dy, dz;
      pair_sep(p, pq, i > q, T, dx, dy, dz);
      const D3 d = d3(dx, dy, dz);
      const LawD w = memb_memb_d(L, dist_sq_exact(dx, dy, dz), p.w + pq.w);
      const D3 dl = li - xyz(lam[q]);
      mu += dt * (w.c * dl + (2.0 * w.dc_dr2 * dot(d, dl)) * d);
      const double ld = dot(li, d);
      g_spring += dt * w.c_spring * ld;
      g_eps += dt * w.c_eps * ld;
    }
    // --- wall
    if (p.z < p.w) wall_back(L, dt, p.z, p.w, li.z, mu, g_eps);
    madj[e] = make_double4(mu.x, mu.y, mu.z, 0.0);
    gmemb[e] = make_double4(g_spring, g_eps, g_bend, 0.0);
  }
}

// Every particle: pair adjoint over the exact connections at X_t, plus the
// membrane terms, into lam_out; parameter partials into gpart.
__global__ void __launch_bounds__(256) k_adj_pairs(DevState S, const double4* __restrict__ lam,
                                                   double4* __restrict__ lam_out,
                                                   const double4* __restrict__ bend,
                                                   const double4* __restrict__ madj,
                                                   const double4* __restrict__ gmemb,
                                                   double4* __restrict__ gpart) {
  const int64_t N = S.n_total;
  GRID_STRIDE(i, 0, N) {
    const uint32_t a = S.attr[i];
    const TissueDev& T = S.tissues[attr_tissue(a)];
    const Laws<double>& L = T.lawd;
    const double dt = T.P.dt;
    const double lt2 = T.P.lj_thresh * T.P.lj_thresh;
    const double4 p = S.pos_cur[i];
    const D3 li = xyz(lam[i]);
    D3 mu = li;
    double g_spring = 0.0, g_eps = 0.0, g_bend = 0.0;
    const uint32_t st = attr_state(a);
    int32_t pair_i = -1, dermis_i = -1;
    if (st != ST_MEMB) {
      pair_i = S.pair[i];
      if (st == ST_FIX || st == ST_MUSUME) dermis_i = S.dermis[i];
    }
    const int32_t nc = cand_count(S, i);
    for (int32_t k = 0; k < nc; ++k) {
      const int32_t q = T.pbase + (int32_t)cand_entry(S, i, k + 1);
      const double4 pq = S.pos_cur[q];
      const double dx = pdiff_h(p.x, pq.x, T.lx, T.hlx), dy = pdiff_h(p.y, pq.y, T.ly, T.hly);
      const double dz = p.z - pq.z;
      const double r2 = dist_sq_exact(dx, dy, dz);
      const double rs = __dadd_rn(p.w, pq.w);
      if (!(r2 <= __dmul_rn(__dmul_rn(lt2, rs), rs))) continue;  // connect_proc :115-119
      const uint32_t aq = S.attr[q];
      const uint32_t sq = attr_state(aq);
      const bool both_old = attr_old(a) && attr_old(aq);
      // the laws i applies while iterating q and q applies while iterating i
      LawD w{0.0, 0.0, 0.0, 0.0};
      if (st != ST_MEMB) {
        const int law = law_of(st, (int32_t)i, pair_i, dermis_i, sq, q);
        if (law != L_NONE) w = w + law_d(law, L, r2, rs, both_old, attr_sfm(a));
      }
      if (sq != ST_MEMB) {
        int32_t pair_q = -1, dermis_q = -1;
        if (sq == ST_FIX || sq == ST_MUSUME) {
          pair_q = S.pair[q];
          dermis_q = S.dermis[q];
        }
        const int law = law_of(sq, q, pair_q, dermis_q, st, (int32_t)i);
        if (law != L_NONE) w = w + law_d(law, L, r2, rs, both_old, attr_sfm(aq));
      }
      const D3 d = d3(dx, dy, dz);
      const D3 dl = li - xyz(lam[q]);
      mu += dt * (w.c * dl + (2.0 * w.dc_dr2 * dot(d, dl)) * d);
      const double ld = dot(li, d);
      g_spring += dt * w.c_spring * ld;
      g_eps += dt * w.c_eps * ld;
    }
    // _pair_interaction (:637-641): the spring to the partner, from the
    // higher index's rest length, in the separation of pair_sep
    if (pair_i >= 0) {
      const int32_t q = pair_i;
      const double4 pq = S.pos_cur[q];
      double dx, dy, dz;
      pair_sep(p, pq, i > q, T, dx, dy, dz);
      const D3 d = d3(dx, dy, dz);
      const LawD w = pair_d(L, dist_sq_exact(dx, dy, dz), S.spr[i > q ? i : q]);
      const D3 dl = li - xyz(lam[q]);
      mu += dt * (w.c * dl + (2.0 * w.dc_dr2 * dot(d, dl)) * d);
      g_spring += dt * w.c_spring * dot(li, d);
    }
    if (st == ST_DER && p.z < p.w) wall_back(L, dt, p.z, p.w, li.z, mu, g_eps);
    if (st == ST_MEMB) {
      const int32_t j = (int32_t)i - T.pbase;
      const int32_t e = T.mbase + j;
      const int32_t NMX = T.nmx, NMY = T.nmy, jj = j % NMX, kk = j / NMX;
      mu += xyz(madj[e]);
      const double4 gm = gmemb[e];
      g_spring += gm.x;
      g_eps += gm.y;
      g_bend += gm.z;
      if (T.lattice == kLatticeTriangular) {
        // slot 1 + d names this site for its neighbour in the opposite
        // direction (d + 3) % 6; slot 7 + k (the site two links away, along
        // (k + 1) % 6 then k) for the particle reached back along the
        // opposite directions, (k + 3) % 6 then (k + 4) % 6
        const int32_t nm = T.nmemb;
        mu += xyz(bend[(int64_t)(T.mbase + j) * kBendStride]);
#pragma unroll
        for (int d = 0; d < 6; ++d) {
          const int32_t src = tri_link(j, (d + 3) % 6, NMX, nm);
          mu += xyz(bend[(int64_t)(T.mbase + src) * kBendStride + 1 + d]);
        }
#pragma unroll
        for (int k = 0; k < 6; ++k) {
          const int32_t src = tri_link(tri_link(j, (k + 3) % 6, NMX, nm), (k + 4) % 6, NMX, nm);
          mu += xyz(bend[(int64_t)(T.mbase + src) * kBendStride + 7 + k]);
        }
      } else {
        // bending products naming this site: slot s of the particle at
        // (jj - dj_s, kk - dk_s)
#pragma unroll
        for (int s = 0; s < kSlots; ++s) {
          int32_t c = jj - kSlotDj[s], w = kk - kSlotDk[s];
          c += c < 0 ? NMX : 0;
          c -= c >= NMX ? NMX : 0;
          w += w < 0 ? NMY : 0;
          w -= w >= NMY ? NMY : 0;
          mu += xyz(bend[(int64_t)(T.mbase + w * NMX + c) * kBendStride + s]);
        }
      }
    }
    lam_out[i] = make_double4(mu.x, mu.y, mu.z, 0.0);
    gpart[i] = make_double4(g_spring, g_eps, g_bend, 0.0);
  }
}

// lambda at the last step: dL/dX_T of L_t = inv_cnt[t] sum |X_T - X*|^2 over
// the loss set (minimum image in x and y); the loss terms go to gpart.w.
__global__ void k_adj_seed(DevState S, const double* __restrict__ target, int32_t cells_only,
                           const double* __restrict__ inv_cnt, double4* __restrict__ lam,
                           double4* __restrict__ gpart) {
  const int64_t N = S.n_total;
  GRID_STRIDE(i, 0, N) {
    const uint32_t a = S.attr[i];
    const uint32_t t = attr_tissue(a);
    const TissueDev& T = S.tissues[t];
    const double4 p = S.pos_cur[i];
    const bool in = !(cells_only && attr_state(a) == ST_MEMB);
    const double w = in ? inv_cnt[t] : 0.0;
    const double dx = pdiff(p.x, target[i], T.lx);
    const double dy = pdiff(p.y, target[N + i], T.ly);
    const double dz = p.z - target[2 * N + i];
    lam[i] = make_double4(2.0 * w * dx, 2.0 * w * dy, 2.0 * w * dz, 0.0);
    gpart[i] = make_double4(0.0, 0.0, 0.0, w * (dx * dx + dy * dy + dz * dz));
  }
}

// Per tissue, in a fixed order: acc[4 t + c] += sum over its particles of
// gpart[i].{x, y, z, w}.
__global__ void __launch_bounds__(256) k_tissue_sum(DevState S, const double4* __restrict__ gpart,
                                                    double* __restrict__ acc) {
  __shared__ double4 sh[256];
  for (int32_t t = blockIdx.x; t < S.ntissues; t += gridDim.x) {
    const TissueDev& T = S.tissues[t];
    double4 s = make_double4(0.0, 0.0, 0.0, 0.0);
    for (int32_t k = threadIdx.x; k < T.n; k += blockDim.x) {
      const double4 g = gpart[T.pbase + k];
      s.x += g.x;
      s.y += g.y;
      s.z += g.z;
      s.w += g.w;
    }
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
      if ((int)threadIdx.x < h) {
        const double4 o = sh[threadIdx.x + h];
        sh[threadIdx.x].x += o.x;
        sh[threadIdx.x].y += o.y;
        sh[threadIdx.x].z += o.z;
        sh[threadIdx.x].w += o.w;
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      acc[4 * t + 0] += sh[0].x;
      acc[4 * t + 1] += sh[0].y;
      acc[4 * t + 2] += sh[0].z;
      acc[4 * t + 3] += sh[0].w;
    }
    __syncthreads();
  }
}

// Flags the tissues whose particles moved more than skin/2 from the
// positions of their last candidate rebuild (the forward step's test, for
// positions loaded from a checkpoint or a stored step).
__global__ void k_gate_check(DevState S) {
  GRID_STRIDE(i, 0, S.n_total) {
    const uint32_t t = attr_tissue(S.attr[i]);
    const TissueDev& T = S.tissues[t];
    const double4 p = S.pos_cur[i];
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

}  // namespace

void launch_gate_check(const DevState& S, const LaunchCfg& lc, cudaStream_t s) {
  if (S.n_total > 0)
    k_gate_check<<<stride_blocks(S.n_total, lc.block, lc), lc.block, 0, s>>>(S);
}

void launch_adjoint_seed(const DevState& S, const double* target, int32_t cells_only,
                         const double* inv_cnt, double4* lam, double4* gpart,
                         const LaunchCfg& lc, cudaStream_t s) {
  if (S.n_total > 0)
    k_adj_seed<<<stride_blocks(S.n_total, lc.block, lc), lc.block, 0, s>>>(
        S, target, cells_only, inv_cnt, lam, gpart);
}

void launch_adjoint_step(const DevState& S, const AdjointBuffers& B, const LaunchCfg& lc,
                         cudaStream_t s) {
  if (S.nprep_memb > 0)
    k_adj_memb<<<stride_blocks(S.nprep_memb, 256, lc), 256, 0, s>>>(S, B.lam_in, B.bend, B.madj,
                                                                     B.gmemb);
  if (S.n_total > 0)
    k_adj_pairs<<<blocks_for(S.n_total, 256), 256, 0, s>>>(S, B.lam_in, B.lam_out, B.bend, B.madj,
                                                           B.gmemb, B.gpart);
}

void launch_tissue_sum(const DevState& S, const double4* gpart, double* acc, const LaunchCfg& lc,
                       cudaStream_t s) {
  const int grid = S.ntissues < lc.num_sms * 8 ? S.ntissues : lc.num_sms * 8;
  if (grid > 0) k_tissue_sum<<<grid, 256, 0, s>>>(S, gpart, acc);
}

}  // namespace epi
