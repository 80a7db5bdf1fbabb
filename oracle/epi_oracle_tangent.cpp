// Forward-mode FP64 gradient of the mechanics step (TEST INFRASTRUCTURE).
//
// The reference gradient the GPU adjoint is checked against. It re-states the
// step of epi_oracle.c -- cell_interaction's membrane bending, membrane
// springs, wall and CI_al_air_de_to_al_air_de_fix_mu pairs
// (epi5_MT/cell_interaction.cpp:48-66, 103-152, 185-234, 287-449, 529-579),
// pos_copy and cell_pos_periodic_fix (epi5_MT/cellmanager.cpp:19-26,
// 395-414) -- as a template over the number type, in the same visiting order
// and with the same expressions. Instantiated with `double` it is the
// oracle's step (the tests require bit-identical positions); instantiated with
// a dual number carrying three tangents it propagates, alongside every value,
// its derivative with respect to three multipliers of the force constants:
//   s_spring  -- der_der_const, k_total, k_desmosome, kspring, kspring_d,
//                kspring_division (every spring constant),
//   s_eps     -- eps_m (the Lennard-Jones depth),
//   s_bend    -- kbend.
// The connection lists of every step come from epi_oracle.c's connect_cell
// applied to the value part. No hand-derived derivative appears here: the
// dual arithmetic differentiates the restated step itself, which makes this
// an independent check of a hand-written reverse-mode adjoint.
//
// Scope: square or triangular membranes (the triangular bending of
// tri_memb_bend, :451-508, restated from epi_oracle.c) and every cell state
// of the path: DER (CI_der_to_der and the wall), FIX and MUSUME (the
// dermis springs, CI_fix_mu_to_fix_mu), ALIVE / DEAD / AIR, and the pair
// springs of dividing cells (:129-183, 281-285, 549-641). The dermis of each
// step comes from epi_oracle.c's connect, like the lists.
#include "epi_oracle.h"

#include <cmath>
#include <cstring>
#include <vector>

namespace {

constexpr int kDir = 3;  // s_spring, s_eps, s_bend

struct Dual {
  double v;
  double d[kDir];
  Dual() : v(0), d{0, 0, 0} {}
  Dual(double x) : v(x), d{0, 0, 0} {}  // NOLINT: constants promote
};

inline Dual operator+(const Dual& a, const Dual& b) {
  Dual r(a.v + b.v);
  for (int k = 0; k < kDir; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
inline Dual operator-(const Dual& a, const Dual& b) {
  Dual r(a.v - b.v);
  for (int k = 0; k < kDir; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
inline Dual operator-(const Dual& a) {
  Dual r(-a.v);
  for (int k = 0; k < kDir; ++k) r.d[k] = -a.d[k];
  return r;
}
inline Dual operator*(const Dual& a, const Dual& b) {
  Dual r(a.v * b.v);
  for (int k = 0; k < kDir; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
inline Dual operator/(const Dual& a, const Dual& b) {
  Dual r(a.v / b.v);
  for (int k = 0; k < kDir; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) / b.v;
  return r;
}
inline Dual& operator+=(Dual& a, const Dual& b) { return a = a + b; }
inline Dual& operator-=(Dual& a, const Dual& b) { return a = a - b; }
inline Dual sqrt(const Dual& a) {
  Dual r(std::sqrt(a.v));
  for (int k = 0; k < kDir; ++k) r.d[k] = a.d[k] / (2.0 * r.v);
  return r;
}
inline double val(const Dual& a) { return a.v; }
inline double val(double a) { return a; }
using std::sqrt;

enum { S_ALIVE = 0, S_DEAD = 1, S_FIX = 4, S_DER = 6, S_MUSUME = 7, S_AIR = 8, S_MEMB = 9 };
inline bool is_aad(uint8_t s) { return s == S_ALIVE || s == S_AIR || s == S_DEAD; }

template <class T>
inline T pow6(const T& v) { return v * v * v * v * v * v; }
template <class T>
inline T pow3(const T& v) { return v * v * v; }

// Force constants; the three scaled families are T, the rest plain doubles.
template <class T>
struct Consts {
  double dt, p_memb, lj_thresh, thresh_sp, delta_r, para_ljp2;
  T eps_m, der_der_const, k_total, k_desmosome, kbend, kspring, kspring_d, kspring_division;
};

// vec3 (vec3.h:5-54) over T, operation by operation as epi_oracle.c's v3
template <class T>
struct V3 {
  T x, y, z;
};
template <class T>
inline V3<T> v3_cross(const V3<T>& a, const V3<T>& b) {
  return V3<T>{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class T>
inline T v3_dot(const V3<T>& a, const V3<T>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class T>
inline T v3_norm(const V3<T>& a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
template <class T>
inline V3<T> v3_normalize(V3<T>* a) {  // in place, like vec3::normalize
  const T nm = v3_norm(*a);
  a->x = a->x / nm;
  a->y = a->y / nm;
  a->z = a->z / nm;
  return *a;
}
template <class T>
inline V3<T> v3_scale(const T& c, const V3<T>& a) { return V3<T>{c * a.x, c * a.y, c * a.z}; }
template <class T>
inline V3<T> v3_div(const V3<T>& a, const T& c) { return V3<T>{a.x / c, a.y / c, a.z / c}; }
template <class T>
inline V3<T> v3_add(const V3<T>& a, const V3<T>& b) { return V3<T>{a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class T>
inline V3<T> v3_sub(const V3<T>& a, const V3<T>& b) { return V3<T>{a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class T>
inline V3<T> tri_rho(const V3<T>& n1, const V3<T>& b1) {  // :470-472
  return v3_sub(b1, v3_scale(v3_dot(n1, b1), n1));
}

template <class T>
struct Tissue {
  int32_t n, nmemb, nmx, nmy, nadj = 4;
  bool tri = false;
  std::vector<int32_t> tri_nb;  // Memb_data::memb[6] per membrane particle
  double lx, ly;
  Consts<T> P;
  std::vector<T> x, y, z, nx, ny, nz;
  std::vector<double> radius, agek, spr;
  std::vector<uint8_t> state;
  std::vector<int32_t> pair, rest_div, dermis;
  std::vector<T> sfm;  // spring_force_to_memb of each MUSUME
  std::vector<int32_t> lat_l, lat_ll, lat_r, lat_b, lat_bb, lat_u;
  std::vector<T> nv, mv, dn, dm, ipn, ipm;
  std::vector<int32_t> off, idx;  // connection lists, the reference's push order

  // utils.h:25-46
  T pdx(const T& a, const T& b) const {
    const T d = a - b;
    if (val(d) > 0.5 * lx) return d - lx;
    if (val(d) <= -0.5 * lx) return d + lx;
    return d;
  }
  T pdy(const T& a, const T& b) const {
    const T d = a - b;
    if (val(d) > 0.5 * ly) return d - ly;
    if (val(d) <= -0.5 * ly) return d + ly;
    return d;
  }
  T dist_sq(int32_t a, int32_t b) const {
    const T dx = pdx(x[a], x[b]);
    const T dy = pdy(y[a], y[b]);
    const T dz = z[a] - z[b];
    return dx * dx + dy * dy + dz * dz;
  }
  // ljmain, is_near, adhesion, CI_al_air_de_to_al_air_de_fix_mu (:103-152)
  T ljmain(int32_t a, int32_t b) const {
    const T d2 = dist_sq(a, b);
    const double rs = radius[a] + radius[b];
    const T lj6 = pow6(rs) / pow3(d2);
    return 4.0 * P.eps_m * lj6 * (lj6 - 1) / d2;
  }
  bool is_near(int32_t a, int32_t b) const {
    return val(dist_sq(a, b)) < (radius[a] + radius[b]) * (radius[a] + radius[b]);
  }
  T adhesion(int32_t a, int32_t b, const T& k) const {
    const double lt = P.lj_thresh;
    const T distlj = sqrt(dist_sq(a, b));
    const double rs = radius[a] + radius[b];
    const T m1 = (distlj / rs) - 1;
    return (val(m1 + 1) > lt ? T(0.0)
                             : -(k / distlj) * m1 * (1 - m1 * m1 / ((lt - 1.0) * (lt - 1.0))));
  }
  T ci_aad(int32_t a, int32_t b) const {
    if (is_near(a, b)) return ljmain(a, b);
    T spf = P.k_desmosome;
    if (agek[a] > P.thresh_sp && agek[b] > P.thresh_sp) spf = P.k_total;
    return adhesion(a, b, spf);
  }
  // CI_der_to_der, :129-139
  T ci_der_to_der(int32_t a, int32_t b) const {
    const double rs = radius[a] + radius[b];
    if (val(sqrt(dist_sq(a, b)) + P.delta_r) < rs) {
      const T dist = sqrt(dist_sq(a, b));
      const T dist2 = dist + P.delta_r;
      const T lj6 = pow6(rs) / pow6(dist2);
      return 4.0 * P.eps_m * lj6 * (lj6 - 1) / (dist * dist2) + P.para_ljp2;
    } else if (is_near(a, b)) {
      return T(P.para_ljp2);
    }
    const T dist = sqrt(dist_sq(a, b));
    const T dist2 = dist + P.delta_r;
    const T lj6 = pow6(rs) / pow6(dist2);
    return 4.0 * P.eps_m * lj6 * (lj6 - 1) / (dist * dist) + P.para_ljp2;
  }
  // CI_fix_mu_to_fix_mu, :154-162
  T ci_fixmu(int32_t a, int32_t b) const {
    if (is_near(a, b)) return ljmain(a, b);
    return adhesion(a, b, P.k_desmosome);
  }
  // CI_mu_to_memb, :164-172
  T ci_mu_memb(int32_t a, int32_t b) const {
    if (is_near(a, b)) return ljmain(a, b);
    return adhesion(a, b, sfm[a]);
  }
  // CI_fix_to_memb, :174-183
  T ci_fix_memb(int32_t a, int32_t b) const {
    if (is_near(a, b)) return ljmain(a, b);
    const T distlj = sqrt(dist_sq(a, b));
    const T lj2 = distlj / (radius[a] + radius[b]);
    return -(P.kspring / distlj) * (lj2 - 1.0);
  }
  // CI_pair, :281-285
  T ci_pair(int32_t a, int32_t b) const {
    const T dist = sqrt(dist_sq(a, b));
    const T force = P.kspring_division * (dist - spr[a]);
    return -force / dist;
  }
  // CI_memb_to_memb, :185-234
  T ci_memb_memb(int32_t a, int32_t b) const {
    const double Pm = P.p_memb;
    const double rs = radius[a] + radius[b];
    const double rs2 = rs * rs;
    double cr2;
    const T d2 = dist_sq(a, b);
    if (val(d2) < (cr2 = rs2 * Pm * Pm)) {
      const T lj6 = pow3(cr2) / pow3(d2);
      return 4.0 * P.eps_m * lj6 * (lj6 - 1) / d2;
    } else if (val(d2) < rs2) {
      const T distlj = sqrt(d2);
      const double cr = rs * Pm;
      return -(P.der_der_const / distlj) * (distlj / cr - 1.0);
    }
    const T distlj = sqrt(d2);
    const double lambda = (1.0 + Pm) * rs;
    const double cr = rs * Pm;
    const T lj6 = pow6(cr) / pow6(lambda - distlj);
    return -(P.der_der_const / rs) * ((1.0 - Pm) / Pm) -
           4 * P.eps_m * (lj6 * (lj6 - 1.0)) / ((lambda - distlj) * distlj);
  }
  // cell_interaction_apply, :48-66
  void apply(int32_t c1, int32_t c2, const T& coef) {
    const T dumx = P.dt * coef * pdx(x[c1], x[c2]);
    const T dumy = P.dt * coef * pdy(y[c1], y[c2]);
    const T dumz = P.dt * coef * (z[c1] - z[c2]);
    nx[c1] += dumx;
    ny[c1] += dumy;
    nz[c1] += dumz;
    nx[c2] -= dumx;
    ny[c2] -= dumy;
    nz[c2] -= dumz;
  }
  // wall_interaction, :287-294
  void wall(int32_t c) {
    const T distlj = 2.0 * z[c];
    const T lj6 = pow6(radius[c]) / pow6(z[c]);
    const T ljm = 4.0 * P.eps_m * lj6 * (lj6 - 1.0) / (distlj * distlj);
    nz[c] += P.dt * ljm * 2.0 * z[c];
  }
  // _memb_bend_calc1..3, :296-449
  void bend_calc1(int32_t m) {
    const int32_t r = lat_r[m], u = lat_u[m];
    const T dnv = sqrt(dist_sq(r, m));
    nv[3 * m + 0] = pdx(x[r], x[m]) / dnv;
    nv[3 * m + 1] = pdy(y[r], y[m]) / dnv;
    nv[3 * m + 2] = (z[r] - z[m]) / dnv;
    dn[m] = dnv;
    const T dmv = sqrt(dist_sq(u, m));
    mv[3 * m + 0] = pdx(x[u], x[m]) / dmv;
    mv[3 * m + 1] = pdy(y[u], y[m]) / dmv;
    mv[3 * m + 2] = (z[u] - z[m]) / dmv;
    dm[m] = dmv;
  }
  void bend_calc2(int32_t m) {
    const int32_t r = lat_r[m], u = lat_u[m];
    ipn[m] = nv[3 * m] * nv[3 * r] + nv[3 * m + 1] * nv[3 * r + 1] + nv[3 * m + 2] * nv[3 * r + 2];
    ipm[m] = mv[3 * m] * mv[3 * u] + mv[3 * m + 1] * mv[3 * u + 1] + mv[3 * m + 2] * mv[3 * u + 2];
  }
  static T bend_factor(const T& c) {
    if (val(c) >= 0) return (1.0 - c);
    return 1.0 / ((1.0 + c) * (1.0 + c));
  }
  void bend_calc3(int32_t m) {
    const int32_t r = lat_r[m], l = lat_l[m], ll = lat_ll[m];
    const int32_t u = lat_u[m], b = lat_b[m], bb = lat_bb[m];
    const T* nvr = &nv[3 * r];
    const T* nvl = &nv[3 * l];
    const T* nvll = &nv[3 * ll];
    const T ipnl = ipn[l], ipnll = ipn[ll];
    const T* mvu = &mv[3 * u];
    const T* mvb = &mv[3 * b];
    const T* mvbb = &mv[3 * bb];
    const T ipmb = ipm[b];
    const T ipmbb = ipn[bb];  // the reference reads ipn here (:380)
    const T dnl = dn[l], dmb = dm[b];
    const T dnm = dn[m], dmm = dm[m];
    const T* nvm = &nv[3 * m];
    const T* mvm = &mv[3 * m];
    const T ipnm = ipn[m], ipmm = ipm[m];
    T f[3];
    for (int k = 0; k < 3; ++k) {
      f[k] = -(bend_factor(ipnm)) * (nvr[k] - ipnm * nvm[k]) / dnm +
             bend_factor(ipnl) * ((nvm[k] - ipnl * nvl[k]) / dnl - (nvl[k] - ipnl * nvm[k]) / dnm) +
             bend_factor(ipnll) * (nvll[k] - ipnll * nvl[k]) / dnl -
             bend_factor(ipmm) * (mvu[k] - ipmm * mvm[k]) / dmm +
             bend_factor(ipmb) * ((mvm[k] - ipmb * mvb[k]) / dmb - (mvb[k] - ipmb * mvm[k]) / dmm) +
             bend_factor(ipmbb) * (mvbb[k] - ipmbb * mvb[k]) / dmb;
    }
    const T s = P.dt * P.kbend;
    nx[m] += s * f[0];
    ny[m] += s * f[1];
    nz[m] += s * f[2];
  }

  // tri_bend_1 / tri_bend_2 / tri_memb_bend, :475-508 (the division by the
  // norm of the already normalised normal kept, as in the reference)
  V3<T> vpos(int32_t c) const { return V3<T>{x[c], y[c], z[c]}; }
  V3<T> vpsub(const V3<T>& a, const V3<T>& b) const {
    return V3<T>{pdx(a.x, b.x), pdy(a.y, b.y), a.z - b.z};
  }
  V3<T> tri_bend_1(int32_t r1, int32_t a1, int32_t b1, int32_t c1) const {
    const V3<T> r1v = vpos(r1), a1v = vpos(a1), b1v = vpos(b1), c1v = vpos(c1);
    V3<T> norm1_pre = v3_cross(vpsub(r1v, b1v), vpsub(a1v, b1v));
    const V3<T> norm1 = v3_normalize(&norm1_pre);
    V3<T> n2 = v3_cross(vpsub(a1v, b1v), vpsub(c1v, b1v));
    const V3<T> norm2 = v3_normalize(&n2);
    const T dot1 = v3_dot(norm1, norm2);
    return v3_scale(bend_factor(dot1),
                    v3_div(v3_cross(vpsub(a1v, b1v), tri_rho(norm1, norm2)), v3_norm(norm1_pre)));
  }
  V3<T> tri_bend_2(int32_t r1, int32_t a1, int32_t b1, int32_t c1) const {
    const V3<T> r1v = vpos(r1), a1v = vpos(a1), b1v = vpos(b1), c1v = vpos(c1);
    V3<T> norm1_pre = v3_cross(vpsub(r1v, c1v), vpsub(b1v, c1v));
    V3<T> norm2_pre = v3_cross(vpsub(r1v, b1v), vpsub(a1v, b1v));
    const V3<T> norm1 = v3_normalize(&norm1_pre), norm2 = v3_normalize(&norm2_pre);
    const T dot1 = v3_dot(norm1, norm2);
    return v3_scale(bend_factor(dot1),
                    v3_add(v3_div(v3_cross(vpsub(b1v, c1v), tri_rho(norm1, norm2)),
                                  v3_norm(norm1_pre)),
                           v3_div(v3_cross(vpsub(a1v, b1v), tri_rho(norm2, norm1)),
                                  v3_norm(norm2_pre))));
  }
  void tri_memb_bend(int32_t m) {
    const int32_t* nb = &tri_nb[6 * (size_t)m];
    V3<T> dr{T(0.0), T(0.0), T(0.0)};
    for (int i = 0; i < 6; ++i) {
      const int32_t b = nb[(i + 1) % 6];
      dr = v3_add(dr, tri_bend_1(m, nb[i], b, tri_nb[6 * (size_t)b + i]));
    }
    for (int i = 0; i < 6; ++i) dr = v3_add(dr, tri_bend_2(m, nb[i], nb[(i + 1) % 6], nb[(i + 2) % 6]));
    nx[m] += P.dt * P.kbend * dr.x;
    ny[m] += P.dt * P.kbend * dr.y;
    nz[m] += P.dt * P.kbend * dr.z;
  }

  // cell_interaction, :648-685, for membrane and ALIVE / DEAD / AIR cells
  void interact() {
    if (tri) {
      for (int32_t m = 0; m < nmemb; ++m) tri_memb_bend(m);
    } else {
      for (int32_t m = 0; m < nmemb; ++m) bend_calc1(m);
      for (int32_t m = 0; m < nmemb; ++m) bend_calc2(m);
      for (int32_t m = 0; m < nmemb; ++m) bend_calc3(m);
    }
    for (int32_t m = 0; m < nmemb; ++m) {  // _MEMB_interaction, :529-547
      if (val(z[m]) < radius[m]) wall(m);
      for (int32_t i = 0; i < nadj; ++i) {
        const int32_t o = idx[off[m] + i];
        if (state[o] == S_MEMB && m > o) apply(m, o, ci_memb_memb(m, o));
      }
    }
    for (int32_t c = nmemb; c < n; ++c) {
      const uint8_t sc = state[c];
      if (sc == S_DER) {  // _DER_interaction, :549-561
        if (val(z[c]) < radius[c]) wall(c);
        for (int32_t k = off[c]; k < off[c + 1]; ++k) {
          const int32_t o = idx[k];
          if (state[o] == S_DER && c > o)
            apply(c, o, ci_der_to_der(c, o));
          else
            apply(c, o, ljmain(c, o));
        }
      } else if (sc == S_FIX) {  // _FIX_interaction, :581-604
        for (int32_t k = off[c]; k < off[c + 1]; ++k) {
          const int32_t o = idx[k];
          const uint8_t so = state[o];
          if (so == S_FIX) {
            if (pair[c] != o && c > o) apply(c, o, ci_fixmu(c, o));
          } else if (so == S_MUSUME) {
            if (pair[c] != o) apply(c, o, ci_fixmu(c, o));
          } else if (so == S_MEMB) {
            if (dermis[c] == o)
              apply(c, o, ci_fix_memb(c, o));
            else
              apply(c, o, ljmain(c, o));
          }
        }
      } else if (sc == S_MUSUME) {  // _MUSUME_interaction, :613-634
        sfm[c] = T(0.0);
        if (pair[c] >= 0 && state[pair[c]] == S_FIX)
          sfm[c] = P.kspring;
        else if (rest_div[c] > 0)
          sfm[c] = P.kspring_d;
        for (int32_t k = off[c]; k < off[c + 1]; ++k) {
          const int32_t o = idx[k];
          const uint8_t so = state[o];
          if (so == S_MEMB) {
            if (dermis[c] == o)
              apply(c, o, ci_mu_memb(c, o));
            else
              apply(c, o, ljmain(c, o));
          } else if (so == S_MUSUME && pair[c] != o && c > o) {
            apply(c, o, ci_fixmu(c, o));
          }
        }
      } else if (is_aad(sc)) {  // _AL_AIR_DE_interaction, :563-579
        for (int32_t k = off[c]; k < off[c + 1]; ++k) {
          const int32_t o = idx[k];
          const uint8_t so = state[o];
          if (is_aad(so)) {
            if (c > o) apply(c, o, ci_aad(c, o));
          } else if (so != S_DER) {
            apply(c, o, ci_aad(c, o));
          }
        }
      }
      // _pair_interaction, :637-641
      if (pair[c] >= 0 && c > pair[c]) apply(c, pair[c], ci_pair(c, pair[c]));
    }
  }
  // pos_copy + cell_pos_periodic_fix (cellmanager.cpp:19-26, 395-414)
  void commit() {
    for (int32_t c = 0; c < n; ++c) {
      x[c] = nx[c];
      y[c] = ny[c];
      z[c] = nz[c];
    }
    for (int32_t c = 0; c < n; ++c) {
      if (val(nx[c]) > lx) x[c] = nx[c] = nx[c] - lx;
      else if (val(nx[c]) < 0) x[c] = nx[c] = nx[c] + lx;
      if (val(ny[c]) > ly) y[c] = ny[c] = ny[c] - ly;
      else if (val(ny[c]) < 0) y[c] = ny[c] = ny[c] + ly;
    }
  }
};

template <class T>
T scaled(double v, int dir);
template <>
double scaled<double>(double v, int) { return v; }
template <>
Dual scaled<Dual>(double v, int dir) {
  Dual r(v);
  r.d[dir] = v;  // d(s * v)/ds at s = 1
  return r;
}

// Runs nsteps steps of the restated mechanics on tissue `o` (whose connect
// supplies the lists). Outputs the final positions' value parts and, for
// T = Dual, the loss and its gradient.
template <class T>
int run(ora_tissue* o, int32_t n, int32_t nmemb, int32_t nmx, int32_t nmy, double lx, double ly,
        const ora_params& p, const double* x, const double* y, const double* z,
        const double* radius, const double* agek, const double* spr, const uint8_t* state,
        const int32_t* pair, const int32_t* rest_div, int32_t nsteps, const double* tx,
        const double* ty, const double* tz, int32_t cells_only, T* loss, double* ox, double* oy,
        double* oz) {
  Tissue<T> t;
  t.n = n; t.nmemb = nmemb; t.nmx = nmx; t.nmy = nmy; t.lx = lx; t.ly = ly;
  t.P.dt = p.dt; t.P.p_memb = p.p_memb; t.P.lj_thresh = p.lj_thresh; t.P.thresh_sp = p.thresh_sp;
  t.P.der_der_const = scaled<T>(p.der_der_const, 0);
  t.P.k_total = scaled<T>(p.k_total, 0);
  t.P.k_desmosome = scaled<T>(p.k_desmosome, 0);
  t.P.eps_m = scaled<T>(p.eps_m, 1);
  t.P.kbend = scaled<T>(p.kbend, 2);
  t.P.kspring = scaled<T>(p.kspring, 0);
  t.P.kspring_d = scaled<T>(p.kspring_d, 0);
  t.P.kspring_division = scaled<T>(p.kspring_division, 0);
  t.P.delta_r = p.delta_r;
  t.P.para_ljp2 = p.para_ljp2;
  t.x.assign(x, x + n); t.y.assign(y, y + n); t.z.assign(z, z + n);
  t.nx = t.x; t.ny = t.y; t.nz = t.z;
  t.radius.assign(radius, radius + n);
  t.agek.assign(agek, agek + n);
  t.state.assign(state, state + n);
  t.spr.assign(spr, spr + n);
  t.pair.assign((size_t)n, -1);
  if (pair) t.pair.assign(pair, pair + n);
  t.rest_div.assign((size_t)n, 0);
  if (rest_div) t.rest_div.assign(rest_div, rest_div + n);
  t.dermis.assign((size_t)n, -1);
  t.sfm.assign((size_t)n, T(0.0));
  t.nv.assign(3 * (size_t)nmemb, T(0.0)); t.mv = t.nv;
  t.dn.assign(nmemb, T(0.0)); t.dm = t.dn; t.ipn = t.dn; t.ipm = t.dn;
  t.lat_l.resize(nmemb); t.lat_ll.resize(nmemb); t.lat_r.resize(nmemb);
  t.lat_b.resize(nmemb); t.lat_bb.resize(nmemb); t.lat_u.resize(nmemb);
  t.tri_nb.assign(6 * (size_t)nmemb, 0);
  if (nmemb > 0 && ora_get_tri_neighbours(o, t.tri_nb.data()) == 0) {
    t.tri = true;  // TRI_MEMB: six lattice links, tri_memb_bend
    t.nadj = 6;
  }
  for (int32_t j = 0; j < nmemb; ++j) {  // _memb_init square branch, cellmanager.cpp:114-158
    const int32_t jj = j % nmx, kk = j / nmx;
    t.lat_l[j] = jj == 0 ? j + nmx - 1 : j - 1;
    t.lat_ll[j] = jj <= 1 ? j + nmx - 2 : j - 2;
    t.lat_r[j] = jj == nmx - 1 ? j - (nmx - 1) : j + 1;
    t.lat_b[j] = kk == 0 ? j + nmx * nmy - nmx : j - nmx;
    t.lat_bb[j] = kk <= 1 ? j + nmx * nmy - 2 * nmx : j - 2 * nmx;
    t.lat_u[j] = kk == nmy - 1 ? j - (nmx * nmy - nmx) : j + nmx;
  }
  std::vector<double> vx(n), vy(n), vz(n);
  auto fetch_lists = [&]() {
    t.off.assign((size_t)n + 1, 0);
    const int64_t tot = ora_get_connections_raw(o, t.off.data(), nullptr, 0);
    t.idx.assign((size_t)(tot > 0 ? tot : 1), 0);
    ora_get_connections_raw(o, t.off.data(), t.idx.data(), tot);
    ora_get_dermis(o, t.dermis.data());
  };
  fetch_lists();
  for (int32_t s = 0; s < nsteps; ++s) {
    t.interact();
    t.commit();
    for (int32_t c = 0; c < n; ++c) {
      vx[c] = val(t.x[c]);
      vy[c] = val(t.y[c]);
      vz[c] = val(t.z[c]);
      if (!std::isfinite(vx[c]) || !std::isfinite(vy[c]) || !std::isfinite(vz[c]))
        return ORA_ERR_NONFINITE;
    }
    ora_set_positions(o, vx.data(), vy.data(), vz.data());
    const int rc = ora_connect(o);
    if (rc != ORA_OK) return rc;
    fetch_lists();
  }
  for (int32_t c = 0; c < n; ++c) {
    ox[c] = val(t.x[c]);
    oy[c] = val(t.y[c]);
    oz[c] = val(t.z[c]);
  }
  if (tx && loss) {
    // mean over the loss set of the squared minimum-image distance to the target
    T sum(0.0);
    int32_t cnt = 0;
    for (int32_t c = cells_only ? nmemb : 0; c < n; ++c) {
      const T dx = t.pdx(t.x[c], T(tx[c]));
      const T dy = t.pdy(t.y[c], T(ty[c]));
      const T dz = t.z[c] - tz[c];
      sum += dx * dx + dy * dy + dz * dz;
      ++cnt;
    }
    *loss = cnt > 0 ? sum / (double)cnt : T(0.0);
  }
  return ORA_OK;
}

}  // namespace

extern "C" int ora_tangent_gradient(
    int32_t n, int32_t nmemb, int32_t nder, int32_t nmx, int32_t nmy, double lx, double ly,
    double lz, const double* params14, const double* x, const double* y, const double* z,
    const double* radius, const double* agek, const double* spr_nat_len, const uint8_t* state,
    const int32_t* pair, const int32_t* rest_div_times, int32_t lattice, int32_t nsteps,
    const double* tx, const double* ty, const double* tz, int32_t cells_only, int32_t use_dual,
    double* loss, double* grad3, double* out_x, double* out_y, double* out_z) {
  if (n <= 0 || nsteps < 0 || !params14) return ORA_ERR_INVALID_ARG;
  for (int32_t i = 0; i < n; ++i)
    if ((i < nmemb) != (state[i] == S_MEMB)) return ORA_ERR_INVALID_ARG;
  ora_tissue* o = ora_new_lattice(n, nmemb, nder, nmx, nmy, lx, ly, lz, params14, x, y, z,
                                  radius, agek, spr_nat_len, state, pair, rest_div_times, lattice);
  if (!o) return ORA_ERR_INVALID_ARG;
  ora_params p;
  std::memcpy(&p, params14, sizeof(p));
  int rc;
  if (use_dual) {
    Dual L;
    rc = run<Dual>(o, n, nmemb, nmx, nmy, lx, ly, p, x, y, z, radius, agek, spr_nat_len, state,
                   pair, rest_div_times, nsteps, tx, ty, tz, cells_only, &L, out_x, out_y, out_z);
    if (rc == ORA_OK && loss) *loss = L.v;
    if (rc == ORA_OK && grad3)
      for (int k = 0; k < kDir; ++k) grad3[k] = L.d[k];
  } else {
    double L = 0;
    rc = run<double>(o, n, nmemb, nmx, nmy, lx, ly, p, x, y, z, radius, agek, spr_nat_len, state,
                     pair, rest_div_times, nsteps, tx, ty, tz, cells_only, &L, out_x, out_y,
                     out_z);
    if (rc == ORA_OK && loss) *loss = L;
  }
  ora_free(o);
  return rc;
}
