/* CPU restatement of the epi5_MT cell-mechanics step (TEST INFRASTRUCTURE).
 *
 * Oracle only: see epi_oracle.h. Every function cites the reference code it
 * restates (paths relative to the reference checkout, epi5_MT/ unless noted).
 * Compile with -ffp-contract=off: the reference's arithmetic is evaluated
 * operation by operation, left to right, and fused multiply-adds would change
 * the rounding.
 */
#include "epi_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

enum { S_ALIVE = 0, S_DEAD = 1, S_FIX = 4, S_DER = 6, S_MUSUME = 7, S_AIR = 8, S_MEMB = 9 };

#define AREA_GRID_ORIGINAL 2.0          /* cell_connection.cpp:16 */
#define AREA_GRID (AREA_GRID_ORIGINAL + 1e-7) /* cell_connection.cpp:19 */
#define BIN_CAP 200                     /* N3, cell_connection.cpp:28 */
#define CONN_CAP 400                    /* N2 / MAX_CONNECT_CELL_NUM, define.h:80 */
#define MEMB_ADJ_SQUARE 4               /* MEMB_ADJ_CONN_NUM, define.h:147-153 */
#define MEMB_ADJ_TRI 6

struct ora_tissue {
  int32_t n, nmemb, nder, nmx, nmy;
  int32_t tri;   /* triangular membrane (TRI_MEMB, define.h:66) */
  int32_t nadj;  /* MEMB_ADJ_CONN_NUM: 4 square, 6 triangular */
  double lx, ly, lz;
  int32_t anx, any, anz;
  ora_params P;
  double *x, *y, *z;    /* current value  (dual_double::d1, DualValue.h:17-26) */
  double *nx, *ny, *nz; /* next value     (dual_double::d2, DualValue.h:28-38) */
  double *radius, *agek, *spr, *sfm;
  uint8_t* state;
  int32_t *pair, *rest_div, *dermis;
  int32_t* conn;        /* n x CONN_CAP, push order (Lockfree_push_stack) */
  int32_t* nconn;
  int32_t *lat_l, *lat_ll, *lat_r, *lat_b, *lat_bb, *lat_u;
  int32_t* tri_nb; /* Memb_data::memb[6] per membrane particle (cell.h:57-59) */
  double *nv, *mv, *dn, *dm, *ipn, *ipm; /* Memb_data scratch, cell.h:60-62 */
  int32_t* bin_cnt;
  int32_t* bin_list;
  int err;
  int32_t err_a, err_b;
  double err_v;
};

/* utils.h:25-46 */
static inline double pdx(const ora_tissue* t, double a, double b) {
  const double d = a - b;
  if (d > 0.5 * t->lx) return d - t->lx;
  if (d <= -0.5 * t->lx) return d + t->lx;
  return d;
}
static inline double pdy(const ora_tissue* t, double a, double b) {
  const double d = a - b;
  if (d > 0.5 * t->ly) return d - t->ly;
  if (d <= -0.5 * t->ly) return d + t->ly;
  return d;
}
/* p_cell_dist_sq(c1, c2), cell.h:287-290 / utils.h:48-53 */
static inline double dist_sq(const ora_tissue* t, int32_t a, int32_t b) {
  const double dx = pdx(t, t->x[a], t->x[b]);
  const double dy = pdy(t, t->y[a], t->y[b]);
  const double dz = t->z[a] - t->z[b];
  return dx * dx + dy * dy + dz * dz;
}
static inline double min0(double a) { return a > 0 ? a : 0; } /* utils.h:55-57 */
#define POW6(v) ((v) * (v) * (v) * (v) * (v) * (v)) /* cell_interaction.cpp:15 */
#define POW3(v) ((v) * (v) * (v))                   /* cell_interaction.cpp:16 */

static void set_err(ora_tissue* t, int code, int32_t a, int32_t b, double v) {
  if (t->err == ORA_OK) {
    t->err = code;
    t->err_a = a;
    t->err_b = b;
    t->err_v = v;
  }
}

static int push_conn(ora_tissue* t, int32_t c, int32_t o) {
  if (t->nconn[c] >= CONN_CAP) {
    set_err(t, ORA_ERR_LIST_OVERFLOW, c, o, 0);
    return 0;
  }
  t->conn[(int64_t)c * CONN_CAP + t->nconn[c]++] = o;
  return 1;
}

/* ---------------------------------------------------------------------------
 * connect_cell, cell_connection.cpp:191-203 (gj_refresh, :133-152, is the
 * chemistry's gap-junction bookkeeping and does not feed the mechanics).
 * ------------------------------------------------------------------------- */

/* grid_init, cell_connection.cpp:38-62 */
static int grid_init(ora_tissue* t) {
  const int32_t nb = t->anx * t->any * t->anz;
  memset(t->bin_cnt, 0, sizeof(int32_t) * (size_t)nb);
  for (int32_t c = 0; c < t->n; ++c) {
    const int32_t aix = (int32_t)((0.5 * t->lx - pdx(t, 0.5 * t->lx, t->x[c])) / AREA_GRID);
    const int32_t aiy = (int32_t)((0.5 * t->ly - pdy(t, 0.5 * t->ly, t->y[c])) / AREA_GRID);
    const int32_t aiz = (int32_t)(min0(t->z[c]) / AREA_GRID);
    if (aix >= t->anx || aiy >= t->any || aiz >= t->anz || aix < 0 || aiy < 0 || aiz < 0) {
      set_err(t, ORA_ERR_BIN_RANGE, c, -1, 0);
      return t->err;
    }
    const int32_t b = (aix * t->any + aiy) * t->anz + aiz;
    if (t->bin_cnt[b] + 1 >= BIN_CAP) { /* assert(aindx < N3) after the push */
      set_err(t, ORA_ERR_BIN_OVERFLOW, c, b, 0);
      return t->err;
    }
    t->bin_list[(int64_t)b * BIN_CAP + t->bin_cnt[b]++] = c;
    t->nconn[c] = t->state[c] == S_MEMB ? t->nadj : 0; /* force_set_count, :60 */
  }
  return ORA_OK;
}

/* connect_proc, cell_connection.cpp:70-129 */
static int connect_proc(ora_tissue* t) {
  const double thr = t->P.lj_thresh * t->P.lj_thresh;
  for (int32_t c = t->nmemb; c < t->n; ++c) {
    const int32_t anx = (int32_t)(t->x[c] / AREA_GRID);
    const int32_t any = (int32_t)(t->y[c] / AREA_GRID);
    const int32_t anz = (int32_t)(t->z[c] / AREA_GRID);
    if (anx >= t->anx || any >= t->any || anz >= t->anz || anx < 0 || any < 0 || anz < 0) {
      set_err(t, ORA_ERR_BIN_RANGE, c, -2, 0); /* assert at :99 */
      return t->err;
    }
    for (int32_t j = anx - 2 + t->anx; j <= anx + 2 + t->anx; ++j) {
      const int32_t aix = j % t->anx;
      for (int32_t k = any - 2 + t->any; k <= any + 2 + t->any; ++k) {
        const int32_t aiy = k % t->any;
        for (int32_t l = anz - 2 + t->anz; l <= anz + 2 + t->anz; ++l) {
          const int32_t aiz = l % t->anz;
          const int32_t b = (aix * t->any + aiy) * t->anz + aiz;
          const int32_t sz = t->bin_cnt[b];
          for (int32_t m = 0; m < sz; ++m) {
            const int32_t o = t->bin_list[(int64_t)b * BIN_CAP + m];
            if (c <= o) continue;
            const double diffx = pdx(t, t->x[c], t->x[o]);
            const double diffy = pdy(t, t->y[c], t->y[o]);
            const double diffz = t->z[c] - t->z[o];
            const double rad_sum = t->radius[c] + t->radius[o];
            if (diffx * diffx + diffy * diffy + diffz * diffz <= thr * rad_sum * rad_sum) {
              if (!push_conn(t, c, o) || !push_conn(t, o, c)) return t->err;
            }
          }
        }
      }
    }
  }
  return ORA_OK;
}

/* find_dermis / set_dermis, cell_connection.cpp:158-185 */
static void set_dermis(ora_tissue* t) {
  for (int32_t c = t->nmemb + t->nder; c < t->n; ++c) {
    if (t->state[c] != S_FIX && t->state[c] != S_MUSUME) continue;
    double d1 = t->lx * t->lx;
    int32_t best = -1;
    for (int32_t k = 0; k < t->nconn[c]; ++k) {
      const int32_t o = t->conn[(int64_t)c * CONN_CAP + k];
      if (t->state[o] == S_MEMB) {
        const double d = dist_sq(t, c, o);
        if (d < d1) {
          d1 = d;
          best = o;
        }
      }
    }
    t->dermis[c] = best;
  }
}

int ora_connect(ora_tissue* t) {
  if (grid_init(t) != ORA_OK) return t->err;
  if (connect_proc(t) != ORA_OK) return t->err;
  set_dermis(t);
  return t->err;
}

/* ---------------------------------------------------------------------------
 * Force laws, cell_interaction.cpp:77-285. Each returns the pair coefficient
 * for (c1, c2); a nonzero *bad flags the reference's abort conditions.
 * ------------------------------------------------------------------------- */

/* ljmain, :103-111 */
static double ljmain(const ora_tissue* t, int32_t a, int32_t b) {
  const double d2 = dist_sq(t, a, b);
  const double rs = t->radius[a] + t->radius[b];
  const double lj6 = POW6(rs) / POW3(d2);
  return 4.0 * t->P.eps_m * lj6 * (lj6 - 1) / d2;
}
/* is_near, :90-93 */
static int is_near(const ora_tissue* t, int32_t a, int32_t b) {
  return dist_sq(t, a, b) < (t->radius[a] + t->radius[b]) * (t->radius[a] + t->radius[b]);
}
/* adhesion, :113-124 */
static double adhesion(const ora_tissue* t, int32_t a, int32_t b, double k) {
  const double lt = t->P.lj_thresh;
  const double distlj = sqrt(dist_sq(t, a, b));
  const double rs = t->radius[a] + t->radius[b];
  const double m1 = (distlj / rs) - 1;
  return (m1 + 1 > lt ? 0.0 : -(k / distlj) * m1 * (1 - m1 * m1 / ((lt - 1.0) * (lt - 1.0))));
}
/* CI_der_to_der, :129-139 with is_der_near / ljmain_der_near / _far, :77-101 */
static double ci_der_to_der(const ora_tissue* t, int32_t a, int32_t b) {
  const double rs = t->radius[a] + t->radius[b];
  if (sqrt(dist_sq(t, a, b)) + t->P.delta_r < rs) {
    const double dist = sqrt(dist_sq(t, a, b));
    const double dist2 = dist + t->P.delta_r;
    const double lj6 = POW6(rs) / POW6(dist2);
    return 4.0 * t->P.eps_m * lj6 * (lj6 - 1) / (dist * dist2) + t->P.para_ljp2;
  } else if (is_near(t, a, b)) {
    return t->P.para_ljp2;
  } else {
    const double dist = sqrt(dist_sq(t, a, b));
    const double dist2 = dist + t->P.delta_r;
    const double lj6 = POW6(rs) / POW6(dist2);
    return 4.0 * t->P.eps_m * lj6 * (lj6 - 1) / (dist * dist) + t->P.para_ljp2;
  }
}
/* CI_al_air_de_to_al_air_de_fix_mu, :141-152 */
static double ci_aad(const ora_tissue* t, int32_t a, int32_t b) {
  if (is_near(t, a, b)) return ljmain(t, a, b);
  double spf = t->P.k_desmosome;
  if (t->agek[a] > t->P.thresh_sp && t->agek[b] > t->P.thresh_sp) spf = t->P.k_total;
  return adhesion(t, a, b, spf);
}
/* CI_fix_mu_to_fix_mu, :154-162 */
static double ci_fixmu(const ora_tissue* t, int32_t a, int32_t b) {
  if (is_near(t, a, b)) return ljmain(t, a, b);
  return adhesion(t, a, b, t->P.k_desmosome);
}
/* CI_mu_to_memb, :164-172 */
static double ci_mu_memb(const ora_tissue* t, int32_t a, int32_t b) {
  if (is_near(t, a, b)) return ljmain(t, a, b);
  return adhesion(t, a, b, t->sfm[a]);
}
/* CI_fix_to_memb, :174-183 */
static double ci_fix_memb(const ora_tissue* t, int32_t a, int32_t b) {
  if (is_near(t, a, b)) return ljmain(t, a, b);
  const double distlj = sqrt(dist_sq(t, a, b));
  const double lj2 = distlj / (t->radius[a] + t->radius[b]);
  return -(t->P.kspring / distlj) * (lj2 - 1.0);
}
/* CI_memb_to_memb, :185-234 (|coef| > 100 aborts in each branch) */
static double ci_memb_memb(ora_tissue* t, int32_t a, int32_t b) {
  const double P = t->P.p_memb;
  const double rs = t->radius[a] + t->radius[b];
  const double rs2 = rs * rs;
  double cr2;
  const double d2 = dist_sq(t, a, b);
  double tmp;
  if (d2 < (cr2 = rs2 * P * P)) {
    const double lj6 = POW3(cr2) / POW3(d2);
    tmp = 4.0 * t->P.eps_m * lj6 * (lj6 - 1) / d2;
  } else if (d2 < rs2) {
    const double distlj = sqrt(d2);
    const double cr = rs * P;
    tmp = -(t->P.der_der_const / distlj) * (distlj / cr - 1.0);
  } else {
    const double distlj = sqrt(d2);
    const double lambda = (1.0 + P) * rs;
    const double cr = rs * P;
    const double lj6 = POW6(cr) / POW6(lambda - distlj);
    tmp = -(t->P.der_der_const / rs) * ((1.0 - P) / P) -
          4 * t->P.eps_m * (lj6 * (lj6 - 1.0)) / ((lambda - distlj) * distlj);
  }
  if (fabs(tmp) > 100) set_err(t, ORA_ERR_MEMB_COEF_RANGE, a, b, tmp);
  return tmp;
}
/* CI_pair, :281-285 */
static double ci_pair(const ora_tissue* t, int32_t a, int32_t b) {
  const double dist = sqrt(dist_sq(t, a, b));
  const double force = t->P.kspring_division * (dist - t->spr[a]);
  return -force / dist;
}

/* cell_interaction_apply, :48-66 */
static void apply(ora_tissue* t, int32_t c1, int32_t c2, double coef) {
  if (fabs(coef) > 1000) {
    set_err(t, ORA_ERR_COEF_RANGE, c1, c2, coef);
  }
  const double dt = t->P.dt;
  const double dumx = dt * coef * pdx(t, t->x[c1], t->x[c2]);
  const double dumy = dt * coef * pdy(t, t->y[c1], t->y[c2]);
  const double dumz = dt * coef * (t->z[c1] - t->z[c2]);
  t->nx[c1] += dumx;
  t->ny[c1] += dumy;
  t->nz[c1] += dumz;
  t->nx[c2] -= dumx;
  t->ny[c2] -= dumy;
  t->nz[c2] -= dumz;
}

/* wall_interaction, :287-294 */
static void wall(ora_tissue* t, int32_t c) {
  const double distlj = 2.0 * t->z[c];
  const double lj6 = POW6(t->radius[c]) / POW6(t->z[c]);
  const double ljm = 4.0 * t->P.eps_m * lj6 * (lj6 - 1.0) / (distlj * distlj);
  t->nz[c] += t->P.dt * ljm * 2.0 * t->z[c];
}

/* Square-membrane bending, _memb_bend_calc1..3, :296-449 (NEW_BEND_POT on,
 * define.h:230; DIAG_BEND off, define.h:67). */
static void bend_calc1(ora_tissue* t, int32_t m) {
  const int32_t r = t->lat_r[m], u = t->lat_u[m];
  const double dn = sqrt(dist_sq(t, r, m));
  t->nv[3 * m + 0] = pdx(t, t->x[r], t->x[m]) / dn;
  t->nv[3 * m + 1] = pdy(t, t->y[r], t->y[m]) / dn;
  t->nv[3 * m + 2] = (t->z[r] - t->z[m]) / dn;
  t->dn[m] = dn;
  const double dm = sqrt(dist_sq(t, u, m));
  t->mv[3 * m + 0] = pdx(t, t->x[u], t->x[m]) / dm;
  t->mv[3 * m + 1] = pdy(t, t->y[u], t->y[m]) / dm;
  t->mv[3 * m + 2] = (t->z[u] - t->z[m]) / dm;
  t->dm[m] = dm;
}
static void bend_calc2(ora_tissue* t, int32_t m) {
  const int32_t r = t->lat_r[m], u = t->lat_u[m];
  t->ipn[m] = t->nv[3 * m] * t->nv[3 * r] + t->nv[3 * m + 1] * t->nv[3 * r + 1] +
              t->nv[3 * m + 2] * t->nv[3 * r + 2];
  t->ipm[m] = t->mv[3 * m] * t->mv[3 * u] + t->mv[3 * m + 1] * t->mv[3 * u + 1] +
              t->mv[3 * m + 2] * t->mv[3 * u + 2];
}
/* _memb_bend_diff_factor, :349-360 */
static inline double bend_factor(double c) {
  if (c >= 0) return (1.0 - c);
  return 1.0 / ((1.0 + c) * (1.0 + c));
}
static void bend_calc3(ora_tissue* t, int32_t m) {
  const int32_t r = t->lat_r[m], l = t->lat_l[m], ll = t->lat_ll[m];
  const int32_t u = t->lat_u[m], b = t->lat_b[m], bb = t->lat_bb[m];
  const double* nvr = &t->nv[3 * r];
  const double* nvl = &t->nv[3 * l];
  const double* nvll = &t->nv[3 * ll];
  const double ipnl = t->ipn[l], ipnll = t->ipn[ll];
  const double* mvu = &t->mv[3 * u];
  const double* mvb = &t->mv[3 * b];
  const double* mvbb = &t->mv[3 * bb];
  const double ipmb = t->ipm[b];
  const double ipmbb = t->ipn[bb]; /* the reference reads ipn here (:380) */
  const double dnl = t->dn[l], dmb = t->dm[b];
  const double dn = t->dn[m], dm = t->dm[m];
  const double* nv = &t->nv[3 * m];
  const double* mv = &t->mv[3 * m];
  const double ipn = t->ipn[m], ipm = t->ipm[m];
  double f[3];
  for (int k = 0; k < 3; ++k) {
    f[k] = -(bend_factor(ipn)) * (nvr[k] - ipn * nv[k]) / dn +
           bend_factor(ipnl) * ((nv[k] - ipnl * nvl[k]) / dnl - (nvl[k] - ipnl * nv[k]) / dn) +
           bend_factor(ipnll) * (nvll[k] - ipnll * nvl[k]) / dnl -
           bend_factor(ipm) * (mvu[k] - ipm * mv[k]) / dm +
           bend_factor(ipmb) * ((mv[k] - ipmb * mvb[k]) / dmb - (mvb[k] - ipmb * mv[k]) / dm) +
           bend_factor(ipmbb) * (mvbb[k] - ipmbb * mvb[k]) / dmb;
  }
  const double s = t->P.dt * t->P.kbend;
  t->nx[m] += s * f[0];
  t->ny[m] += s * f[1];
  t->nz[m] += s * f[2];
}

/* Triangular-membrane bending, tri_memb_bend and tri_bend_1 / tri_bend_2,
 * :451-499, with vec3 (vec3.h:5-54) restated operation by operation.
 * normalize() works in place (vec3.h:40-44), so the reference's divisions
 * by norm1_pre.norm() / norm2_pre.norm() divide by the norm of an already
 * normalised vector; kept as is. */
typedef struct { double x, y, z; } v3;
static inline v3 v3_pos(const ora_tissue* t, int32_t c) { v3 r = {t->x[c], t->y[c], t->z[c]}; return r; }
static inline v3 v3_psub(const ora_tissue* t, v3 a, v3 b) { /* vpsub */
  v3 r = {pdx(t, a.x, b.x), pdy(t, a.y, b.y), a.z - b.z};
  return r;
}
static inline v3 v3_cross(v3 a, v3 b) {
  v3 r = {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
  return r;
}
static inline double v3_dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline double v3_norm(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline v3 v3_normalize(v3* a) {
  const double nm = v3_norm(*a);
  a->x /= nm; a->y /= nm; a->z /= nm;
  return *a;
}
static inline v3 v3_scale(double c, v3 a) { v3 r = {c * a.x, c * a.y, c * a.z}; return r; }
static inline v3 v3_div(v3 a, double c) { v3 r = {a.x / c, a.y / c, a.z / c}; return r; }
static inline v3 v3_add(v3 a, v3 b) { v3 r = {a.x + b.x, a.y + b.y, a.z + b.z}; return r; }
static inline v3 v3_sub(v3 a, v3 b) { v3 r = {a.x - b.x, a.y - b.y, a.z - b.z}; return r; }
/* tri_rho, :470-472 */
static inline v3 tri_rho(v3 n1, v3 b1) { return v3_sub(b1, v3_scale(v3_dot(n1, b1), n1)); }
/* tri_bend_1, :475-481 */
static v3 tri_bend_1(const ora_tissue* t, int32_t r1, int32_t a1, int32_t b1, int32_t c1) {
  const v3 r1v = v3_pos(t, r1), a1v = v3_pos(t, a1), b1v = v3_pos(t, b1), c1v = v3_pos(t, c1);
  v3 norm1_pre = v3_cross(v3_psub(t, r1v, b1v), v3_psub(t, a1v, b1v));
  const v3 norm1 = v3_normalize(&norm1_pre);
  v3 n2 = v3_cross(v3_psub(t, a1v, b1v), v3_psub(t, c1v, b1v));
  const v3 norm2 = v3_normalize(&n2);
  const double dot1 = v3_dot(norm1, norm2);
  return v3_scale(bend_factor(dot1),
                  v3_div(v3_cross(v3_psub(t, a1v, b1v), tri_rho(norm1, norm2)), v3_norm(norm1_pre)));
}
/* tri_bend_2, :483-495 */
static v3 tri_bend_2(const ora_tissue* t, int32_t r1, int32_t a1, int32_t b1, int32_t c1) {
  const v3 r1v = v3_pos(t, r1), a1v = v3_pos(t, a1), b1v = v3_pos(t, b1), c1v = v3_pos(t, c1);
  v3 norm1_pre = v3_cross(v3_psub(t, r1v, c1v), v3_psub(t, b1v, c1v));
  v3 norm2_pre = v3_cross(v3_psub(t, r1v, b1v), v3_psub(t, a1v, b1v));
  const v3 norm1 = v3_normalize(&norm1_pre), norm2 = v3_normalize(&norm2_pre);
  const double dot1 = v3_dot(norm1, norm2);
  return v3_scale(bend_factor(dot1),
                  v3_add(v3_div(v3_cross(v3_psub(t, b1v, c1v), tri_rho(norm1, norm2)),
                                v3_norm(norm1_pre)),
                         v3_div(v3_cross(v3_psub(t, a1v, b1v), tri_rho(norm2, norm1)),
                                v3_norm(norm2_pre))));
}
/* tri_memb_bend, :497-508 */
static void tri_memb_bend(ora_tissue* t, int32_t m) {
  const int32_t* nb = &t->tri_nb[6 * m];
  v3 dr = {0, 0, 0};
  for (int i = 0; i < 6; ++i) {
    const int32_t b = nb[(i + 1) % 6];
    dr = v3_add(dr, tri_bend_1(t, m, nb[i], b, t->tri_nb[6 * b + i]));
  }
  for (int i = 0; i < 6; ++i) dr = v3_add(dr, tri_bend_2(t, m, nb[i], nb[(i + 1) % 6], nb[(i + 2) % 6]));
  t->nx[m] += t->P.dt * t->P.kbend * dr.x;
  t->ny[m] += t->P.dt * t->P.kbend * dr.y;
  t->nz[m] += t->P.dt * t->P.kbend * dr.z;
}

static inline int is_aad(uint8_t s) { return s == S_ALIVE || s == S_AIR || s == S_DEAD; }

/* cell_interaction, :648-685, with the per-state bodies :529-641 */
int ora_interact(ora_tissue* t) {
  const int64_t C = CONN_CAP;
  if (t->tri) { /* memb_bend, TRI_MEMB branch, :501-506 */
    for (int32_t m = 0; m < t->nmemb; ++m) tri_memb_bend(t, m);
  } else {
    for (int32_t m = 0; m < t->nmemb; ++m) bend_calc1(t, m);
    for (int32_t m = 0; m < t->nmemb; ++m) bend_calc2(t, m);
    for (int32_t m = 0; m < t->nmemb; ++m) bend_calc3(t, m);
  }
  /* _MEMB_interaction, :529-547 */
  for (int32_t m = 0; m < t->nmemb; ++m) {
    if (t->z[m] < t->radius[m]) wall(t, m);
    for (int32_t i = 0; i < t->nadj; ++i) {
      const int32_t o = t->conn[m * C + i];
      if (t->state[o] == S_MEMB && m > o) apply(t, m, o, ci_memb_memb(t, m, o));
    }
  }
  for (int32_t c = t->nmemb; c < t->n; ++c) {
    const uint8_t sc = t->state[c];
    const int32_t* row = &t->conn[c * C];
    const int32_t nc = t->nconn[c];
    if (sc == S_DER) { /* _DER_interaction, :549-561 */
      if (t->z[c] < t->radius[c]) wall(t, c);
      for (int32_t k = 0; k < nc; ++k) {
        const int32_t o = row[k];
        if (t->state[o] == S_DER && c > o)
          apply(t, c, o, ci_der_to_der(t, c, o));
        else
          apply(t, c, o, ljmain(t, c, o));
      }
    } else if (sc == S_FIX) { /* _FIX_interaction, :581-604 */
      for (int32_t k = 0; k < nc; ++k) {
        const int32_t o = row[k];
        const uint8_t so = t->state[o];
        if (so == S_FIX) {
          if (t->pair[c] != o && c > o) apply(t, c, o, ci_fixmu(t, c, o));
        } else if (so == S_MUSUME) {
          if (t->pair[c] != o) apply(t, c, o, ci_fixmu(t, c, o));
        } else if (so == S_MEMB) {
          if (t->dermis[c] == o)
            apply(t, c, o, ci_fix_memb(t, c, o));
          else
            apply(t, c, o, ljmain(t, c, o));
        }
      }
    } else if (sc == S_MUSUME) { /* _MUSUME_interaction, :613-634 */
      t->sfm[c] = 0;
      if (t->pair[c] >= 0 && t->state[t->pair[c]] == S_FIX)
        t->sfm[c] = t->P.kspring;
      else if (t->rest_div[c] > 0)
        t->sfm[c] = t->P.kspring_d;
      for (int32_t k = 0; k < nc; ++k) {
        const int32_t o = row[k];
        const uint8_t so = t->state[o];
        if (so == S_MEMB) {
          if (t->dermis[c] == o)
            apply(t, c, o, ci_mu_memb(t, c, o));
          else
            apply(t, c, o, ljmain(t, c, o));
        } else if (so == S_MUSUME && t->pair[c] != o && c > o) {
          apply(t, c, o, ci_fixmu(t, c, o));
        }
      }
    } else if (is_aad(sc)) { /* _AL_AIR_DE_interaction, :563-579 */
      for (int32_t k = 0; k < nc; ++k) {
        const int32_t o = row[k];
        const uint8_t so = t->state[o];
        if (is_aad(so)) {
          if (c > o) apply(t, c, o, ci_aad(t, c, o));
        } else if (so != S_DER) {
          apply(t, c, o, ci_aad(t, c, o));
        }
      }
    }
    /* _pair_interaction, :637-641 */
    if (t->pair[c] >= 0 && c > t->pair[c]) apply(t, c, t->pair[c], ci_pair(t, c, t->pair[c]));
  }
  return t->err;
}

/* pos_copy, cellmanager.cpp:19-26 */
void ora_pos_copy(ora_tissue* t) {
  for (int32_t c = 0; c < t->n; ++c) {
    t->x[c] = t->nx[c];
    t->y[c] = t->ny[c];
    t->z[c] = t->nz[c];
  }
}

/* cell_pos_periodic_fix, cellmanager.cpp:395-414 */
void ora_periodic_fix(ora_tissue* t) {
  for (int32_t c = 0; c < t->n; ++c) {
    if (t->nx[c] > t->lx) {
      t->x[c] = t->nx[c] = t->nx[c] - t->lx;
    } else if (t->nx[c] < 0) {
      t->x[c] = t->nx[c] = t->nx[c] + t->lx;
    }
    if (t->ny[c] > t->ly) {
      t->y[c] = t->ny[c] = t->ny[c] - t->ly;
    } else if (t->ny[c] < 0) {
      t->y[c] = t->ny[c] = t->ny[c] + t->ly;
    }
  }
}

int ora_step(ora_tissue* t, int32_t nsteps) {
  for (int32_t s = 0; s < nsteps; ++s) {
    if (ora_interact(t) != ORA_OK) return t->err;
    ora_pos_copy(t);
    ora_periodic_fix(t);
    for (int32_t c = 0; c < t->n; ++c) {
      if (!isfinite(t->x[c]) || !isfinite(t->y[c]) || !isfinite(t->z[c])) {
        set_err(t, ORA_ERR_NONFINITE, c, -1, 0);
        return t->err;
      }
    }
    if (ora_connect(t) != ORA_OK) return t->err;
  }
  return t->err;
}

/* Square lattice wiring, _memb_init, cellmanager.cpp:114-166. */
/* Triangular lattice wiring, _memb_init TRI_MEMB branch, cellmanager.cpp:70-111:
 * memb[0] right, [3] left; rows alternate their offset, so the upper / lower
 * neighbours depend on the row's parity. */
static void wire_membrane_tri(ora_tissue* t) {
  const int32_t NMX = t->nmx, nm = t->nmemb;
  for (int32_t j = 0; j < nm; ++j) {
    const int32_t jj = j % NMX;
    t->tri_nb[6 * j + 3] = jj == 0 ? j + NMX - 1 : j - 1;
    t->tri_nb[6 * j + 0] = jj == NMX - 1 ? j - (NMX - 1) : j + 1;
  }
  for (int32_t j = 0; j < nm; ++j) {
    const int32_t kk = j / NMX;
    const int32_t top = (j - NMX + nm) % nm, bot = (j + NMX) % nm;
    int32_t* nb = &t->tri_nb[6 * j];
    if (kk % 2 == 0) {
      nb[1] = top;
      nb[2] = t->tri_nb[6 * top + 3];
      nb[4] = t->tri_nb[6 * bot + 3];
      nb[5] = bot;
    } else {
      nb[1] = t->tri_nb[6 * top + 0];
      nb[2] = top;
      nb[4] = bot;
      nb[5] = t->tri_nb[6 * bot + 0];
    }
    t->nconn[j] = 0;
    for (int i = 0; i < 6; ++i) push_conn(t, j, nb[i]);
  }
}

static void wire_membrane(ora_tissue* t) {
  const int32_t NMX = t->nmx, NMY = t->nmy;
  for (int32_t j = 0; j < t->nmemb; ++j) {
    const int32_t jj = j % NMX, kk = j / NMX;
    t->lat_l[j] = jj == 0 ? j + NMX - 1 : j - 1;
    t->lat_ll[j] = jj <= 1 ? j + NMX - 2 : j - 2;
    t->lat_r[j] = jj == NMX - 1 ? j - (NMX - 1) : j + 1;
    t->lat_b[j] = kk == 0 ? j + NMX * NMY - NMX : j - NMX;
    t->lat_bb[j] = kk <= 1 ? j + NMX * NMY - 2 * NMX : j - 2 * NMX;
    t->lat_u[j] = kk == NMY - 1 ? j - (NMX * NMY - NMX) : j + NMX;
    t->nconn[j] = 0;
    push_conn(t, j, t->lat_l[j]);
    push_conn(t, j, t->lat_r[j]);
    push_conn(t, j, t->lat_b[j]);
    push_conn(t, j, t->lat_u[j]);
  }
}

#define ALLOC(p, cnt) \
  do { (p) = calloc((size_t)(cnt) > 0 ? (size_t)(cnt) : 1, sizeof(*(p))); if (!(p)) goto fail; } while (0)

ora_tissue* ora_new(int32_t n, int32_t nmemb, int32_t nder, int32_t nmx, int32_t nmy,
                    double lx, double ly, double lz, const double* params14,
                    const double* x, const double* y, const double* z,
                    const double* radius, const double* agek, const double* spr_nat_len,
                    const uint8_t* state, const int32_t* pair, const int32_t* rest_div_times) {
  return ora_new_lattice(n, nmemb, nder, nmx, nmy, lx, ly, lz, params14, x, y, z, radius, agek,
                         spr_nat_len, state, pair, rest_div_times, 0);
}

ora_tissue* ora_new_lattice(int32_t n, int32_t nmemb, int32_t nder, int32_t nmx, int32_t nmy,
                            double lx, double ly, double lz, const double* params14,
                            const double* x, const double* y, const double* z,
                            const double* radius, const double* agek, const double* spr_nat_len,
                            const uint8_t* state, const int32_t* pair,
                            const int32_t* rest_div_times, int32_t lattice) {
  if (n < 0 || nmemb < 0 || nder < 0 || nmemb + nder > n || nmx < 3 || nmy < 3 ||
      nmemb != nmx * nmy || lattice < 0 || lattice > 1 || (lattice == 1 && nmy % 2 != 0))
    return NULL;
  ora_tissue* t = calloc(1, sizeof(ora_tissue));
  if (!t) return NULL;
  t->n = n; t->nmemb = nmemb; t->nder = nder; t->nmx = nmx; t->nmy = nmy;
  t->tri = lattice;
  t->nadj = lattice ? MEMB_ADJ_TRI : MEMB_ADJ_SQUARE;
  t->lx = lx; t->ly = ly; t->lz = lz;
  /* ANX, ANY, ANZ, cell_connection.cpp:22-26 */
  t->anx = (int32_t)(lx / AREA_GRID_ORIGINAL + 0.5);
  t->any = (int32_t)(ly / AREA_GRID_ORIGINAL + 0.5);
  t->anz = (int32_t)(lz / AREA_GRID_ORIGINAL);
  memcpy(&t->P, params14, sizeof(ora_params));
  ALLOC(t->x, n); ALLOC(t->y, n); ALLOC(t->z, n);
  ALLOC(t->nx, n); ALLOC(t->ny, n); ALLOC(t->nz, n);
  ALLOC(t->radius, n); ALLOC(t->agek, n); ALLOC(t->spr, n); ALLOC(t->sfm, n);
  ALLOC(t->state, n); ALLOC(t->pair, n); ALLOC(t->rest_div, n); ALLOC(t->dermis, n);
  ALLOC(t->conn, (int64_t)n * CONN_CAP); ALLOC(t->nconn, n);
  ALLOC(t->lat_l, nmemb); ALLOC(t->lat_ll, nmemb); ALLOC(t->lat_r, nmemb);
  ALLOC(t->lat_b, nmemb); ALLOC(t->lat_bb, nmemb); ALLOC(t->lat_u, nmemb);
  ALLOC(t->tri_nb, 6 * (int64_t)nmemb);
  ALLOC(t->nv, 3 * (int64_t)nmemb); ALLOC(t->mv, 3 * (int64_t)nmemb);
  ALLOC(t->dn, nmemb); ALLOC(t->dm, nmemb); ALLOC(t->ipn, nmemb); ALLOC(t->ipm, nmemb);
  ALLOC(t->bin_cnt, (int64_t)t->anx * t->any * t->anz);
  ALLOC(t->bin_list, (int64_t)t->anx * t->any * t->anz * BIN_CAP);
  for (int32_t i = 0; i < n; ++i) {
    t->x[i] = t->nx[i] = x[i];
    t->y[i] = t->ny[i] = y[i];
    t->z[i] = t->nz[i] = z[i];
    t->radius[i] = radius[i];
    t->agek[i] = agek[i];
    t->spr[i] = spr_nat_len[i];
    t->state[i] = state[i];
    t->pair[i] = pair[i];
    t->rest_div[i] = rest_div_times[i];
    t->dermis[i] = -1;
  }
  if (t->tri)
    wire_membrane_tri(t);
  else
    wire_membrane(t);
  ora_connect(t);
  return t;
fail:
  ora_free(t);
  return NULL;
}

void ora_free(ora_tissue* t) {
  if (!t) return;
  free(t->x); free(t->y); free(t->z); free(t->nx); free(t->ny); free(t->nz);
  free(t->radius); free(t->agek); free(t->spr); free(t->sfm); free(t->state);
  free(t->pair); free(t->rest_div); free(t->dermis); free(t->conn); free(t->nconn);
  free(t->lat_l); free(t->lat_ll); free(t->lat_r); free(t->lat_b); free(t->lat_bb);
  free(t->lat_u); free(t->nv); free(t->mv); free(t->dn); free(t->dm); free(t->ipn);
  free(t->ipm); free(t->bin_cnt); free(t->bin_list); free(t->tri_nb);
  free(t);
}

void ora_get_positions(const ora_tissue* t, double* x, double* y, double* z) {
  memcpy(x, t->x, sizeof(double) * (size_t)t->n);
  memcpy(y, t->y, sizeof(double) * (size_t)t->n);
  memcpy(z, t->z, sizeof(double) * (size_t)t->n);
}

void ora_set_positions(ora_tissue* t, const double* x, const double* y, const double* z) {
  for (int32_t i = 0; i < t->n; ++i) {
    t->x[i] = t->nx[i] = x[i];
    t->y[i] = t->ny[i] = y[i];
    t->z[i] = t->nz[i] = z[i];
  }
}

static int cmp_i32(const void* a, const void* b) {
  const int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

static int64_t get_conn(const ora_tissue* t, int32_t* offsets, int32_t* idx, int64_t cap,
                        int sorted) {
  int64_t tot = 0;
  offsets[0] = 0;
  for (int32_t c = 0; c < t->n; ++c) {
    const int32_t k = t->nconn[c];
    if (idx && tot + k <= cap) {
      memcpy(idx + tot, &t->conn[(int64_t)c * CONN_CAP], sizeof(int32_t) * (size_t)k);
      if (sorted) qsort(idx + tot, (size_t)k, sizeof(int32_t), cmp_i32);
    }
    tot += k;
    offsets[c + 1] = (int32_t)tot;
  }
  return tot;
}

int64_t ora_get_connections(const ora_tissue* t, int32_t* offsets, int32_t* idx, int64_t cap) {
  return get_conn(t, offsets, idx, cap, 1);
}

int64_t ora_get_connections_raw(const ora_tissue* t, int32_t* offsets, int32_t* idx,
                                int64_t cap) {
  return get_conn(t, offsets, idx, cap, 0);
}

void ora_get_dermis(const ora_tissue* t, int32_t* dermis) {
  memcpy(dermis, t->dermis, sizeof(int32_t) * (size_t)t->n);
}

int ora_get_tri_neighbours(const ora_tissue* t, int32_t* nb) {
  if (!t->tri) return -1;
  memcpy(nb, t->tri_nb, sizeof(int32_t) * 6 * (size_t)t->nmemb);
  return 0;
}

int ora_error_info(const ora_tissue* t, int32_t* a, int32_t* b, double* value) {
  if (a) *a = t->err_a;
  if (b) *b = t->err_b;
  if (value) *value = t->err_v;
  return t->err;
}

/* ---------------------------------------------------------------------------
 * Cell maps and external-stimulus diffusion: the rest of the reference's
 * per-step loop before its chemistry (epi5_MT/proc.cpp:152-157). Grids are
 * (nx+1) x (ny+1) x (nz+1), z fastest, like FArr3D (define.h:243).
 * ------------------------------------------------------------------------- */
struct ora_field {
  int32_t nx, ny, nz;
  double dx, dy, dz, inv_dx, inv_dy, inv_dz;
  int32_t* cmap1;  /* cell index, -1 for none (FArr3D<const Cell*>) */
  uint8_t* cmap2;  /* FArr3D<cmask_ty> */
  double* ext[2];  /* SwapData<FArr3D<double>>: ext[cur] is first() */
  int cur;
};

#define FIELD_RAD 1.4         /* Rad, map.cpp:26 */
#define FIELD_FAC_MAP 2.0     /* FAC_MAP, define.h:184 */
#define FIELD_R_MAX 1.4       /* R_max, define.h:116 */
#define FIELD_DT_CA 0.01      /* DT_Ca, define.h:89 */
#define FIELD_DB 0.0009       /* DB, ext_stim.cpp:20 */
#define FIELD_KB 0.025        /* kb, ext_stim.cpp:10 */
#define FIELD_DUR_ALIVE 0.5   /* ext_stim.cpp:11 */
#define FIELD_DUR_DEAD 2.0    /* ext_stim.cpp:12 */
#define FIELD_THRESH_DEAD 22.0 /* define.h:156 */

static inline size_t fidx(const ora_field* f, int32_t a, int32_t b, int32_t c) {
  return ((size_t)a * (size_t)(f->ny + 1) + (size_t)b) * (size_t)(f->nz + 1) + (size_t)c;
}

ora_field* ora_field_new(const ora_tissue* t, int32_t nx, int32_t ny, int32_t nz) {
  if (!t || nx < 3 || ny < 3 || nz < 3) return NULL;
  ora_field* f = calloc(1, sizeof(ora_field));
  if (!f) return NULL;
  f->nx = nx; f->ny = ny; f->nz = nz;
  /* cdefd dx = LX / NX; inv_dx = NX / LX (define.h:111-113) */
  f->dx = t->lx / (double)nx; f->inv_dx = (double)nx / t->lx;
  f->dy = t->ly / (double)ny; f->inv_dy = (double)ny / t->ly;
  f->dz = t->lz / (double)nz; f->inv_dz = (double)nz / t->lz;
  const size_t nv = (size_t)(nx + 1) * (size_t)(ny + 1) * (size_t)(nz + 1);
  f->cmap1 = malloc(sizeof(int32_t) * nv);
  f->cmap2 = calloc(nv, 1);
  f->ext[0] = calloc(nv, sizeof(double));
  f->ext[1] = calloc(nv, sizeof(double));
  if (!f->cmap1 || !f->cmap2 || !f->ext[0] || !f->ext[1]) {
    ora_field_free(f);
    return NULL;
  }
  for (size_t v = 0; v < nv; ++v) f->cmap1[v] = -1;
  return f;
}

void ora_field_free(ora_field* f) {
  if (!f) return;
  free(f->cmap1); free(f->cmap2); free(f->ext[0]); free(f->ext[1]);
  free(f);
}

static inline int fafm(uint8_t s) { return s == S_ALIVE || s == S_FIX || s == S_MUSUME; }

/* setup_map_lat, map.cpp:24-167 (cells visited in index order, so where
 * spheres overlap the last, highest-index cell is the one cmap1 keeps) */
static void field_map(const ora_tissue* t, ora_field* f) {
  const int32_t NX = f->nx, NY = f->ny, NZ = f->nz;
  const size_t nv = (size_t)(NX + 1) * (size_t)(NY + 1) * (size_t)(NZ + 1);
  for (size_t v = 0; v < nv; ++v) { f->cmap1[v] = -1; f->cmap2[v] = 0; }
  const int irx = (int)(FIELD_RAD * (double)NX / t->lx);
  const int iry = (int)(FIELD_RAD * (double)NY / t->ly);
  const int irz = (int)(FIELD_RAD * (double)NZ / t->lz);
  for (int32_t c = 0; c < t->n; ++c) {
    /* set_lattice, map.cpp:18-22 */
    const int lat0 = (int)(((size_t)((int)(t->x[c] * f->inv_dx)) + (size_t)NX) % (size_t)NX);
    const int lat1 = (int)(((size_t)((int)(t->y[c] * f->inv_dy)) + (size_t)NY) % (size_t)NY);
    const int lat2 = (int)(((size_t)((int)(t->z[c] * f->inv_dz)) + (size_t)NZ) % (size_t)NZ);
    const int afm = fafm(t->state[c]);
    const int rx = afm ? 2 * irx : irx, ry = afm ? 2 * iry : iry, rz = afm ? 2 * irz : irz;
    const double normal_radSq = t->radius[c] * t->radius[c];
    const double crad = FIELD_FAC_MAP * t->radius[c];
    const double cradSq = crad * crad;
    const int ymin = lat1 - ry, ymax = lat1 + ry;
    const int z_b = lat2 - rz, z_u = lat2 + rz;
    const int zmin = z_b >= 1 ? z_b : 1;
    const int zmax = z_u < NZ ? z_u : NZ - 1;
    for (int k = lat0 - rx; k <= lat0 + rx; ++k) {
      const double mx = k * f->dx;
      const int ipx = (k + NX) % NX;
      const double diffx = pdx(t, mx, t->x[c]);
      const double diffxSq = diffx * diffx;
      for (int l = ymin; l <= ymax; ++l) {
        const double my = l * f->dy;
        const int ipy = (l + NY) % NY;
        const double diffy = pdy(t, my, t->y[c]);
        const double tmps = diffxSq + diffy * diffy;
        for (int m = zmin; m <= zmax; ++m) {
          const double mz = m * f->dz;
          const double diffz = mz - t->z[c];
          const double distSq = tmps + diffz * diffz;
          const size_t v = fidx(f, ipx, ipy, m);
          if (afm) {
            if (distSq < cradSq) {
              f->cmap2[v] = 1;
              if (distSq < normal_radSq) f->cmap1[v] = c;
            }
          } else if (distSq < normal_radSq) {
            f->cmap1[v] = c;
          }
        }
      }
    }
  }
  for (int32_t l = 0; l < NZ; ++l) { /* periodic copies, map.cpp:156-166 */
    for (int32_t j = 0; j <= NX; ++j) {
      f->cmap2[fidx(f, j, NY, l)] = f->cmap2[fidx(f, j, 0, l)];
      f->cmap1[fidx(f, j, NY, l)] = f->cmap1[fidx(f, j, 0, l)];
    }
    for (int32_t k = 0; k <= NY; ++k) {
      f->cmap2[fidx(f, NX, k, l)] = f->cmap2[fidx(f, 0, k, l)];
      f->cmap1[fidx(f, NX, k, l)] = f->cmap1[fidx(f, 0, k, l)];
    }
  }
}

/* fB, ext_stim.cpp:8-16 */
static inline double field_fB(double age, double B, int cornif) {
  return (cornif && age > FIELD_THRESH_DEAD - FIELD_DUR_ALIVE &&
                  age <= FIELD_THRESH_DEAD + FIELD_DUR_DEAD
              ? 1
              : 0) -
         FIELD_KB * B;
}

/* calc_ext_stim, ext_stim.cpp:18-69 */
static int field_ext_stim(const ora_tissue* t, ora_field* f, double zzmax) {
  const int32_t NX = f->nx, NY = f->ny, NZ = f->nz;
  const int iz_bound = (int)((zzmax + FIELD_FAC_MAP * FIELD_R_MAX) * f->inv_dz);
  if (iz_bound > NZ) return ORA_ERR_INVALID_ARG; /* the reference would read past the grid */
  const double* carr = f->ext[f->cur];
  double* narr = f->ext[f->cur ^ 1];
  for (int32_t j = 0; j < NX; ++j) {
    const int32_t px = j == 0 ? NX - 1 : j - 1, nxi = j + 1 == NX ? 0 : j + 1;
    for (int32_t k = 0; k < NY; ++k) {
      const int32_t py = k == 0 ? NY - 1 : k - 1, nyi = k + 1 == NY ? 0 : k + 1;
      for (int32_t l = 0; l < iz_bound; ++l) {
        const int32_t pz = l == 0 ? 1 : l - 1, nzi = l + 1 == NZ ? NZ - 1 : l + 1;
        double dum_age = 0;
        int cornif = 0;
        const int32_t cm = f->cmap1[fidx(f, j, k, l)];
        if (cm >= 0 && (t->state[cm] == S_DEAD || t->state[cm] == S_ALIVE)) {
          dum_age = t->agek[cm];
          cornif = 1;
        }
        const double cext = carr[fidx(f, j, k, l)];
        narr[fidx(f, j, k, l)] =
            cext + FIELD_DT_CA *
                       (FIELD_DB *
                            (f->cmap2[fidx(f, px, k, l)] * (carr[fidx(f, px, k, l)] - cext) +
                             f->cmap2[fidx(f, j, py, l)] * (carr[fidx(f, j, py, l)] - cext) +
                             f->cmap2[fidx(f, j, k, pz)] * (carr[fidx(f, j, k, pz)] - cext) +
                             f->cmap2[fidx(f, j, k, nzi)] * (carr[fidx(f, j, k, nzi)] - cext) +
                             f->cmap2[fidx(f, j, nyi, l)] * (carr[fidx(f, j, nyi, l)] - cext) +
                             f->cmap2[fidx(f, nxi, k, l)] * (carr[fidx(f, nxi, k, l)] - cext)) *
                            f->inv_dz * f->inv_dz +
                        field_fB(dum_age, cext, cornif));
      }
    }
  }
  for (int32_t l = 0; l < iz_bound; ++l) { /* periodic copies, ext_stim.cpp:63-66 */
    for (int32_t j = 0; j < NX; ++j) narr[fidx(f, j, NY, l)] = narr[fidx(f, j, 0, l)];
    for (int32_t k = 0; k <= NY; ++k) narr[fidx(f, NX, k, l)] = narr[fidx(f, 0, k, l)];
  }
  f->cur ^= 1; /* ext_stim.swap() */
  return ORA_OK;
}

/* calc_zzmax, proc.cpp:34-43 */
static double field_zzmax(const ora_tissue* t) {
  double zmax = 0;
  for (int32_t c = t->nmemb + t->nder; c < t->n; ++c) {
    const uint8_t s = t->state[c];
    if ((s == S_DEAD || s == S_ALIVE || s == S_MUSUME || s == S_FIX) && zmax < t->z[c]) zmax = t->z[c];
  }
  return zmax;
}

int ora_field_step(const ora_tissue* t, ora_field* f, double* zzmax_out) {
  const double zzmax = field_zzmax(t);
  if (zzmax_out) *zzmax_out = zzmax;
  field_map(t, f);
  return field_ext_stim(t, f, zzmax);
}

void ora_field_get(const ora_field* f, int32_t* cmap1, uint8_t* cmap2, double* ext) {
  const size_t nv = (size_t)(f->nx + 1) * (size_t)(f->ny + 1) * (size_t)(f->nz + 1);
  if (cmap1) memcpy(cmap1, f->cmap1, sizeof(int32_t) * nv);
  if (cmap2) memcpy(cmap2, f->cmap2, nv);
  if (ext) memcpy(ext, f->ext[f->cur], sizeof(double) * nv);
}
