/* CPU restatement of the epi5_MT cell-mechanics step (TEST INFRASTRUCTURE).
 *
 * This is the oracle: a plain-C, FP64, single-threaded restatement of the
 * reference's connect_cell / cell_interaction / pos_copy /
 * cell_pos_periodic_fix (epi5_MT, square membrane build). Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it, and
 * only as the checker; the product library never links it.
 *
 * It visits cells and connections in exactly the order the reference does
 * when its TBB loops run serially, so its FP64 results are bit-identical to
 * the compiled reference built with the serial TBB stand-in (pinned by
 * tests/test_oracle.py against oracle/_ref and tests/golden). Unlike the
 * reference it takes the force constants at run time, which the ensemble and
 * adjoint checks need.
 *
 * Error codes share their values with include/epi_mech.h.
 */
#ifndef EPI_ORACLE_H
#define EPI_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  ORA_OK = 0,
  ORA_ERR_INVALID_ARG = 1,
  ORA_ERR_BIN_RANGE = 5,
  ORA_ERR_BIN_OVERFLOW = 6,
  ORA_ERR_LIST_OVERFLOW = 7,
  ORA_ERR_COEF_RANGE = 8,
  ORA_ERR_MEMB_COEF_RANGE = 9,
  ORA_ERR_NONFINITE = 10
};

/* Same field order as epi_params in include/epi_mech.h. */
typedef struct ora_params {
  double dt, eps_m, p_memb, der_der_const, k_total, k_desmosome, kspring,
      kspring_d, kbend, delta_r, para_ljp2, kspring_division, lj_thresh, thresh_sp;
} ora_params;

typedef struct ora_tissue ora_tissue;

/* Creates a tissue and runs the initial connect (as cman_init does,
 * epi5_MT/cell_init.cpp:132-137). Returns NULL on bad arguments. */
ora_tissue* ora_new(int32_t n, int32_t nmemb, int32_t nder, int32_t nmx, int32_t nmy,
                    double lx, double ly, double lz, const double* params14,
                    const double* x, const double* y, const double* z,
                    const double* radius, const double* agek, const double* spr_nat_len,
                    const uint8_t* state, const int32_t* pair, const int32_t* rest_div_times);
/* Same, with the membrane lattice: 0 square (TRI_MEMB undefined), 1
 * triangular (TRI_MEMB, the reference's default; nmy = number of rows, even). */
ora_tissue* ora_new_lattice(int32_t n, int32_t nmemb, int32_t nder, int32_t nmx, int32_t nmy,
                            double lx, double ly, double lz, const double* params14,
                            const double* x, const double* y, const double* z,
                            const double* radius, const double* agek, const double* spr_nat_len,
                            const uint8_t* state, const int32_t* pair,
                            const int32_t* rest_div_times, int32_t lattice);
void ora_free(ora_tissue* t);

int ora_connect(ora_tissue* t);         /* connect_cell without gj_refresh */
int ora_interact(ora_tissue* t);        /* cell_interaction into the next buffer */
void ora_pos_copy(ora_tissue* t);       /* pos_copy */
void ora_periodic_fix(ora_tissue* t);   /* cell_pos_periodic_fix */
int ora_step(ora_tissue* t, int32_t nsteps);

void ora_get_positions(const ora_tissue* t, double* x, double* y, double* z);
void ora_set_positions(ora_tissue* t, const double* x, const double* y, const double* z);
/* Per-cell connection lists, each sorted ascending, CSR form. Returns the
 * total number of entries; writes at most cap indices. */
int64_t ora_get_connections(const ora_tissue* t, int32_t* offsets, int32_t* idx, int64_t cap);
/* Lists in the reference's own push order (unsorted). */
int64_t ora_get_connections_raw(const ora_tissue* t, int32_t* offsets, int32_t* idx, int64_t cap);
void ora_get_dermis(const ora_tissue* t, int32_t* dermis);
/* Triangular lattice: the six neighbours of each membrane particle
 * (Memb_data::memb[6], 6 * nmemb entries). Returns 0, or -1 (nothing
 * written) for a square lattice. */
int ora_get_tri_neighbours(const ora_tissue* t, int32_t* nb);
int ora_error_info(const ora_tissue* t, int32_t* a, int32_t* b, double* value);

/* Cell maps and external-stimulus diffusion on an (nx+1) x (ny+1) x (nz+1)
 * grid (define.h NX, NY, NZ), z fastest: the reference's per-step
 * calc_zzmax, setup_map_lat and calc_ext_stim (epi5_MT/proc.cpp:152-157,
 * map.cpp:24-167, ext_stim.cpp:18-69) on the tissue's current positions. */
typedef struct ora_field ora_field;
ora_field* ora_field_new(const ora_tissue* t, int32_t nx, int32_t ny, int32_t nz);
void ora_field_free(ora_field* f);
int ora_field_step(const ora_tissue* t, ora_field* f, double* zzmax);
/* cmap1: cell index or -1; ext: the current external stimulus */
void ora_field_get(const ora_field* f, int32_t* cmap1, uint8_t* cmap2, double* ext);

#ifdef __cplusplus
}
#endif
#endif
