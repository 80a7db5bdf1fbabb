// Internal launch interface of the mechanics kernels (not part of the C ABI).
#pragma once
#include "epi_common.cuh"

namespace epi {

// Half-open particle, bin and tissue ranges a launch covers: the whole batch,
// or one tissue for the unbatched launch pattern.
struct Range {
  int32_t p0, p1;  // particles
  int32_t b0, b1;  // bins
  int32_t t0, t1;  // tissues
};

struct ScanScratch {
  int32_t* partial;  // ceil(n / kScanTile) entries
  int32_t capacity;
};
constexpr int kScanTile = 2048;

struct LaunchCfg {
  int num_sms;      // grid-stride kernels use a few blocks per SM
  int block;        // threads per block of the grid-stride kernels
  int simple;       // batch holds only ALIVE / DEAD / AIR / MEMB, no pairs
  int any_old;      // some cell is older than THRESH_SP
  int variant;      // step-kernel instantiation (pipeline depth / residency), see epi_config
  int search_switch;  // rebuilt particles from which the search takes a thread per particle
};

// Kernel classes, for per-class timing.
enum KernelClass : int {
  KC_STEP = 0, KC_PREPASS, KC_REBUILD_BIN, KC_REBUILD_SCAN, KC_REBUILD_SORT,
  KC_REBUILD_SEARCH, KC_GATE, KC_COUNT
};
extern const char* const kKernelClassNames[KC_COUNT];

struct Timer;  // optional per-class CUDA-event recorder (host side)
void timer_begin(Timer* tm, int cls, cudaStream_t s);
void timer_end(Timer* tm, int cls, cudaStream_t s);

// Exclusive scan: out[k] = init + sum(in[0..k)) for k in [0, n], out[n] the
// total. When gate is non-null the kernels do nothing unless *gate != 0.
void launch_scan(const int32_t* in, int32_t* out, int32_t n, int32_t init,
                 const ScanScratch& sc, const int32_t* gate, const LaunchCfg& lc,
                 cudaStream_t s);

// Verlet candidate rebuild of every tissue of r whose gate is set (all
// kernels exit at once when none is): work list -> bin -> scan -> scatter ->
// per-bin sort -> candidate search (which also resets the listed gates).
// listed: the work list was already built (launch_rebuild_condition).
void launch_rebuild(const DevState& S, const Range& r, const ScanScratch& sc,
                    const LaunchCfg& lc, cudaStream_t s, Timer* tm, bool listed = false);
// Membrane bending scratch (_memb_bend_calc1) and dermis (find_dermis) for
// prep entries [m0, m1) (membrane role) and [f0, f1) (FIX / MUSUME role).
void launch_prepass(const DevState& S, int32_t m0, int32_t m1, int32_t f0, int32_t f1,
                    int precision, const LaunchCfg& lc, cudaStream_t s, Timer* tm);
// The two halves of launch_prepass: the membrane sums of prep[m0, m1) (reads
// positions only, so it may run beside a candidate rebuild) and the dermis of
// the FIX / MUSUME cells prep[f0, f1) (reads the candidate lists).
void launch_memb_force(const DevState& S, int32_t m0, int32_t m1, int precision,
                       const LaunchCfg& lc, cudaStream_t s, Timer* tm);
void launch_dermis(const DevState& S, int32_t f0, int32_t f1, const LaunchCfg& lc,
                   cudaStream_t s, Timer* tm);
// cell_interaction + pos_copy + cell_pos_periodic_fix from the current
// positions into S.pos_nxt; flags tissues whose particles moved more than
// skin/2 since their last rebuild.
void launch_step(const DevState& S, const Range& r, int precision, const LaunchCfg& lc,
                 cudaStream_t s, Timer* tm);
// Exact connection lists (connect_cell's result) into S.nbr / S.nn.
void launch_exact_lists(const DevState& S, const Range& r, const LaunchCfg& lc,
                        cudaStream_t s);
void launch_set_gates(const DevState& S, int32_t ntissues, cudaStream_t s);
// Builds the rebuild work list of r's flagged tissues and sets conditional
// handle h to (the list is not empty).
void launch_rebuild_condition(const DevState& S, const Range& r, cudaGraphConditionalHandle h,
                              cudaStream_t s);
// WHILE-node bookkeeping of the step graph: set the number of passes left,
// and decrement it at the end of a pass (setting h to "more passes").
void launch_set_counter(int32_t* remaining, int32_t value, cudaStream_t s);
void launch_loop_tick(int32_t* remaining, cudaGraphConditionalHandle h,
                      unsigned long long* launches, cudaStream_t s);

// CSR export of the connection lists (tissue-local indices, rows sorted).
void launch_rowlen(const DevState& S, int32_t* rowlen, int32_t n, cudaStream_t s);
void launch_fill_csr(const DevState& S, const int32_t* rowoff, int32_t* idx, int32_t n,
                     cudaStream_t s);
void launch_dermis_local(const DevState& S, int32_t* out, int32_t n, cudaStream_t s);
void launch_unpack_positions(const DevState& S, double* x, double* y, double* z, int32_t n,
                             cudaStream_t s);
void launch_pack_positions(const DevState& S, const double* x, const double* y,
                           const double* z, int32_t n, cudaStream_t s);
// Host step, particles [p0, p1): staged positions into both buffers with the
// displacement test (pack_gate); positions of S.pos_cur out to staging.
void launch_pack_gate(const DevState& S, const double* x, const double* y, const double* z,
                      int32_t p0, int32_t p1, const LaunchCfg& lc, cudaStream_t s);
void launch_unpack_range(const DevState& S, double* x, double* y, double* z, int32_t p0,
                         int32_t p1, const LaunchCfg& lc, cudaStream_t s);
// FP32 copies of the current positions (S.posf_cur from S.pos_cur).
void launch_posf(const DevState& S, const LaunchCfg& lc, cudaStream_t s);

// ---- cell maps and external-stimulus diffusion (FP64) ----
struct FieldDev {   // one tissue's grid
  int64_t base;     // first grid point of the tissue in the field arrays
  int32_t nx, ny, nz, irx, iry, irz;
  double dx, dy, dz, inv_dx, inv_dy, inv_dz;
};
struct FieldState {
  const FieldDev* fd;  // per tissue
  int32_t* cmap1;      // tissue-local cell index + 1 (0: none)
  uint8_t* cmap2;      // the ALIVE / FIX / MUSUME mask
  const double* cur;   // external stimulus, current
  double* nxt;         // external stimulus, next
  double* zzmax;       // per tissue
  int32_t* izb;        // per tissue: grid planes below the diffusion's z bound
  int64_t nvox;        // grid points over all tissues
  const double* agek;  // per particle
};
// Grid spacing and stamp radii of a tissue's (nx+1) x (ny+1) x (nz+1) grid.
void field_params(FieldDev& F, double lx, double ly, double lz, int32_t nx, int32_t ny,
                  int32_t nz);
// zzmax, cell maps, external-stimulus update into FS.nxt (the caller swaps).
// wmax: the widest stamp window over the batch's tissues, 2 (2 irx) + 1.
void launch_field_step(const DevState& S, const FieldState& FS, int32_t wmax,
                       const LaunchCfg& lc, cudaStream_t s);

// ---- reverse-mode adjoint (FP64), membrane + ALIVE / DEAD / AIR tissues ----
struct AdjointBuffers {
  const double4* lam_in;  // dL/dX_{t+1}
  double4* lam_out;       // dL/dX_t
  double4* bend;          // 13 bending-product slots per membrane particle
  double4* madj;          // lattice + wall product per membrane particle
  double4* gmemb;         // membrane parameter partials
  double4* gpart;         // per-particle parameter partials (spring, eps, bend, loss)
};
// Sets the gate of every tissue with a particle farther than skin/2 from
// its last rebuild position.
void launch_gate_check(const DevState& S, const LaunchCfg& lc, cudaStream_t s);
// lambda_T and the loss terms (gpart.w) of L_t = inv_cnt[t] sum |X - X*|^2;
// target holds x | y | z (3 n doubles).
void launch_adjoint_seed(const DevState& S, const double* target, int32_t cells_only,
                         const double* inv_cnt, double4* lam, double4* gpart,
                         const LaunchCfg& lc, cudaStream_t s);
// One backward step at positions S.pos_cur (lists: exact predicate over the
// current candidates, which must be valid for S.pos_cur).
void launch_adjoint_step(const DevState& S, const AdjointBuffers& B, const LaunchCfg& lc,
                         cudaStream_t s);
// acc[4 t + c] += per-tissue sums of gpart (fixed order: deterministic).
void launch_tissue_sum(const DevState& S, const double4* gpart, double* acc, const LaunchCfg& lc,
                       cudaStream_t s);

}  // namespace epi
