// Internal launch interface of the mechanics kernels (not part of the C ABI).
#pragma once
#include "epi_common.cuh"

namespace epi {

// Half-open particle and bin ranges a launch covers: the whole batch, or one
// tissue for the unbatched launch pattern.
struct Range {
  int32_t p0, p1;  // particles [p0, p1)
  int32_t b0, b1;  // bins [b0, b1)
};

struct ScanScratch {
  int32_t* partial;  // ceil(n / kScanTile) entries
  int32_t capacity;
};
constexpr int kScanTile = 2048;

// Kernel classes, for per-class timing.
enum KernelClass : int { KC_FORCE = 0, KC_BIN, KC_SCAN, KC_SCATTER, KC_BINSORT, KC_SEARCH, KC_COUNT };
extern const char* const kKernelClassNames[KC_COUNT];

struct Timer;  // optional per-class CUDA-event recorder (host side)
void timer_begin(Timer* tm, int cls, cudaStream_t s);
void timer_end(Timer* tm, int cls, cudaStream_t s);

// Exclusive scan: out[k] = init + sum(in[0..k)) for k in [0, n], out[n] the total.
void launch_scan(const int32_t* in, int32_t* out, int32_t n, int32_t init,
                 const ScanScratch& sc, cudaStream_t s);

// connect_cell: bin -> scan -> scatter -> per-bin sort -> neighbour search.
void launch_connect(const DevState& S, const Range& r, int precision, const ScanScratch& sc,
                    cudaStream_t s, Timer* tm);
// cell_interaction + pos_copy + cell_pos_periodic_fix (writes S.pos_nxt).
void launch_interact_commit(const DevState& S, const Range& r, int precision, cudaStream_t s,
                            Timer* tm);

// CSR export of the connection lists (tissue-local indices, rows sorted).
void launch_rowlen(const DevState& S, int32_t* rowlen, int32_t n, cudaStream_t s);
void launch_fill_csr(const DevState& S, const int32_t* rowoff, int32_t* idx, int32_t n,
                     cudaStream_t s);
void launch_dermis_local(const DevState& S, int32_t* out, int32_t n, cudaStream_t s);
void launch_unpack_positions(const DevState& S, double* x, double* y, double* z, int32_t n,
                             cudaStream_t s);
void launch_pack_positions(const DevState& S, const double* x, const double* y,
                           const double* z, int32_t n, cudaStream_t s);

}  // namespace epi
