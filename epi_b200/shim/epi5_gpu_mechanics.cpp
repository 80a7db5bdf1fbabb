// Drop-in GPU mechanics for epi5_MT.
//
// Build this file into epi5_MT in place of the reference's
// cell_connection.cpp and cell_interaction.cpp (epi5_MT.pro SOURCES) and link
// libepi_mech.so. It defines the two functions those files export, with the
// reference's signatures (epi5_MT/cell_connection.h:3,
// epi5_MT/cell_interaction.h:5), so cell_dynamics (epi5_MT/proc.cpp:22-32)
// and cman_init (epi5_MT/cell_init.cpp:132-137) run unchanged:
//
//   connect_cell(cman)      uploads the CellManager's cells (state renewal may
//                           have changed them), connects on the GPU, and
//                           writes back what the rest of the program reads:
//                           connected_cell (membrane rows keep their four
//                           lattice links first), the gap-junction map
//                           bookkeeping of gj_refresh, and dermis.
//   cell_interaction(cman)  runs interaction + commit + wrap on the GPU from
//                           the state of the last connect_cell and stores the
//                           new, unwrapped positions in each coordinate's
//                           next value; the reference's own pos_copy and
//                           cell_pos_periodic_fix then commit and wrap them.
//
// Errors end the program with the library's message and exit(1), as the
// reference's asserts and aborts do. EPI_MECH_PRECISION=fp64 selects FP64
// forces (default: FP32 forces, FP64 sums and positions); EPI_MECH_DEVICE
// selects the GPU.
//
// The host work around the library calls -- gathering the cells, writing
// connected_cell, the gap-junction maps and dermis back, storing the new
// positions -- touches each cell's own members only, so built with OpenMP
// (-fopenmp) its per-cell loops run on all host threads; without it they
// run serially and give the same result. Rows and gap-junction maps of
// cells whose partners did not change since the last connect are left as
// they are (they already hold what a rewrite would give).
#include "cell.h"
#include "cell_connection.h"
#include "cell_interaction.h"
#include "cellmanager.h"
#include "define.h"
#include "epi_mech.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <vector>

namespace {

class GpuMechanics {
 public:
  void connect(CellManager& cman) {
    gather(cman);
    check(epi_upload(ctx(), 1, &view_, &params_), "connect_cell");
    const int32_t n = view_.n;
    off_.resize(n + 1);
    // one export per step: the index buffer keeps the last step's size plus
    // a margin, and only a list that outgrew it asks a second time
    if (idx_.size() < 8 * (size_t)n) idx_.resize(8 * (size_t)n);
    int64_t total = 0;
    const int rc = epi_get_connections(ctx_, off_.data(), idx_.data(), (int64_t)idx_.size(),
                                       &total);
    if (rc == EPI_ERR_INVALID_ARG && total > (int64_t)idx_.size()) {
      idx_.resize((size_t)(total + total / 4));
      check(epi_get_connections(ctx_, off_.data(), idx_.data(), (int64_t)idx_.size(), &total),
            "connect_cell");
    } else {
      check(rc, "connect_cell");
    }
    dermis_.assign(n, -1);
    check(epi_get_dermis(ctx_, dermis_.data()), "connect_cell");
    const size_t nprev = prev_cells_.size();
#pragma omp parallel for schedule(dynamic, 256)
    for (int32_t i = 0; i < n; ++i) {
      Cell* c = cells_[i];
      // connected_cell: the lattice links _memb_init pushed stay first
      // (cellmanager.cpp:70-166), then the listed partners; rewritten only
      // where it differs from that
      const size_t first = c->state == MEMB ? cont::MEMB_ADJ_CONN_NUM : 0;
      auto lattice = [&](Cell* o) {
        bool l = false;
        for (size_t m = 0; m < first; ++m) l |= c->connected_cell[m] == o;
        return l;
      };
      size_t pos = first;
      bool same = c->connected_cell.size() >= first;
      for (int32_t k = off_[i]; same && k < off_[i + 1]; ++k) {
        Cell* o = cells_[idx_[k]];
        if (lattice(o)) continue;
        same = pos < c->connected_cell.size() && c->connected_cell[pos] == o;
        ++pos;
      }
      if (!same || pos != c->connected_cell.size()) {
        c->connected_cell.force_set_count(first);
        for (int32_t k = off_[i]; k < off_[i + 1]; ++k) {
          Cell* o = cells_[idx_[k]];
          if (!lattice(o)) c->connected_cell.push_back(o);
        }
      }
      // gj_refresh (cell_connection.cpp:133-152): mark the connected, reset
      // the rest. After a refresh the connected entries are marked and all
      // others reset, and only this refresh changes marks or touches entries
      // of cells not connected (the chemistry updates connected ones,
      // ca2p.cpp:204-207), so a cell that is the same object at the same
      // index with the same partners as at the last connect keeps its map.
      bool kept = (size_t)i < nprev && prev_cells_[i] == c &&
                  prev_off_[i + 1] - prev_off_[i] == off_[i + 1] - off_[i];
      for (int32_t k = 0; kept && k < off_[i + 1] - off_[i]; ++k)
        kept = prev_row_[prev_off_[i] + k] == cells_[idx_[off_[i] + k]];
      if (!kept) {
        for (auto& kv : c->gj) kv.second.uncheck();
        c->connected_cell.foreach([&](Cell* o) { c->gj[o].check(); });
        for (auto& kv : c->gj)
          if (!kv.second.is_checked()) kv.second.reset();
      }
      // set_dermis (:178-185), FIX and MUSUME only
      if (c->state == FIX || c->state == MUSUME)
        c->set_dermis(dermis_[i] >= 0 ? cells_[dermis_[i]] : nullptr);
    }
    // this connect's rows, for the next one's comparison
    prev_cells_ = cells_;
    prev_off_.assign(off_.begin(), off_.begin() + n + 1);
    prev_row_.resize((size_t)off_[n]);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < (int64_t)off_[n]; ++k) prev_row_[k] = cells_[idx_[k]];
  }

  void interact(CellManager& cman) {
    if (!ctx_ || (size_t)view_.n != cman.size()) connect(cman);
    check(epi_interact_commit(ctx_), "cell_interaction");
    const int32_t n = view_.n;
    nx_.resize(n); ny_.resize(n); nz_.resize(n);
    check(epi_download_positions(ctx_, nx_.data(), ny_.data(), nz_.data()), "cell_interaction");
#pragma omp parallel for schedule(static)
    for (int32_t i = 0; i < n; ++i) {
      Cell* c = cells_[i];
      // The reference runs cell_state_renew between pos_copy and
      // cell_pos_periodic_fix (proc.cpp:23-28), so it sees next positions
      // before the wrap. The library has already wrapped; undo it for the
      // particles that crossed x or y = 0 or L this step. An upward crossing
      // (w = x' - L) is undone exactly; a downward one (w = x' + L) to within
      // an ulp of L, and either way the host's periodic fix then restores w
      // exactly.
      c->x._next() = unwrap(nx_[i], x_[i], view_.lx);
      c->y._next() = unwrap(ny_[i], y_[i], view_.ly);
      c->z._next() = nz_[i];
      // set by _MUSUME_interaction (cell_interaction.cpp:612-618)
      if (c->state == MUSUME) {
        c->spring_force_to_memb = 0;
        if (c->pair && c->pair->state == FIX) c->spring_force_to_memb = params_.kspring;
        else if (c->rest_div_times > 0) c->spring_force_to_memb = params_.kspring_d;
      }
    }
  }

 private:
  // w: wrapped next coordinate, prev: coordinate before the step
  static double unwrap(double w, double prev, double l) {
    if (prev - w > 0.5 * l) return w + l;
    if (w - prev > 0.5 * l) {
      // w = l: x' + l rounded up to l; any negative x' wraps back to it
      const double u = w - l;
      return u < 0 ? u : -std::numeric_limits<double>::denorm_min();
    }
    return w;
  }

  epi_ctx* ctx() {
    if (!ctx_) {
      epi_config cfg;
      epi_config_default(&cfg);
      const char* prec = std::getenv("EPI_MECH_PRECISION");
      if (prec && std::strcmp(prec, "fp64") == 0) cfg.precision = EPI_PREC_FP64;
      const char* dev = std::getenv("EPI_MECH_DEVICE");
      if (dev) cfg.device = std::atoi(dev);
      cfg.max_conn = 128;
      cfg.max_cand = 256;
      check(epi_create(&ctx_, &cfg), "epi_create");
      // constants of define.h; the force constants that lived in
      // cell_interaction.cpp (:21-45) are the library's defaults
      epi_params_default(&params_);
      params_.dt = cont::DT_Cell;
      params_.lj_thresh = cont::LJ_THRESH;
      params_.thresh_sp = cont::THRESH_SP;
      params_.p_memb = 1. / cont::COMPRESS_FACTOR;
      params_.delta_r = 0.4 * cont::R_der;
    }
    return ctx_;
  }

  void gather(CellManager& cman) {
    const size_t n = cman.size();
    cells_.assign(n, nullptr);
    cman.all_foreach_with_index([&](Cell* c, size_t i) { cells_[i] = c; });
    x_.resize(n); y_.resize(n); z_.resize(n); r_.resize(n); agek_.resize(n); spr_.resize(n);
    state_.resize(n); pair_.resize(n); rest_.resize(n);
    int32_t nmemb = 0, nder = 0;
#pragma omp parallel for schedule(static) reduction(+ : nmemb, nder)
    for (size_t i = 0; i < n; ++i) {
      const Cell* c = cells_[i];
      x_[i] = c->x();
      y_[i] = c->y();
      z_[i] = c->z();
      r_[i] = c->radius;
      agek_[i] = c->agek;
      spr_[i] = c->spr_nat_len;
      state_[i] = (uint8_t)c->state;
      pair_[i] = c->pair ? (int32_t)c->pair->get_index() : -1;
      rest_[i] = c->rest_div_times;
      nmemb += c->state == MEMB;
      nder += c->state == DER;
    }
    view_.n = (int32_t)n;
    view_.nmemb = nmemb;
    view_.nder = nder;
    view_.nmx = (int32_t)cont::NMX;
    // rows of the lattice: NMY for the square build; the triangular build
    // wires by NMX and the membrane count only (cellmanager.cpp:70-111)
    view_.nmy = nmemb / (int32_t)cont::NMX;
    view_.lx = cont::LX;
    view_.ly = cont::LY;
    view_.lz = cont::LZ;
    view_.x = x_.data();
    view_.y = y_.data();
    view_.z = z_.data();
    view_.radius = r_.data();
    view_.agek = agek_.data();
    view_.spr_nat_len = spr_.data();
    view_.state = state_.data();
    view_.pair = pair_.data();
    view_.rest_div_times = rest_.data();
#ifdef TRI_MEMB
    view_.lattice = EPI_LATTICE_TRIANGULAR;  // define.h:66
#else
    view_.lattice = EPI_LATTICE_SQUARE;
#endif
    view_.reserved = 0;
  }

  void check(int rc, const char* where) {
    if (rc == EPI_OK) return;
    int32_t t = -1, a = -1, b = -1;
    double v = 0;
    if (ctx_) epi_error_info(ctx_, &t, &a, &b, &v);
    std::printf("%s: %s (cell %d, partner %d, value %g)\n", where, epi_strerror(rc), a, b, v);
    std::exit(1);
  }

  epi_ctx* ctx_ = nullptr;
  epi_params params_{};
  epi_tissue_view view_{};
  std::vector<Cell*> cells_;
  std::vector<double> x_, y_, z_, r_, agek_, spr_, nx_, ny_, nz_;
  std::vector<uint8_t> state_;
  std::vector<int32_t> pair_, rest_, off_, idx_, dermis_;
  // the previous connect's cells and rows (partner pointers, CSR)
  std::vector<Cell*> prev_cells_, prev_row_;
  std::vector<int32_t> prev_off_;
};

// One GPU context per process, created on first use. It is not destroyed at
// exit: process teardown releases it.
GpuMechanics& gpu() {
  static GpuMechanics* g = new GpuMechanics();
  return *g;
}

}  // namespace

void connect_cell(CellManager& cman) { gpu().connect(cman); }

void cell_interaction(CellManager& cman) { gpu().interact(cman); }
