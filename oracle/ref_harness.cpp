// Harness around the UNMODIFIED epi5_MT mechanics sources (test infrastructure).
//
// This file is the oracle's driver, not product code. It is compiled together
// with the reference's own cellmanager.cpp / cell.cpp / cell_connection.cpp /
// cell_interaction.cpp / cell_init.cpp (see oracle/build_ref.py) and replaces
// only the reference's proc() loop, which stops on an interactive stdin prompt
// (epi5_MT/proc.cpp:100-118). The step it runs is the reference's
// cell_dynamics (epi5_MT/proc.cpp:22-32) without cell_state_renew:
//     cell_interaction -> pos_copy -> cell_pos_periodic_fix -> connect_cell
// Initialisation is the reference's cman_init (epi5_MT/cell_init.cpp:132-142),
// which loads the text cell file, wires the membrane lattice and runs the
// first connect_cell.
//
// Modes:
//   ref_harness run  <cells.dat> <nsteps> <out.bin> <dump_every>
//       writes frames (positions, per-cell sorted connection lists, dermis)
//       at step 0, every dump_every steps and at the last step.
//   ref_harness dyn  <cells.dat> <nsteps> <out.bin> <dump_every>
//       the same with the reference's complete cell_dynamics
//       (epi5_MT/proc.cpp:22-32): cell_interaction -> pos_copy ->
//       cell_state_renew -> cell_pos_periodic_fix -> connect_cell, so cells
//       divide, cornify and are removed (frames then differ in size).
//   ref_harness field <cells.dat> <nsteps> <out.bin> <dump_every>
//       after each mechanics step, the rest of the reference's per-step loop
//       up to the chemistry (epi5_MT/proc.cpp:152-157): zzmax, the cell maps
//       (setup_map_lat, map.cpp:24-167) and the external-stimulus diffusion
//       (calc_ext_stim, ext_stim.cpp:18-69); writes field frames (positions,
//       zzmax, cell map as cell indices, mask map, external stimulus).
//   ref_harness time <cells.dat> <warmup> <steps>
//       times each step with steady_clock and prints one JSON line.
//   ref_harness time_field <cells.dat> <warmup> <steps>
//       the same for the field part of the step only (zzmax, cell maps,
//       external-stimulus update), each after a mechanics step.
//
// genrand_real (epi5_MT/Random_gen.cpp) seeds itself from std::random_device,
// so no two runs of the reference agree once a division test draws from it.
// The harness builds leave Random_gen.cpp out and define genrand_real here:
// a std::mt19937_64 with a fixed seed (EPI_HARNESS_SEED, default 1) and the
// same uniform [0, 1) distribution, or, with EPI_HARNESS_RNG=zero, always 0
// (every division test that is reached passes), so that two builds see the
// same draws.
#include "cellmanager.h"
#include "cell.h"
#include "cell_connection.h"
#include "cell_interaction.h"
#include "cell_init.h"
#include "cell_state_renew.h"
#include "Random_gen.h"
#include "ext_stim.h"
#include "map.h"
#include "swapdata.h"
#include "utils.h"

#include <tbb/tbb_shim_config.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fcntl.h>
#include <memory>
#include <random>
#include <string>
#include <unistd.h>
#include <unordered_set>
#include <vector>

double genrand_real() {
  static thread_local bool zero = [] {
    const char* m = std::getenv("EPI_HARNESS_RNG");
    return m && std::strcmp(m, "zero") == 0;
  }();
  static thread_local std::mt19937_64 mt([] {
    const char* v = std::getenv("EPI_HARNESS_SEED");
    return (std::mt19937_64::result_type)(v ? std::strtoull(v, nullptr, 10) : 1ull);
  }());
  static thread_local std::uniform_real_distribution<double> dist(0.0, 1.0);
  return zero ? 0.0 : dist(mt);
}

namespace {

// cman_init prints one line per loaded cell; keep the harness output clean.
struct SilenceStdout {
  int saved = -1;
  SilenceStdout() {
    std::fflush(stdout);
    saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    dup2(devnull, 1);
    close(devnull);
  }
  ~SilenceStdout() {
    std::fflush(stdout);
    dup2(saved, 1);
    close(saved);
  }
};

// Built with NDEBUG (the loader's DER-first assert rejects DER-free inputs),
// so re-check the per-cell connection capacity the reference asserts on
// (cell_connection.cpp:122, N2 = 400).
void check_capacity(CellManager& cman) {
  bool bad = false;
  cman.all_foreach([&](Cell* c) {
    if (c->connected_cell.size() >= 400) bad = true;
  });
  if (bad) {
    std::fprintf(stderr, "connection list overflow (>= 400)\n");
    std::exit(4);
  }
}

void one_step(CellManager& cman) {
  cell_interaction(cman);
  pos_copy(cman);
  cell_pos_periodic_fix(cman);
  connect_cell(cman);
}

// cell_dynamics, epi5_MT/proc.cpp:22-32
void dynamics_step(CellManager& cman) {
  cell_interaction(cman);
  pos_copy(cman);
  cell_state_renew(cman);
  cell_pos_periodic_fix(cman);
  connect_cell(cman);
}

// CellManager keeps its cell array private; the public loop accessor
// (epi5_MT/cellmanager.h:15-21, all_foreach_with_index) gives index order.
std::vector<Cell*> cells_of(CellManager& cman) {
  std::vector<Cell*> v(cman.size(), nullptr);
  cman.all_foreach_with_index([&](Cell* c, size_t i) { v[i] = c; });
  return v;
}

void write_frame(std::FILE* f, CellManager& cman, int step) {
  const std::vector<Cell*> cells = cells_of(cman);
  const int32_t n = static_cast<int32_t>(cells.size());
  const int32_t tag = 0x454d5246;  // "FRME"
  std::fwrite(&tag, 4, 1, f);
  std::fwrite(&step, 4, 1, f);
  std::fwrite(&n, 4, 1, f);
  std::vector<double> buf(n);
  for (int32_t i = 0; i < n; ++i) buf[i] = cells[i]->x();
  std::fwrite(buf.data(), 8, n, f);
  for (int32_t i = 0; i < n; ++i) buf[i] = cells[i]->y();
  std::fwrite(buf.data(), 8, n, f);
  for (int32_t i = 0; i < n; ++i) buf[i] = cells[i]->z();
  std::fwrite(buf.data(), 8, n, f);
  std::vector<int32_t> off(n + 1, 0), idx, dermis(n, -1);
  for (int32_t i = 0; i < n; ++i) {
    Cell* c = cells[i];
    std::vector<int32_t> row;
    for (size_t k = 0; k < c->connected_cell.size(); ++k)
      row.push_back(static_cast<int32_t>(c->connected_cell[k]->get_index()));
    std::sort(row.begin(), row.end());
    idx.insert(idx.end(), row.begin(), row.end());
    off[i + 1] = static_cast<int32_t>(idx.size());
    if (c->dermis() != nullptr) dermis[i] = static_cast<int32_t>(c->dermis()->get_index());
  }
  std::fwrite(off.data(), 4, n + 1, f);
  if (!idx.empty()) std::fwrite(idx.data(), 4, idx.size(), f);
  std::fwrite(dermis.data(), 4, n, f);
}

// Gap-junction bookkeeping of every cell, as gj_refresh leaves it
// (epi5_MT/cell_connection.cpp:133-152; read by ca2p.cpp:204-207): per cell,
// the number of map keys that point to a live cell, the number that do not
// (the reference keeps keys of removed cells until CellManager::clean_up),
// then (partner index, value, checked) of the live ones sorted by index.
// Keys of removed cells are never dereferenced.
void write_gj(std::FILE* f, CellManager& cman, int step) {
  const std::vector<Cell*> cells = cells_of(cman);
  const int32_t n = static_cast<int32_t>(cells.size());
  std::unordered_set<const Cell*> live(cells.begin(), cells.end());
  const int32_t tag = 0x504d4a47;  // "GJMP"
  std::fwrite(&tag, 4, 1, f);
  std::fwrite(&step, 4, 1, f);
  std::fwrite(&n, 4, 1, f);
  for (int32_t i = 0; i < n; ++i) {
    struct Entry {
      int32_t idx;
      int32_t checked;
      double value;
    };
    std::vector<Entry> row;
    int32_t dead = 0;
    for (auto& kv : cells[i]->gj) {
      if (!live.count(kv.first)) {
        ++dead;
        continue;
      }
      row.push_back({static_cast<int32_t>(kv.first->get_index()), kv.second.is_checked() ? 1 : 0,
                     kv.second()});
    }
    std::sort(row.begin(), row.end(), [](const Entry& a, const Entry& b) { return a.idx < b.idx; });
    const int32_t m = static_cast<int32_t>(row.size());
    std::fwrite(&m, 4, 1, f);
    std::fwrite(&dead, 4, 1, f);
    for (const Entry& e : row) {
      std::fwrite(&e.idx, 4, 1, f);
      std::fwrite(&e.checked, 4, 1, f);
      std::fwrite(&e.value, 8, 1, f);
    }
  }
}

// Highest z of a DEAD / ALIVE / MUSUME / FIX cell, 0 if none: the zzmax the
// reference's loop computes before its maps (calc_zzmax, proc.cpp:34-43).
double highest_cell_z(CellManager& cman) {
  double zmax = 0;
  cman.other_foreach([&](Cell* c) {
    const CELL_STATE st = c->state;
    if ((st == DEAD || st == ALIVE || st == MUSUME || st == FIX) && c->z() > zmax) zmax = c->z();
  });
  return zmax;
}

struct FieldState {
  std::unique_ptr<FArr3D<const Cell*>> map1{new FArr3D<const Cell*>()};
  std::unique_ptr<FArr3D<cmask_ty>> map2{new FArr3D<cmask_ty>()};
  std::unique_ptr<SwapData<FArr3D<double>>> ext{new SwapData<FArr3D<double>>()};
};

void write_field_frame(std::FILE* f, CellManager& cman, int step, double zzmax, FieldState& F) {
  const std::vector<Cell*> cells = cells_of(cman);
  const int32_t n = static_cast<int32_t>(cells.size());
  const int32_t dims[3] = {(int32_t)cont::NX + 1, (int32_t)cont::NY + 1, (int32_t)cont::NZ + 1};
  const int32_t tag = 0x46444C46;  // "FLDF"
  std::fwrite(&tag, 4, 1, f);
  std::fwrite(&step, 4, 1, f);
  std::fwrite(&n, 4, 1, f);
  std::fwrite(dims, 4, 3, f);
  std::fwrite(&zzmax, 8, 1, f);
  std::vector<double> buf(n);
  for (int32_t i = 0; i < n; ++i) buf[i] = cells[i]->x();
  std::fwrite(buf.data(), 8, n, f);
  for (int32_t i = 0; i < n; ++i) buf[i] = cells[i]->y();
  std::fwrite(buf.data(), 8, n, f);
  for (int32_t i = 0; i < n; ++i) buf[i] = cells[i]->z();
  std::fwrite(buf.data(), 8, n, f);
  const size_t nv = (size_t)dims[0] * dims[1] * dims[2];
  std::vector<int32_t> m1(nv);
  std::vector<uint8_t> m2(nv);
  std::vector<double> ex(nv);
  size_t v = 0;
  for (int32_t a = 0; a < dims[0]; ++a)
    for (int32_t b = 0; b < dims[1]; ++b)
      for (int32_t c = 0; c < dims[2]; ++c, ++v) {
        const Cell* p = (*F.map1)()[a][b][c];
        m1[v] = p ? static_cast<int32_t>(p->get_index()) : -1;
        m2[v] = static_cast<uint8_t>((*F.map2)()[a][b][c]);
        ex[v] = F.ext->first()()[a][b][c];
      }
  std::fwrite(m1.data(), 4, nv, f);
  std::fwrite(m2.data(), 1, nv, f);
  std::fwrite(ex.data(), 8, nv, f);
}

int usage() {
  std::fprintf(stderr,
               "usage: ref_harness run <cells.dat> <nsteps> <out.bin> <dump_every>\n"
               "       ref_harness dyn <cells.dat> <nsteps> <out.bin> <dump_every>\n"
               "       ref_harness field <cells.dat> <nsteps> <out.bin> <dump_every>\n"
               "       ref_harness time <cells.dat> <warmup> <steps>\n");
  return 2;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 2) return usage();
  const std::string mode = argv[1];
  auto cman = std::unique_ptr<CellManager>(new CellManager());
  if ((mode == "run" || mode == "dyn") && argc == 6) {
    const bool dyn = mode == "dyn";
    const int nsteps = std::atoi(argv[3]);
    const int every = std::max(1, std::atoi(argv[5]));
    {
      SilenceStdout quiet;
      cman_init(*cman, argv[2]);
    }
    std::FILE* f = std::fopen(argv[4], "wb");
    if (!f) return 3;
    // EPI_HARNESS_GJ=<path>: the gap-junction maps beside every frame
    const char* gj_path = std::getenv("EPI_HARNESS_GJ");
    std::FILE* g = gj_path ? std::fopen(gj_path, "wb") : nullptr;
    if (gj_path && !g) return 3;
    check_capacity(*cman);
    write_frame(f, *cman, 0);
    if (g) write_gj(g, *cman, 0);
    for (int s = 1; s <= nsteps; ++s) {
      if (dyn) {
        SilenceStdout quiet;  // state renewal reports every division / cornification
        dynamics_step(*cman);
      } else {
        one_step(*cman);
      }
      check_capacity(*cman);
      if (s % every == 0 || s == nsteps) {
        write_frame(f, *cman, s);
        if (g) write_gj(g, *cman, s);
      }
    }
    std::fclose(f);
    if (g) std::fclose(g);
    return 0;
  }
  if (mode == "field" && argc == 6) {
    const int nsteps = std::atoi(argv[3]);
    const int every = std::max(1, std::atoi(argv[5]));
    {
      SilenceStdout quiet;
      cman_init(*cman, argv[2]);
    }
    init_precalc_lat();
    init_precalc_per();
    FieldState F;
    std::FILE* f = std::fopen(argv[4], "wb");
    if (!f) return 3;
    for (int s = 1; s <= nsteps; ++s) {
      one_step(*cman);
      check_capacity(*cman);
      const double zzmax = highest_cell_z(*cman);
      setup_map_lat(*cman, *F.map1, *F.map2);
      calc_ext_stim(*F.ext, *F.map1, *F.map2, zzmax);
      if (s % every == 0 || s == nsteps) write_field_frame(f, *cman, s, zzmax, F);
    }
    std::fclose(f);
    return 0;
  }
  if (mode == "time_field" && argc == 5) {
    const int warmup = std::atoi(argv[3]);
    const int steps = std::atoi(argv[4]);
    {
      SilenceStdout quiet;
      cman_init(*cman, argv[2]);
    }
    init_precalc_lat();
    init_precalc_per();
    FieldState F;
    std::vector<double> t(steps);
    for (int s = 0; s < warmup + steps; ++s) {
      one_step(*cman);
      auto a = std::chrono::steady_clock::now();
      const double zzmax = highest_cell_z(*cman);
      setup_map_lat(*cman, *F.map1, *F.map2);
      calc_ext_stim(*F.ext, *F.map1, *F.map2, zzmax);
      auto b = std::chrono::steady_clock::now();
      if (s >= warmup) t[s - warmup] = std::chrono::duration<double>(b - a).count();
    }
    std::vector<double> sorted = t;
    std::sort(sorted.begin(), sorted.end());
    std::printf("{\"cells\": %zu, \"steps\": %d, \"threads\": %d, \"median_s\": %.9g, "
                "\"grid\": [%zu, %zu, %zu]}\n",
                cman->size(), steps, tbb::shim_threads(), steps > 0 ? sorted[steps / 2] : 0.0,
                (size_t)cont::NX, (size_t)cont::NY, (size_t)cont::NZ);
    return 0;
  }
  if (mode == "time" && argc == 5) {
    const int warmup = std::atoi(argv[3]);
    const int steps = std::atoi(argv[4]);
    {
      SilenceStdout quiet;
      cman_init(*cman, argv[2]);
    }
    for (int s = 0; s < warmup; ++s) one_step(*cman);
    std::vector<double> t(steps);
    for (int s = 0; s < steps; ++s) {
      auto a = std::chrono::steady_clock::now();
      one_step(*cman);
      auto b = std::chrono::steady_clock::now();
      t[s] = std::chrono::duration<double>(b - a).count();
    }
    std::vector<double> sorted = t;
    std::sort(sorted.begin(), sorted.end());
    double total = 0;
    for (double v : t) total += v;
    const double median = steps > 0 ? sorted[steps / 2] : 0.0;
    std::printf(
        "{\"cells\": %zu, \"steps\": %d, \"warmup\": %d, \"threads\": %d, "
        "\"median_s\": %.9g, \"mean_s\": %.9g, \"total_s\": %.9g}\n",
        cman->size(), steps, warmup, tbb::shim_threads(), median,
        steps > 0 ? total / steps : 0.0, total);
    return 0;
  }
  return usage();
}
