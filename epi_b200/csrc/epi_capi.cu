// C ABI of the mechanics library: context, upload, step drivers, export.
//
// Host-side mirror of the reference's call surface (include/epi_mech.h lists
// the reference function each entry point stands for). All device memory is
// owned by the context; every entry point returns an epi_status and catches
// everything so no exception crosses the ABI.
#include "epi_mech.h"
#include "epi_kernels.h"

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

using namespace epi;

namespace epi {

struct Timer {
  struct Pair {
    cudaEvent_t a, b;
  };
  std::vector<Pair> ev[KC_COUNT];
  cudaEvent_t open[KC_COUNT] = {};
  ~Timer() {
    for (auto& v : ev)
      for (auto& p : v) {
        cudaEventDestroy(p.a);
        cudaEventDestroy(p.b);
      }
  }
};

void timer_begin(Timer* tm, int cls, cudaStream_t s) {
  if (!tm) return;
  cudaEventCreate(&tm->open[cls]);
  cudaEventRecord(tm->open[cls], s);
}

void timer_end(Timer* tm, int cls, cudaStream_t s) {
  if (!tm) return;
  cudaEvent_t e;
  cudaEventCreate(&e);
  cudaEventRecord(e, s);
  tm->ev[cls].push_back({tm->open[cls], e});
}

}  // namespace epi

namespace {

// NVTX range over a scope: every entry point and the phases it queues show
// up by name on a profiler's timeline (no cost without a tool attached).
struct Nvtx {
  explicit Nvtx(const char* name) { nvtxRangePushA(name); }
  ~Nvtx() { nvtxRangePop(); }
  Nvtx(const Nvtx&) = delete;
  Nvtx& operator=(const Nvtx&) = delete;
};

// epi_step_host splits the batch into at most this many groups of tissues
// (on the 512-tissue ensemble 4 groups measured 3.31 ms per chained step,
// 6 groups 3.47, 8 groups 3.48 and 16 groups 3.90: fewer, larger copies and
// launch sequences, with successive steps overlapping each other anyway).
constexpr int kHostStepGroups = 4;
// Rebuilt particles from which the candidate search takes one thread per
// particle (epi_config.search_switch = 0).
constexpr int kDefaultSearchSwitch = 48 * 1024;

// Host-side bookkeeping of one tissue in the batch.
struct TissueHost {
  int32_t prep_m;  // offset of its membrane particles in the prep list
  int32_t prep_f;  // offset of its FIX / MUSUME cells in the FIX/MUSUME block
  int32_t nfm;     // number of FIX / MUSUME cells
};

}  // namespace

struct epi_ctx {
  epi_config cfg{};
  cudaStream_t stream = nullptr;
  cudaStream_t side = nullptr;  // captures the bodies of conditional graph nodes
  // the membrane sums run on `aux` beside the candidate rebuild (fork / join)
  cudaStream_t aux = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  LaunchCfg lc{148, 256, 0, 0, 0, kDefaultSearchSwitch};
  bool loaded = false;
  bool lists_fresh = false;  // nbr / nn / dermis match the current positions
  int32_t ntissues = 0;
  int64_t n = 0;
  int32_t nbins = 0;
  int32_t nprep = 0, nprep_memb = 0;
  std::vector<TissueDev> tissues_h;
  // what the candidate lists depend on besides positions, as last uploaded
  // (radius and attribute word per particle), to re-gate only changed tissues
  std::vector<double> h_radius;
  std::vector<uint32_t> h_attr;
  std::vector<TissueHost> thost;
  // device buffers
  TissueDev* tissues = nullptr;
  double4* pos[2] = {nullptr, nullptr};
  float4* posf[2] = {nullptr, nullptr};
  bool posf_stale = true;  // pos[cur] was written outside the step kernel
  int cur = 0;
  uint32_t* attr = nullptr;
  int32_t* pair = nullptr;
  double* spr = nullptr;
  int32_t* dermis = nullptr;
  uint4* cand = nullptr;  // candidate rows, cand_chunks 16-byte chunks per particle
  int32_t cand16 = 1;     // 16-bit row entries (every tissue below 65,537 particles)
  int32_t cand_chunks = 0;
  float4* bpos = nullptr;
  int32_t* nbr = nullptr;
  int32_t* nn = nullptr;
  double4* fmemb = nullptr;
  int32_t* bin = nullptr;
  int32_t* rank = nullptr;
  int32_t* counts = nullptr;
  int32_t* starts = nullptr;
  uint32_t* skey = nullptr;
  float4* spos = nullptr;
  int32_t* gate = nullptr;
  int32_t* rl = nullptr;    // rebuild work list: [count | list (T) | ppre (T+1) | bpre (T+1)]
  int32_t* prep = nullptr;
  double* stage = nullptr;        // 3n doubles: x | y | z for host transfers
  // epi_step_host: copy streams, per-chunk events, the outbound staging (3n)
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  std::vector<cudaEvent_t> ev_in, ev_done, ev_d2h;
  double* stage_out = nullptr;
  // the last work queued on the compute stream was a host step (its inbound
  // staging is then guarded per group, not by the whole stream)
  bool after_host_step = false;
  DevStatus* status = nullptr;
  DevStatus* status_h = nullptr;  // pinned
  // pinned host staging of epi_upload's per-particle arrays (grown on demand)
  unsigned char* upin = nullptr;
  size_t upin_bytes = 0;
  unsigned long long* rebuilds = nullptr;
  int32_t* loop_left = nullptr;  // passes left in the step graph's device loop
  unsigned long long* launches = nullptr;  // step-sequence kernels executed
  ScanScratch scan{};
  // graphs: one per buffer parity, each replaying two steps
  cudaGraphExec_t graph[2] = {nullptr, nullptr};
  // cell maps and external stimulus (epi_field_*)
  double* agek = nullptr;  // per particle, for the stimulus source
  bool field_on = false;
  int32_t fnx = 0, fny = 0, fnz = 0;
  int64_t nvox = 0;
  std::vector<FieldDev> fd_h;
  FieldDev* fd = nullptr;
  int32_t* cmap1 = nullptr;
  uint8_t* cmap2 = nullptr;
  double* ext[2] = {nullptr, nullptr};
  int ext_cur = 0;
  double* zzmax = nullptr;
  int32_t* izb = nullptr;
  // export buffers of epi_get_connections / epi_get_dermis, kept between
  // calls (the drop-in exports every step) and grown on demand
  int32_t* x_rowlen = nullptr;   // n
  int32_t* x_rowoff = nullptr;   // n + 1
  int32_t* x_partial = nullptr;  // scan partials
  int32_t* x_idx = nullptr;      // x_idx_cap entries
  int64_t x_idx_cap = 0;
  int64_t x_n = 0;               // particles the row buffers hold
  // last error details
  DevStatus last{};
};

namespace {

int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return EPI_OK;
  if (e == cudaErrorMemoryAllocation) return EPI_ERR_OOM;
  if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return EPI_ERR_NO_DEVICE;
  return EPI_ERR_CUDA;
}

#define EPI_CUDA(call)                             \
  do {                                             \
    const cudaError_t e_ = (call);                 \
    if (e_ != cudaSuccess) return cuda_status(e_); \
  } while (0)

template <typename T>
int dev_alloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  return cuda_status(cudaMalloc((void**)p, sizeof(T) * count));
}

void destroy_graphs(epi_ctx* c) {
  for (auto& g : c->graph) {
    if (g) cudaGraphExecDestroy(g);
    g = nullptr;
  }
}

void free_field(epi_ctx* c) {
  void* ptrs[] = {c->fd, c->cmap1, c->cmap2, c->ext[0], c->ext[1], c->zzmax, c->izb};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  c->fd = nullptr; c->cmap1 = nullptr; c->cmap2 = nullptr;
  c->ext[0] = c->ext[1] = nullptr; c->zzmax = nullptr; c->izb = nullptr;
  c->field_on = false;
  c->nvox = 0;
  c->fd_h.clear();
}

void free_export(epi_ctx* c) {
  void* ptrs[] = {c->x_rowlen, c->x_rowoff, c->x_partial, c->x_idx};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  c->x_rowlen = c->x_rowoff = c->x_partial = c->x_idx = nullptr;
  c->x_idx_cap = 0;
  c->x_n = 0;
}

void free_buffers(epi_ctx* c) {
  destroy_graphs(c);
  free_field(c);
  free_export(c);
  if (c->agek) cudaFree(c->agek);
  c->agek = nullptr;
  void* ptrs[] = {c->tissues, c->pos[0], c->pos[1], c->posf[0], c->posf[1], c->attr, c->pair, c->spr, c->dermis,
                  c->cand, c->bpos, c->nbr, c->nn, c->fmemb, c->bin,
                  c->rank, c->counts, c->starts, c->skey, c->spos, c->gate, c->rl, c->prep,
                  c->scan.partial, c->stage, c->stage_out};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  c->tissues = nullptr;
  c->pos[0] = c->pos[1] = nullptr;
  c->posf[0] = c->posf[1] = nullptr;
  c->attr = nullptr; c->pair = nullptr; c->spr = nullptr; c->dermis = nullptr;
  c->cand = nullptr; c->bpos = nullptr;
  c->nbr = nullptr; c->nn = nullptr; c->fmemb = nullptr;
  c->bin = nullptr; c->rank = nullptr; c->counts = nullptr; c->starts = nullptr;
  c->skey = nullptr; c->spos = nullptr; c->gate = nullptr; c->rl = nullptr; c->prep = nullptr;
  c->scan.partial = nullptr; c->stage = nullptr; c->stage_out = nullptr;
  c->loaded = false;
  c->lists_fresh = false;
}

DevState make_state(epi_ctx* c, int cur) {
  DevState S;
  S.tissues = c->tissues;
  S.pos_cur = c->pos[cur];
  S.pos_nxt = c->pos[cur ^ 1];
  S.posf_cur = c->posf[cur];
  S.posf_nxt = c->posf[cur ^ 1];
  S.attr = c->attr;
  S.pair = c->pair;
  S.spr = c->spr;
  S.dermis = c->dermis;
  S.cand = c->cand;
  S.cand16 = c->cand16;
  S.bpos = c->bpos;
  S.nbr = c->nbr;
  S.nn = c->nn;
  S.fmemb = c->fmemb;
  S.bin = c->bin;
  S.rank = c->rank;
  S.counts = c->counts;
  S.starts = c->starts;
  S.skey = c->skey;
  S.spos = c->spos;
  S.gate = c->gate;
  S.rl_count = c->rl;
  S.rl_list = c->rl ? c->rl + 1 : nullptr;
  S.rl_ppre = c->rl ? c->rl + 1 + c->ntissues : nullptr;
  S.rl_bpre = c->rl ? c->rl + 2 + 2 * c->ntissues : nullptr;
  S.ntissues = c->ntissues;
  S.prep = c->prep;
  S.nprep = c->nprep;
  S.nprep_memb = c->nprep_memb;
  S.status = c->status;
  S.rebuilds = c->rebuilds;
  S.launches = c->launches;
  S.n_total = c->n;
  S.max_conn = c->cfg.max_conn;
  S.max_cand = c->cfg.max_cand;
  S.skin = c->cfg.skin;
  return S;
}

Range whole(const epi_ctx* c) { return Range{0, (int32_t)c->n, 0, c->nbins, 0, c->ntissues}; }

Range tissue_range(const epi_ctx* c, int t) {
  const TissueDev& T = c->tissues_h[t];
  return Range{T.pbase, T.pbase + T.n, T.binbase, T.binbase + T.anx * T.any * T.anz + 1, t, t + 1};
}

void prepass_all(epi_ctx* c, int cur, Timer* tm) {
  launch_prepass(make_state(c, cur), 0, c->nprep_memb, c->nprep_memb, c->nprep,
                 c->cfg.precision, c->lc, c->stream, tm);
}

void prepass_tissue(epi_ctx* c, int cur, int t) {
  const TissueDev& T = c->tissues_h[t];
  const TissueHost& H = c->thost[t];
  const int32_t f0 = c->nprep_memb + H.prep_f;
  launch_prepass(make_state(c, cur), H.prep_m, H.prep_m + T.nmemb, f0, f0 + H.nfm,
                 c->cfg.precision, c->lc, c->stream, nullptr);
}

// Refreshes the FP32 position copy of the current parity after positions
// were written by anything but the step kernel (upload, restore, ...).
void ensure_posf(epi_ctx* c) {
  if (!c->posf_stale) return;
  launch_posf(make_state(c, c->cur), c->lc, c->stream);
  c->posf_stale = false;
}

// The membrane sums read only positions, so they run on c->aux beside the
// candidate rebuild (whose kernels are short and occupy few SMs): fork_memb
// starts them after the work queued so far, join_memb makes the step kernel
// wait for them. Recorded the same way inside a stream capture, the fork and
// join become edges of the captured graph.
cudaError_t fork_memb(epi_ctx* c, int cur, Timer* tm) {
  if (c->nprep_memb == 0) return cudaSuccess;
  cudaError_t e = cudaEventRecord(c->ev_fork, c->stream);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(c->aux, c->ev_fork, 0);
  if (e != cudaSuccess) return e;
  launch_memb_force(make_state(c, cur), 0, c->nprep_memb, c->cfg.precision, c->lc, c->aux, tm);
  return cudaEventRecord(c->ev_join, c->aux);
}

cudaError_t join_memb(epi_ctx* c) {
  if (c->nprep_memb == 0) return cudaSuccess;
  return cudaStreamWaitEvent(c->stream, c->ev_join, 0);
}

// The dermis of FIX / MUSUME cells reads the candidate lists: after the rebuild.
void dermis_all(epi_ctx* c, int cur, Timer* tm) {
  launch_dermis(make_state(c, cur), c->nprep_memb, c->nprep, c->lc, c->stream, tm);
}

// One reference step over the batch: [rebuild] and the membrane sums side by
// side, the dermis, then the fused step. Errors of the stream calls surface
// at the next synchronising call.
void enqueue_step(epi_ctx* c, int& cur, Timer* tm) {
  ensure_posf(c);
  {
    Nvtx r("membrane sums");
    (void)fork_memb(c, cur, tm);
  }
  {
    Nvtx r("candidate rebuild");
    launch_rebuild(make_state(c, cur), whole(c), c->scan, c->lc, c->stream, tm);
  }
  dermis_all(c, cur, tm);
  (void)join_memb(c);
  {
    Nvtx r("interaction + commit");
    launch_step(make_state(c, cur), whole(c), c->cfg.precision, c->lc, c->stream, tm);
  }
  cur ^= 1;
}

// Whether the step graph puts the candidate rebuild in a conditional node
// that skips its kernels on steps with nothing to rebuild: by default for a
// single tissue (most of its steps rebuild nothing), not for a batch (some
// tissue rebuilds at almost every step, and the node costs more than the
// kernels' early exit).
bool conditional_rebuild(const epi_ctx* c) {
  return c->cfg.rebuild_gate == 1 || (c->cfg.rebuild_gate == 0 && c->ntissues == 1);
}

// Skin, step-kernel variant, candidate-search switch and rebuild node of the
// context; the captured graphs hold them, so they are dropped.
void apply_tuning(epi_ctx* c, double skin, int32_t variant, int32_t search_switch,
                  int32_t rebuild_gate) {
  c->cfg.skin = skin;
  c->cfg.variant = variant;
  c->cfg.search_switch = search_switch;
  c->cfg.rebuild_gate = rebuild_gate;
  c->lc.variant = variant == 0 ? 3 : variant;
  c->lc.search_switch = search_switch > 0 ? search_switch : kDefaultSearchSwitch;
  destroy_graphs(c);
}

// Appends to the graph being captured on c->stream a conditional (IF) node
// whose body, captured on c->side, is the candidate rebuild; a one-block
// kernel before it builds the rebuild work list and sets the condition to
// "the list is not empty", so steps that need no rebuild launch none of the
// rebuild's kernels.
cudaError_t capture_conditional_rebuild(epi_ctx* c, int cur) {
  cudaStreamCaptureStatus st;
  cudaGraph_t g;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  cudaError_t e = cudaStreamGetCaptureInfo(c->stream, &st, nullptr, &g, &deps, &nd);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle h;
  if ((e = cudaGraphConditionalHandleCreate(&h, g, 0, 0)) != cudaSuccess) return e;
  launch_rebuild_condition(make_state(c, cur), whole(c), h, c->stream);
  if ((e = cudaStreamGetCaptureInfo(c->stream, &st, nullptr, &g, &deps, &nd)) != cudaSuccess)
    return e;
  cudaGraphNodeParams p{};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = h;
  p.conditional.type = cudaGraphCondTypeIf;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if ((e = cudaGraphAddNode(&node, g, deps, nd, &p)) != cudaSuccess) return e;
  cudaGraph_t body = p.conditional.phGraph_out[0];
  if ((e = cudaStreamBeginCaptureToGraph(c->side, body, nullptr, nullptr, 0,
                                         cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
    return e;
  launch_rebuild(make_state(c, cur), whole(c), c->scan, c->lc, c->side, nullptr, true);
  if ((e = cudaStreamEndCapture(c->side, &body)) != cudaSuccess) return e;
  return cudaStreamUpdateCaptureDependencies(c->stream, &node, 1,
                                             cudaStreamSetCaptureDependencies);
}

// The step graph of parity cur0: one launch runs a whole sequence of steps.
// A WHILE node repeats its body -- two steps (per step: the membrane sums
// forked beside the conditional rebuild, the dermis, the fused step), then a
// one-thread kernel that
// counts down the passes left (set before each launch) and sets the loop
// condition -- so the device drives the loop and the host launches once.
cudaError_t capture_step_graph(epi_ctx* c, int cur0, cudaGraphExec_t* out) {
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  cudaGraphConditionalHandle hw;
  e = cudaGraphConditionalHandleCreate(&hw, g, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams p{};
  cudaGraphNode_t loop;
  if (e == cudaSuccess) {
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = hw;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    e = cudaGraphAddNode(&loop, g, nullptr, 0, &p);
  }
  if (e == cudaSuccess) {
    cudaGraph_t body = p.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(c->stream, body, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      int cur = cur0;
      for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
        e = fork_memb(c, cur, nullptr);
        if (e == cudaSuccess) {
          if (conditional_rebuild(c))
            e = capture_conditional_rebuild(c, cur);
          else
            launch_rebuild(make_state(c, cur), whole(c), c->scan, c->lc, c->stream, nullptr);
        }
        if (e != cudaSuccess) break;
        dermis_all(c, cur, nullptr);
        if ((e = join_memb(c)) != cudaSuccess) break;
        launch_step(make_state(c, cur), whole(c), c->cfg.precision, c->lc, c->stream, nullptr);
        cur ^= 1;
      }
      if (e == cudaSuccess) launch_loop_tick(c->loop_left, hw, c->launches, c->stream);
      const cudaError_t e_end = cudaStreamEndCapture(c->stream, &body);
      if (e == cudaSuccess) e = e_end;
    }
  }
  // each captured kernel keeps its stream's priority
  if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, cudaGraphInstantiateFlagUseNodePriority);
  cudaGraphDestroy(g);
  return e;
}

// connect_cell's results for the current positions: lists and dermis.
void enqueue_materialize(epi_ctx* c) {
  const DevState S = make_state(c, c->cur);
  launch_rebuild(S, whole(c), c->scan, c->lc, c->stream, nullptr);
  prepass_all(c, c->cur, nullptr);
  launch_exact_lists(S, whole(c), c->lc, c->stream);
}

// Waits for the stream and converts any sticky kernel error to a status.
int check_status(epi_ctx* c) {
  EPI_CUDA(cudaMemcpyAsync(c->status_h, c->status, sizeof(DevStatus), cudaMemcpyDeviceToHost,
                           c->stream));
  EPI_CUDA(cudaStreamSynchronize(c->stream));
  EPI_CUDA(cudaGetLastError());
  if (c->status_h->code != 0) {
    c->last = *c->status_h;
    EPI_CUDA(cudaMemsetAsync(c->status, 0, sizeof(DevStatus), c->stream));
    EPI_CUDA(cudaStreamSynchronize(c->stream));
    return c->last.code;
  }
  return EPI_OK;
}

// nsteps steps replayed from the two-step graph of the current parity
// (both parities' graphs captured on first use), plus one eager step for
// an odd count.
int enqueue_graph_steps(epi_ctx* c, int32_t nsteps) {
  ensure_posf(c);  // never inside the captured graph
  const int32_t pairs = nsteps / 2;
  if (pairs > 0) {
    // both parities' graphs at first use: an odd step count (its last step
    // runs eagerly) leaves the next run on the other parity, whose capture
    // would otherwise hold up that run's first launch
    for (int par = 0; par < 2; ++par)
      if (!c->graph[par]) EPI_CUDA(capture_step_graph(c, par, &c->graph[par]));
    cudaGraphExec_t& ge = c->graph[c->cur];
    launch_set_counter(c->loop_left, pairs, c->stream);
    EPI_CUDA(cudaGraphLaunch(ge, c->stream));
  }
  if (nsteps % 2) enqueue_step(c, c->cur, nullptr);
  if (nsteps > 0) c->lists_fresh = false;
  return EPI_OK;
}

int materialize(epi_ctx* c) {
  if (c->lists_fresh) return EPI_OK;
  enqueue_materialize(c);
  const int rc = check_status(c);
  if (rc == EPI_OK) c->lists_fresh = true;
  return rc;
}

// Every entry point starts here; any work it queues that is not a host step
// ends a chain of host steps (see enqueue_host_step).
int set_device(epi_ctx* c) {
  c->after_host_step = false;
  return cuda_status(cudaSetDevice(c->cfg.device));
}

#define EPI_GUARD_BEGIN try {
#define EPI_GUARD_END             \
  }                               \
  catch (const std::bad_alloc&) { \
    return EPI_ERR_OOM;           \
  }                               \
  catch (...) {                   \
    return EPI_ERR_CUDA;          \
  }

// Smallest non-negative double x <= hi with pred(x) true, for a predicate that
// is false then true as x grows; +inf when pred(hi) is false. Non-negative
// doubles order like their bit patterns, so this bisects on the bits.
template <class F>
double first_true(double hi, F pred) {
  if (!pred(hi)) return INFINITY;
  if (pred(0.0)) return 0.0;
  uint64_t lo_b = 0, hi_b;
  std::memcpy(&hi_b, &hi, 8);
  while (hi_b - lo_b > 1) {
    const uint64_t mid = lo_b + (hi_b - lo_b) / 2;
    double m;
    std::memcpy(&m, &mid, 8);
    if (pred(m)) hi_b = mid;
    else lo_b = mid;
  }
  double r;
  std::memcpy(&r, &hi_b, 8);
  return r;
}

double host_pdiff(double a, double b, double L) {
  const double d = a - b;
  if (d > 0.5 * L) return d - L;
  if (d <= -0.5 * L) return d + L;
  return d;
}

// Range-assert thresholds of grid_init / connect_proc for a wrapped position
// (cell_connection.cpp:44-53, :95-99), evaluated with the same IEEE double
// operations the reference uses.
void range_thresholds(TissueDev& T) {
  const double AG = kAreaGrid;
  auto grid_fails = [&](double v, double L, int32_t an) {
    const int32_t k = (int32_t)((0.5 * L - host_pdiff(0.5 * L, v, L)) / AG);
    return k >= an || k < 0;
  };
  const double below_lx = std::nextafter(T.lx, 0.0), below_ly = std::nextafter(T.ly, 0.0);
  T.gx_hi = first_true(below_lx, [&](double v) { return grid_fails(v, T.lx, T.anx); });
  T.gy_hi = first_true(below_ly, [&](double v) { return grid_fails(v, T.ly, T.any); });
  T.cx_hi = first_true(T.lx, [&](double v) { return (int32_t)(v / AG) >= T.anx; });
  T.cy_hi = first_true(T.ly, [&](double v) { return (int32_t)(v / AG) >= T.any; });
  const double zbig = 4.0 * (T.lz + 4.0);
  T.gz_hi = first_true(zbig, [&](double v) { return (int32_t)(v / AG) >= T.anz; });
  T.cz_hi = T.gz_hi;
  T.cz_lo = -first_true(zbig, [&](double w) { return (int32_t)(w / AG) >= 1; });
}

// FP32 box constants and the band around the connection threshold inside
// which the mixed path defers to the FP64 predicate. With u = 2^-24 (FP32
// unit roundoff), M a bound on |coordinate| and D = LJ_THRESH * 2 rmax the
// longest connection: each coordinate rounds by <= M u, a separation
// component (difference, then possibly +-L) by <= 4 M u =: e; d2 in FP32
// then errs by <= 2 sqrt(3) D e + 3 e^2 + 4 D^2 u, and the FP32 threshold
// LJ_THRESH^2 (r_i + r_j)^2 by <= 9 D^2 u. ftol is twice the sum (plus the
// FP64 predicate's own rounding, far below).
void set_fp32_bounds(TissueDev& T) {
  T.lxf = (float)T.lx;
  T.lyf = (float)T.ly;
  T.ilxf = (float)(1.0 / T.lx);
  T.ilyf = (float)(1.0 / T.ly);
  T.lt2f = (float)(T.P.lj_thresh * T.P.lj_thresh);
  const double u = std::ldexp(1.0, -24);
  const double M = std::max(std::max(T.lx, T.ly), T.lz) + 8.0;
  const double e = 4.0 * M * u;
  const double D = T.P.lj_thresh * 2.0 * T.rmax;
  const double tol = 2.0 * (2.0 * std::sqrt(3.0) * D * e + 3.0 * e * e + 13.0 * D * D * u) +
                     1e-14 * D * D;
  T.ftol = (float)(tol * (1.0 + 1e-3));
}

int validate_tissue(const epi_tissue_view& v, const epi_params& P) {
  if (v.n < 0 || v.nmemb < 0 || v.nder < 0 || v.nmemb + v.nder > v.n) return EPI_ERR_INVALID_ARG;
  if (v.n > 0 && (!v.x || !v.y || !v.z || !v.radius || !v.state)) return EPI_ERR_INVALID_ARG;
  if (!(v.lx > 0) || !(v.ly > 0) || !(v.lz > 0)) return EPI_ERR_INVALID_ARG;
  if (v.nmemb != v.nmx * v.nmy || v.nmx < 3 || v.nmy < 3) return EPI_ERR_UNSUPPORTED;
  if (v.lattice != EPI_LATTICE_SQUARE && v.lattice != EPI_LATTICE_TRIANGULAR)
    return EPI_ERR_INVALID_ARG;
  if (v.reserved != 0) return EPI_ERR_INVALID_ARG;
  // the triangular wiring alternates row offsets: an odd row count breaks
  // the periodic wrap (cellmanager.cpp:95-108)
  if (v.lattice == EPI_LATTICE_TRIANGULAR && v.nmy % 2 != 0) return EPI_ERR_UNSUPPORTED;
  // The 5-bin search window of connect_proc must not wrap onto itself
  // (cell_connection.cpp:101-109), else the reference pushes pairs twice.
  const int anx = (int)(v.lx / 2.0 + 0.5), any = (int)(v.ly / 2.0 + 0.5), anz = (int)(v.lz / 2.0);
  if (anx < 5 || any < 5 || anz < 5) return EPI_ERR_UNSUPPORTED;
  double rmax = 0;
  for (int32_t i = 0; i < v.n; ++i) {
    const uint8_t s = v.state[i];
    if (s > ST_MEMB) return EPI_ERR_INVALID_ARG;
    if ((i < v.nmemb) != (s == ST_MEMB)) return EPI_ERR_INVALID_ARG;
    if (i >= v.nmemb && i < v.nmemb + v.nder && s != ST_DER) return EPI_ERR_INVALID_ARG;
    if (i >= v.nmemb + v.nder && s == ST_DER) return EPI_ERR_INVALID_ARG;
    if (!(v.radius[i] > 0) || !std::isfinite(v.radius[i])) return EPI_ERR_INVALID_ARG;
    if (!std::isfinite(v.x[i]) || !std::isfinite(v.y[i]) || !std::isfinite(v.z[i]))
      return EPI_ERR_NONFINITE;
    rmax = std::max(rmax, v.radius[i]);
    if (v.pair) {
      const int32_t q = v.pair[i];
      if (q >= v.n || q < -1) return EPI_ERR_INVALID_ARG;
      if (q >= 0 && (q == i || v.pair[q] != i || q < v.nmemb || i < v.nmemb))
        return EPI_ERR_INVALID_ARG;
    }
  }
  // Constants: finite; DT > 0; LJ_THRESH > 1 (adhesion divides by
  // (LJ_THRESH - 1)^2, cell_interaction.cpp:113-124).
  const double* pv = reinterpret_cast<const double*>(&P);
  for (size_t k = 0; k < sizeof(epi_params) / sizeof(double); ++k)
    if (!std::isfinite(pv[k])) return EPI_ERR_INVALID_ARG;
  if (!(P.dt > 0) || !(P.lj_thresh > 1.0)) return EPI_ERR_INVALID_ARG;
  // Every pair the reference can connect must lie inside its +-2 bin window:
  // LJ_THRESH * (r_i + r_j) < 2 * AREA_GRID (cell_connection.cpp:92-109).
  if (P.lj_thresh * 2.0 * rmax >= 4.0 - 1e-6) return EPI_ERR_UNSUPPORTED;
  return EPI_OK;
}

}  // namespace

namespace {
// Device allocations released when the call returns.
struct ScopedDeviceMemory {
  std::vector<void*> ptrs;
  ~ScopedDeviceMemory() {
    for (void* p : ptrs) cudaFree(p);
  }
  template <typename T>
  int get(T** p, size_t count) {
    const int rc = dev_alloc(p, count);
    if (rc == EPI_OK) ptrs.push_back(*p);
    return rc;
  }
};
}  // namespace

extern "C" {

void epi_params_default(epi_params* p) {
  if (!p) return;
  p->dt = 0.01;                 // DT_Cell, define.h:86
  p->eps_m = 0.01;              // cell_interaction.cpp:21
  p->p_memb = 1. / 4;           // 1 / COMPRESS_FACTOR, :26 and define.h:125
  p->der_der_const = 0.2;       // :29
  p->k_total = 3.0;             // :30
  p->k_desmosome = 3.0 * 0.01;  // K_TOTAL * K_DESMOSOME_RATIO, :31-32
  p->kspring = 25.0;            // :33
  p->kspring_d = 5.0;           // :34
  p->kbend = 0.5;               // :37
  p->delta_r = 0.4 * 1.4;       // 0.4 * R_der, :42
  p->para_ljp2 = 0.005;         // :44
  p->kspring_division = 5.0;    // :45
  p->lj_thresh = 1.2;           // define.h:135
  p->thresh_sp = 3.0;           // define.h:132
}

void epi_config_default(epi_config* c) {
  if (!c) return;
  c->device = 0;
  c->precision = EPI_PREC_MIXED;
  c->max_conn = 64;
  c->max_cand = 96;
  c->skin = 0.1;
  c->variant = 0;
  c->search_switch = 0;
  c->rebuild_gate = 0;
  c->reserved = 0;
}

const char* epi_strerror(int s) {
  switch (s) {
    case EPI_OK: return "ok";
    case EPI_ERR_INVALID_ARG: return "invalid argument";
    case EPI_ERR_NO_DEVICE: return "no usable CUDA device";
    case EPI_ERR_CUDA: return "CUDA runtime error";
    case EPI_ERR_OOM: return "device out of memory";
    case EPI_ERR_BIN_RANGE: return "particle outside the grid (grid_init range assert)";
    case EPI_ERR_BIN_OVERFLOW: return "grid bin holds more than 199 particles";
    case EPI_ERR_LIST_OVERFLOW: return "connection or candidate list capacity exceeded";
    case EPI_ERR_COEF_RANGE: return "pair interaction coefficient above 1000 (too strong interaction)";
    case EPI_ERR_MEMB_COEF_RANGE: return "membrane interaction coefficient above 100";
    case EPI_ERR_NONFINITE: return "non-finite position";
    case EPI_ERR_TIMEOUT: return "bounded device wait timed out";
    case EPI_ERR_STATE: return "call out of order";
    case EPI_ERR_UNSUPPORTED: return "unsupported geometry";
    case EPI_ERR_CHECK: return "index check failed (bounds-checked build)";
    default: return "unknown status";
  }
}

int epi_create(epi_ctx** out, const epi_config* cfg) {
  if (!out) return EPI_ERR_INVALID_ARG;
  *out = nullptr;
  EPI_GUARD_BEGIN
  epi_config c;
  epi_config_default(&c);
  if (cfg) c = *cfg;
  if (c.max_conn <= 0 || c.max_conn > 400 || c.max_cand < c.max_conn || c.max_cand > 1024)
    return EPI_ERR_INVALID_ARG;
  if (!(c.skin > 0) || c.skin > 2.0) return EPI_ERR_INVALID_ARG;
  if (c.variant < 0 || c.variant > 4) return EPI_ERR_INVALID_ARG;
  if (c.precision != EPI_PREC_FP64 && c.precision != EPI_PREC_MIXED) return EPI_ERR_INVALID_ARG;
  if (c.search_switch < 0 || c.rebuild_gate < 0 || c.rebuild_gate > 2) return EPI_ERR_INVALID_ARG;
  if (c.reserved != 0) return EPI_ERR_INVALID_ARG;
  int ndev = 0;
  const cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev <= 0) return EPI_ERR_NO_DEVICE;
  if (c.device < 0 || c.device >= ndev) return EPI_ERR_INVALID_ARG;
  EPI_CUDA(cudaSetDevice(c.device));
  epi_ctx* ctx = new epi_ctx();
  ctx->cfg = c;
  ctx->lc.variant = c.variant == 0 ? 3 : c.variant;
  ctx->lc.search_switch = c.search_switch > 0 ? c.search_switch : kDefaultSearchSwitch;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c.device) == cudaSuccess &&
      sms > 0)
    ctx->lc.num_sms = sms;
  // The step sequence's stream gets the highest priority and the membrane
  // sums' side stream the lowest, so the rebuild chain (the critical path
  // of a step) takes SM slots first and the membrane blocks fill the rest.
  int prio_least = 0, prio_greatest = 0;
  cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  int rc = cuda_status(
      cudaStreamCreateWithPriority(&ctx->stream, cudaStreamNonBlocking, prio_greatest));
  if (rc == EPI_OK) rc = cuda_status(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
  if (rc == EPI_OK)
    rc = cuda_status(cudaStreamCreateWithPriority(&ctx->aux, cudaStreamNonBlocking, prio_least));
  if (rc == EPI_OK)
    rc = cuda_status(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
  if (rc == EPI_OK)
    rc = cuda_status(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
  if (rc == EPI_OK) rc = dev_alloc(&ctx->status, 1);
  if (rc == EPI_OK) rc = cuda_status(cudaMallocHost((void**)&ctx->status_h, sizeof(DevStatus)));
  if (rc == EPI_OK) rc = cuda_status(cudaMemset(ctx->status, 0, sizeof(DevStatus)));
  if (rc == EPI_OK) rc = dev_alloc(&ctx->rebuilds, 1);
  if (rc == EPI_OK) rc = dev_alloc(&ctx->loop_left, 1);
  if (rc == EPI_OK) rc = dev_alloc(&ctx->launches, 1);
  if (rc == EPI_OK) rc = cuda_status(cudaMemset(ctx->launches, 0, sizeof(unsigned long long)));
  if (rc == EPI_OK) rc = cuda_status(cudaMemset(ctx->rebuilds, 0, sizeof(unsigned long long)));
  if (rc != EPI_OK) {
    epi_destroy(ctx);
    return rc;
  }
  *out = ctx;
  return EPI_OK;
  EPI_GUARD_END
}

void epi_destroy(epi_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->cfg.device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  free_buffers(ctx);
  if (ctx->status) cudaFree(ctx->status);
  if (ctx->rebuilds) cudaFree(ctx->rebuilds);
  if (ctx->loop_left) cudaFree(ctx->loop_left);
  if (ctx->launches) cudaFree(ctx->launches);
  if (ctx->status_h) cudaFreeHost(ctx->status_h);
  if (ctx->upin) cudaFreeHost(ctx->upin);
  if (ctx->copy_in) cudaStreamSynchronize(ctx->copy_in);
  if (ctx->copy_out) cudaStreamSynchronize(ctx->copy_out);
  for (cudaEvent_t e : ctx->ev_in) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->ev_done) cudaEventDestroy(e);
  for (cudaEvent_t e : ctx->ev_d2h) cudaEventDestroy(e);
  if (ctx->copy_in) cudaStreamDestroy(ctx->copy_in);
  if (ctx->copy_out) cudaStreamDestroy(ctx->copy_out);
  if (ctx->aux) cudaStreamSynchronize(ctx->aux);
  if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
  if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
  if (ctx->aux) cudaStreamDestroy(ctx->aux);
  if (ctx->side) cudaStreamDestroy(ctx->side);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int epi_upload(epi_ctx* c, int32_t ntissues, const epi_tissue_view* tv, const epi_params* params) {
  if (!c || ntissues <= 0 || !tv) return EPI_ERR_INVALID_ARG;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_upload");
  int rc = set_device(c);
  if (rc) return rc;
  int64_t n = 0;
  int64_t nbins = 0;
  for (int t = 0; t < ntissues; ++t) {
    epi_params P;
    if (params) P = params[t];
    else epi_params_default(&P);
    if ((rc = validate_tissue(tv[t], P))) return rc;
    n += tv[t].n;
    nbins += (int64_t)((int)(tv[t].lx / 2.0 + 0.5)) * (int)(tv[t].ly / 2.0 + 0.5) *
                 (int)(tv[t].lz / 2.0) + 1;
  }
  if (n > (int64_t)0x7fffffff || nbins > (int64_t)0x7ffffff0 || ntissues >= (1 << 24))
    return EPI_ERR_UNSUPPORTED;
  // Candidate rows hold tissue-local indices: 16-bit entries when every
  // tissue has at most 65,536 particles, else 32-bit. Each row has room for
  // the count and max_cand entries, and at least the chunks the step kernel
  // loads up front (2 of 16-bit entries, 4 of 32-bit).
  int32_t nmax = 0;
  for (int t = 0; t < ntissues; ++t) nmax = std::max(nmax, tv[t].n);
  const int32_t cand16 = nmax <= 65536 ? 1 : 0;
  const int32_t per_chunk = cand16 ? 8 : 4;
  const int32_t chunks = std::max((c->cfg.max_cand + 1 + per_chunk - 1) / per_chunk, cand16 ? 2 : 4);
  // A re-upload of the same shape (the per-step connect of an application
  // that renews cell state on the host) keeps the device buffers.
  const bool reuse = c->loaded && c->ntissues == ntissues && c->n == n && c->nbins == nbins &&
                     c->cand16 == cand16 && c->cand_chunks == chunks;
  const int32_t old_nprep = c->nprep;
  destroy_graphs(c);
  // The field grids depend on the tissue count and the grid size only: they
  // survive an upload that keeps the tissue count (divisions, removals).
  epi_ctx kept;
  const bool keep_field = c->field_on && c->ntissues == ntissues;
  if (keep_field && !reuse) {
    kept.fd = c->fd; kept.cmap1 = c->cmap1; kept.cmap2 = c->cmap2;
    kept.ext[0] = c->ext[0]; kept.ext[1] = c->ext[1]; kept.zzmax = c->zzmax; kept.izb = c->izb;
    c->fd = nullptr; c->cmap1 = nullptr; c->cmap2 = nullptr;
    c->ext[0] = c->ext[1] = nullptr; c->zzmax = nullptr; c->izb = nullptr;
  } else if (!keep_field) {
    free_field(c);
  }
  const int32_t fnx = c->fnx, fny = c->fny, fnz = c->fnz, fcur = c->ext_cur;
  const int64_t fnvox = c->nvox;
  const std::vector<FieldDev> ffd = c->fd_h;
  if (!reuse) free_buffers(c);
  c->lists_fresh = false;
  if (keep_field && !reuse) {
    c->fd = kept.fd; c->cmap1 = kept.cmap1; c->cmap2 = kept.cmap2;
    c->ext[0] = kept.ext[0]; c->ext[1] = kept.ext[1]; c->zzmax = kept.zzmax; c->izb = kept.izb;
    kept.fd = nullptr; kept.cmap1 = nullptr; kept.cmap2 = nullptr;
    kept.ext[0] = kept.ext[1] = nullptr; kept.zzmax = nullptr; kept.izb = nullptr;
    c->field_on = true;
    c->fnx = fnx; c->fny = fny; c->fnz = fnz; c->ext_cur = fcur; c->nvox = fnvox;
    c->fd_h = ffd;
  }
  c->loaded = false;
  c->ntissues = ntissues;
  c->n = n;
  c->nbins = (int32_t)nbins;
  c->cand16 = cand16;
  c->cand_chunks = chunks;
  const std::vector<TissueDev> old_tissues = reuse ? c->tissues_h : std::vector<TissueDev>();
  c->tissues_h.assign(ntissues, TissueDev{});
  c->thost.assign(ntissues, TissueHost{});
  // The per-particle arrays are assembled in pinned host memory, so their
  // copies to the device run at full bus speed; every entry is written below.
  const size_t need = (sizeof(double4) + 2 * sizeof(double) + sizeof(uint32_t) +
                       sizeof(int32_t)) * (size_t)std::max<int64_t>(n, 1);
  if (c->upin_bytes < need) {
    if (c->upin) cudaFreeHost(c->upin);
    c->upin = nullptr;
    c->upin_bytes = 0;
    if ((rc = cuda_status(cudaMallocHost((void**)&c->upin, need)))) {
      free_buffers(c);
      return rc;
    }
    c->upin_bytes = need;
  }
  double4* pos = reinterpret_cast<double4*>(c->upin);
  double* spr = reinterpret_cast<double*>(pos + n);
  double* agek = spr + n;
  uint32_t* attr = reinterpret_cast<uint32_t*>(agek + n);
  int32_t* pair = reinterpret_cast<int32_t*>(attr + n);
  std::vector<int32_t> prep_m, prep_f;
  int32_t pbase = 0, binbase = 0;
  bool simple = true, any_old = false;
  for (int t = 0; t < ntissues; ++t) {
    const epi_tissue_view& v = tv[t];
    epi_params P;
    if (params) P = params[t];
    else epi_params_default(&P);
    TissueDev& T = c->tissues_h[t];
    TissueHost& H = c->thost[t];
    T.pbase = pbase;
    T.n = v.n;
    T.nmemb = v.nmemb;
    T.nder = v.nder;
    T.nmx = v.nmx;
    T.nmy = v.nmy;
    T.anx = (int32_t)(v.lx / 2.0 + 0.5);  // ANX / ANY / ANZ, cell_connection.cpp:22-26
    T.any = (int32_t)(v.ly / 2.0 + 0.5);
    T.anz = (int32_t)(v.lz / 2.0);
    T.binbase = binbase;
    T.lattice = v.lattice;
    T.nadj = v.lattice == EPI_LATTICE_TRIANGULAR ? kMembAdjTri : kMembAdj;
    T.mbase = (int32_t)prep_m.size();
    T.lx = v.lx;
    T.ly = v.ly;
    T.lz = v.lz;
    T.hlx = 0.5 * v.lx;
    T.hly = 0.5 * v.ly;
    std::memcpy(&T.P, &P, sizeof(Params));
    T.lawf = make_laws<float>(T.P);
    T.lawd = make_laws<double>(T.P);
    range_thresholds(T);
    H.prep_m = (int32_t)prep_m.size();
    H.prep_f = (int32_t)prep_f.size();
    double rmax = 0, rmax_nm = 0;
    for (int32_t i = 0; i < v.n; ++i) {
      const int64_t g = pbase + i;
      pos[g] = make_double4(v.x[i], v.y[i], v.z[i], v.radius[i]);
      const uint32_t st = v.state[i];
      rmax = std::max(rmax, v.radius[i]);
      if (st != ST_MEMB) rmax_nm = std::max(rmax_nm, v.radius[i]);
      uint32_t a = st | ((uint32_t)t << 8);
      if (v.agek && v.agek[i] > P.thresh_sp) {
        a |= 1u << 4;
        any_old = true;
      }
      if (st != ST_MEMB && st != ST_ALIVE && st != ST_DEAD && st != ST_AIR) simple = false;
      const int32_t q = v.pair ? v.pair[i] : -1;
      if (st == ST_MUSUME) {
        // spring_force_to_memb, cell_interaction.cpp:614-620
        uint32_t code = 0;
        if (q >= 0 && v.state[q] == ST_FIX) code = 1;
        else if (v.rest_div_times && v.rest_div_times[i] > 0) code = 2;
        a |= code << 5;
      }
      attr[g] = a;
      pair[g] = q >= 0 ? pbase + q : -1;
      if (q >= 0) simple = false;
      spr[g] = v.spr_nat_len ? v.spr_nat_len[i] : 0.0;
      agek[g] = v.agek ? v.agek[i] : 0.0;
      if (st == ST_MEMB) prep_m.push_back((int32_t)g);
      if (st == ST_FIX || st == ST_MUSUME) prep_f.push_back((int32_t)g);
    }
    T.rmax = rmax;
    T.rmax_nm = rmax_nm;
    set_fp32_bounds(T);
    H.nfm = (int32_t)prep_f.size() - H.prep_f;
    pbase += v.n;
    binbase += T.anx * T.any * T.anz + 1;  // + sentinel (end offset of the tissue)
  }
  c->lc.simple = simple ? 1 : 0;
  c->lc.any_old = any_old ? 1 : 0;
  c->nprep_memb = (int32_t)prep_m.size();
  c->nprep = c->nprep_memb + (int32_t)prep_f.size();
  std::vector<int32_t> prep(prep_m);
  prep.insert(prep.end(), prep_f.begin(), prep_f.end());
  const size_t C = (size_t)c->cfg.max_conn, CC = (size_t)chunks;
  if (reuse && (int32_t)prep.size() > old_nprep) {
    cudaFree(c->prep);
    c->prep = nullptr;
    if ((rc = dev_alloc(&c->prep, prep.size()))) {
      free_buffers(c);
      return rc;
    }
  }
  if (!reuse && ((rc = dev_alloc(&c->tissues, ntissues)) || (rc = dev_alloc(&c->pos[0], n)) ||
      (rc = dev_alloc(&c->pos[1], n)) || (rc = dev_alloc(&c->posf[0], n)) ||
      (rc = dev_alloc(&c->posf[1], n)) || (rc = dev_alloc(&c->attr, n)) ||
      (rc = dev_alloc(&c->pair, n)) || (rc = dev_alloc(&c->spr, n)) ||
      (rc = dev_alloc(&c->dermis, n)) || (rc = dev_alloc(&c->cand, CC * n)) ||
      (rc = dev_alloc(&c->bpos, n)) ||
      (rc = dev_alloc(&c->nbr, C * n)) || (rc = dev_alloc(&c->nn, n)) ||
      (rc = dev_alloc(&c->fmemb, n)) ||
      (rc = dev_alloc(&c->bin, n)) || (rc = dev_alloc(&c->rank, n)) ||
      (rc = dev_alloc(&c->counts, nbins)) || (rc = dev_alloc(&c->starts, nbins + 1)) ||
      (rc = dev_alloc(&c->skey, n)) || (rc = dev_alloc(&c->spos, n)) ||
      (rc = dev_alloc(&c->gate, (size_t)ntissues + 1)) ||
      (rc = dev_alloc(&c->rl, 3 + 3 * (size_t)ntissues)) ||
      (rc = dev_alloc(&c->prep, prep.size())) || (rc = dev_alloc(&c->stage, 3 * (size_t)n)) ||
      (rc = dev_alloc(&c->agek, n)))) {
    free_buffers(c);
    return rc;
  }
  if (!reuse) {
    c->scan.capacity = (int32_t)((std::max<int64_t>(nbins, n) + kScanTile - 1) / kScanTile) + 1;
    if ((rc = dev_alloc(&c->scan.partial, c->scan.capacity))) {
      free_buffers(c);
      return rc;
    }
  }
  cudaStream_t s = c->stream;
  EPI_CUDA(cudaMemcpyAsync(c->tissues, c->tissues_h.data(), sizeof(TissueDev) * ntissues,
                           cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemcpyAsync(c->pos[0], pos, sizeof(double4) * n, cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemcpyAsync(c->pos[1], c->pos[0], sizeof(double4) * n, cudaMemcpyDeviceToDevice, s));
  c->posf_stale = true;
  EPI_CUDA(cudaMemcpyAsync(c->attr, attr, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemcpyAsync(c->pair, pair, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemcpyAsync(c->spr, spr, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemcpyAsync(c->agek, agek, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  if (c->field_on) {
    // boxes may have changed: refresh the grids' spacing
    for (int32_t t = 0; t < ntissues; ++t)
      field_params(c->fd_h[t], c->tissues_h[t].lx, c->tissues_h[t].ly, c->tissues_h[t].lz,
                   c->fnx, c->fny, c->fnz);
    EPI_CUDA(cudaMemcpyAsync(c->fd, c->fd_h.data(), sizeof(FieldDev) * ntissues,
                             cudaMemcpyHostToDevice, s));
  }
  if (!prep.empty())
    EPI_CUDA(cudaMemcpyAsync(c->prep, prep.data(), sizeof(int32_t) * prep.size(),
                             cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemsetAsync(c->counts, 0, sizeof(int32_t) * (size_t)std::max<int64_t>(nbins, 1), s));
  // Candidate lists stay valid for a same-shape upload wherever the radii,
  // states and box are unchanged and no particle moved skin/2 from the
  // positions of its tissue's last candidate build: gate only the others.
  std::vector<int32_t> gates;
  if (reuse && c->h_radius.size() == (size_t)n && c->h_attr.size() == (size_t)n) {
    gates.assign(1 + (size_t)ntissues, 0);
    for (int32_t t = 0; t < ntissues; ++t) {
      const TissueDev& A = old_tissues[t];
      const TissueDev& B = c->tissues_h[t];
      bool changed = A.n != B.n || A.lx != B.lx || A.ly != B.ly || A.lz != B.lz ||
                     A.lattice != B.lattice || A.nmx != B.nmx || A.nmy != B.nmy ||
                     std::memcmp(&A.P, &B.P, sizeof(Params)) != 0;
      for (int32_t i = B.pbase; !changed && i < B.pbase + B.n; ++i)
        changed = c->h_radius[i] != pos[i].w || c->h_attr[i] != attr[i];
      gates[1 + t] = changed ? 1 : 0;
      gates[0] |= gates[1 + t];
    }
  }
  c->h_radius.resize(n);
  c->h_attr.assign(attr, attr + n);
  for (int64_t i = 0; i < n; ++i) c->h_radius[i] = pos[i].w;
  if (gates.empty()) {
    EPI_CUDA(cudaMemsetAsync(c->nn, 0, sizeof(int32_t) * n, s));
    EPI_CUDA(cudaMemsetAsync(c->cand, 0, sizeof(uint4) * n, s));  // row counts (chunk 0)
    EPI_CUDA(cudaMemsetAsync(c->dermis, 0xff, sizeof(int32_t) * n, s));
  }
  EPI_CUDA(cudaMemsetAsync(c->status, 0, sizeof(DevStatus), s));
  c->cur = 0;
  c->loaded = true;
  if (gates.empty()) {
    launch_set_gates(make_state(c, c->cur), ntissues, s);
  } else {
    EPI_CUDA(cudaMemcpyAsync(c->gate, gates.data(), sizeof(int32_t) * gates.size(),
                             cudaMemcpyHostToDevice, s));
    launch_gate_check(make_state(c, c->cur), c->lc, s);
  }
  // the copies read the pinned staging, which the next upload rewrites:
  // finish before return
  return materialize(c);
  EPI_GUARD_END
}

int epi_adjoint(epi_ctx* c, int32_t nsteps, int32_t K, const epi_loss* loss, double* loss_out,
                double* grad) {
  if (!c || nsteps < 0 || K < 1 || !loss || !loss->target_x || !loss->target_y ||
      !loss->target_z || loss->reserved != 0 || (loss->cells_only != 0 && loss->cells_only != 1))
    return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_adjoint");
  int rc = set_device(c);
  if (rc) return rc;
  const size_t n = (size_t)c->n;
  const int32_t nt = c->ntissues;
  const int32_t nseg = (nsteps + K - 1) / K;
  const size_t hist_len = (size_t)std::max(1, std::min(K, nsteps));
  cudaStream_t s = c->stream;
  ScopedDeviceMemory mem;
  double4 *lam0, *lam1, *bend, *madj, *gmemb, *gpart, *ckpt, *hist, *xT;
  double *acc, *target, *inv_cnt;
  const size_t nm = (size_t)std::max(c->nprep_memb, 1);
  if ((rc = mem.get(&lam0, n)) || (rc = mem.get(&lam1, n)) || (rc = mem.get(&gpart, n)) ||
      (rc = mem.get(&bend, 13 * nm)) || (rc = mem.get(&madj, nm)) || (rc = mem.get(&gmemb, nm)) ||
      (rc = mem.get(&ckpt, n * (size_t)std::max(nseg, 1))) || (rc = mem.get(&hist, n * hist_len)) ||
      (rc = mem.get(&xT, n)) || (rc = mem.get(&acc, 4 * (size_t)nt)) ||
      (rc = mem.get(&target, 3 * n)) || (rc = mem.get(&inv_cnt, (size_t)nt)))
    return rc;
  const size_t pbytes = sizeof(double4) * n;
  EPI_CUDA(cudaMemcpyAsync(target, loss->target_x, 8 * n, cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemcpyAsync(target + n, loss->target_y, 8 * n, cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemcpyAsync(target + 2 * n, loss->target_z, 8 * n, cudaMemcpyHostToDevice, s));
  std::vector<double> inv(nt);
  for (int32_t t = 0; t < nt; ++t) {
    const int32_t cnt = c->tissues_h[t].n - (loss->cells_only ? c->tissues_h[t].nmemb : 0);
    inv[t] = cnt > 0 ? 1.0 / cnt : 0.0;
  }
  EPI_CUDA(cudaMemcpyAsync(inv_cnt, inv.data(), 8 * (size_t)nt, cudaMemcpyHostToDevice, s));
  EPI_CUDA(cudaMemsetAsync(acc, 0, 32 * (size_t)nt, s));
  // forward, keeping a checkpoint every K steps
  for (int32_t t = 0; t < nsteps; ++t) {
    if (t % K == 0)
      EPI_CUDA(cudaMemcpyAsync(ckpt + (size_t)(t / K) * n, c->pos[c->cur], pbytes,
                               cudaMemcpyDeviceToDevice, s));
    enqueue_step(c, c->cur, nullptr);
  }
  c->lists_fresh = false;
  if ((rc = check_status(c))) return rc;
  EPI_CUDA(cudaMemcpyAsync(xT, c->pos[c->cur], pbytes, cudaMemcpyDeviceToDevice, s));
  launch_adjoint_seed(make_state(c, c->cur), target, loss->cells_only, inv_cnt, lam0,
                      gpart, c->lc, s);
  launch_tissue_sum(make_state(c, c->cur), gpart, acc, c->lc, s);
  double4* lam[2] = {lam0, lam1};
  int a = 0;
  for (int32_t seg = nseg - 1; seg >= 0; --seg) {
    const int32_t t0 = seg * K, t1 = std::min(t0 + K, nsteps);
    // recompute X_t0 .. X_{t1-1} from the checkpoint
    EPI_CUDA(cudaMemcpyAsync(c->pos[c->cur], ckpt + (size_t)seg * n, pbytes,
                             cudaMemcpyDeviceToDevice, s));
    c->posf_stale = true;
    launch_gate_check(make_state(c, c->cur), c->lc, s);
    for (int32_t t = t0; t < t1; ++t) {
      EPI_CUDA(cudaMemcpyAsync(hist + (size_t)(t - t0) * n, c->pos[c->cur], pbytes,
                               cudaMemcpyDeviceToDevice, s));
      if (t + 1 < t1) enqueue_step(c, c->cur, nullptr);
    }
    // and differentiate them in reverse
    for (int32_t t = t1 - 1; t >= t0; --t) {
      DevState St = make_state(c, c->cur);
      St.pos_cur = hist + (size_t)(t - t0) * n;
      launch_gate_check(St, c->lc, s);
      launch_rebuild(St, whole(c), c->scan, c->lc, s, nullptr);
      // the dermis of FIX / MUSUME cells at X_t selects their membrane law
      launch_dermis(St, c->nprep_memb, c->nprep, c->lc, s, nullptr);
      const AdjointBuffers B{lam[a], lam[a ^ 1], bend, madj, gmemb, gpart};
      launch_adjoint_step(St, B, c->lc, s);
      launch_tissue_sum(St, gpart, acc, c->lc, s);
      a ^= 1;
    }
    if ((rc = check_status(c))) return rc;
  }
  // the context ends at X_T; its candidates are rebuilt before the next step
  EPI_CUDA(cudaMemcpyAsync(c->pos[c->cur], xT, pbytes, cudaMemcpyDeviceToDevice, s));
  c->posf_stale = true;
  launch_set_gates(make_state(c, c->cur), nt, s);
  std::vector<double> h(4 * (size_t)nt);
  EPI_CUDA(cudaMemcpyAsync(h.data(), acc, 32 * (size_t)nt, cudaMemcpyDeviceToHost, s));
  if ((rc = check_status(c))) return rc;
  for (int32_t t = 0; t < nt; ++t) {
    if (loss_out) loss_out[t] = h[4 * t + 3];
    if (grad)
      for (int k = 0; k < 3; ++k) grad[3 * t + k] = h[4 * t + k];
  }
  return EPI_OK;
  EPI_GUARD_END
}

int epi_field_init(epi_ctx* c, int32_t nx, int32_t ny, int32_t nz) {
  if (!c || nx < 3 || ny < 3 || nz < 3) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_field_init");
  int rc = set_device(c);
  if (rc) return rc;
  free_field(c);
  const int32_t nt = c->ntissues;
  if (nt > 65535) return EPI_ERR_UNSUPPORTED;  // one grid row of blocks per tissue
  const int64_t per = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  c->fd_h.assign(nt, FieldDev{});
  for (int32_t t = 0; t < nt; ++t) {
    FieldDev& F = c->fd_h[t];
    F.base = per * t;
    field_params(F, c->tissues_h[t].lx, c->tissues_h[t].ly, c->tissues_h[t].lz, nx, ny, nz);
    // a stamp window must not wrap onto itself (it spans 2 x 2 ir + 1 points)
    if (2 * F.irx >= nx || 2 * F.iry >= ny || 2 * F.irz >= nz) {
      c->fd_h.clear();
      return EPI_ERR_UNSUPPORTED;
    }
  }
  c->nvox = per * nt;
  if ((rc = dev_alloc(&c->fd, nt)) || (rc = dev_alloc(&c->cmap1, c->nvox)) ||
      (rc = dev_alloc(&c->cmap2, c->nvox)) || (rc = dev_alloc(&c->ext[0], c->nvox)) ||
      (rc = dev_alloc(&c->ext[1], c->nvox)) || (rc = dev_alloc(&c->zzmax, nt)) ||
      (rc = dev_alloc(&c->izb, nt))) {
    free_field(c);
    return rc;
  }
  c->field_on = true;
  c->fnx = nx; c->fny = ny; c->fnz = nz;
  c->ext_cur = 0;
  cudaStream_t s = c->stream;
  EPI_CUDA(cudaMemcpyAsync(c->fd, c->fd_h.data(), sizeof(FieldDev) * nt, cudaMemcpyHostToDevice, s));
  // ext_stim_init = 0 (define.h:180); Field zero-initialises (Field.h:16)
  EPI_CUDA(cudaMemsetAsync(c->ext[0], 0, sizeof(double) * c->nvox, s));
  EPI_CUDA(cudaMemsetAsync(c->ext[1], 0, sizeof(double) * c->nvox, s));
  EPI_CUDA(cudaMemsetAsync(c->cmap1, 0, sizeof(int32_t) * c->nvox, s));
  EPI_CUDA(cudaMemsetAsync(c->cmap2, 0, c->nvox, s));
  EPI_CUDA(cudaMemsetAsync(c->zzmax, 0, sizeof(double) * nt, s));
  EPI_CUDA(cudaMemsetAsync(c->izb, 0, sizeof(int32_t) * nt, s));
  return check_status(c);
  EPI_GUARD_END
}

int epi_field_step(epi_ctx* c, int32_t nsteps) {
  if (!c || nsteps < 0) return EPI_ERR_INVALID_ARG;
  if (!c->loaded || !c->field_on) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_field_step");
  int rc = set_device(c);
  if (rc) return rc;
  for (int32_t k = 0; k < nsteps; ++k) {
    FieldState FS;
    FS.fd = c->fd;
    FS.cmap1 = c->cmap1;
    FS.cmap2 = c->cmap2;
    FS.cur = c->ext[c->ext_cur];
    FS.nxt = c->ext[c->ext_cur ^ 1];
    FS.zzmax = c->zzmax;
    FS.izb = c->izb;
    FS.nvox = c->nvox;
    FS.agek = c->agek;
    int32_t wmax = 1;
    for (const FieldDev& F : c->fd_h) wmax = std::max(wmax, 4 * std::max(F.irx, F.iry) + 1);
    launch_field_step(make_state(c, c->cur), FS, wmax, c->lc, c->stream);
    c->ext_cur ^= 1;  // ext_stim.swap()
  }
  return check_status(c);
  EPI_GUARD_END
}

int epi_field_get(epi_ctx* c, int32_t tissue, int32_t* cmap1, uint8_t* cmap2, double* ext,
                  double* zzmax) {
  if (!c || tissue < 0) return EPI_ERR_INVALID_ARG;
  if (!c->loaded || !c->field_on) return EPI_ERR_STATE;
  if (tissue >= c->ntissues) return EPI_ERR_INVALID_ARG;
  EPI_GUARD_BEGIN
  int rc = set_device(c);
  if (rc) return rc;
  const FieldDev& F = c->fd_h[tissue];
  const size_t per = (size_t)(F.nx + 1) * (F.ny + 1) * (F.nz + 1);
  cudaStream_t s = c->stream;
  if (cmap1)
    EPI_CUDA(cudaMemcpyAsync(cmap1, c->cmap1 + F.base, sizeof(int32_t) * per,
                             cudaMemcpyDeviceToHost, s));
  if (cmap2) EPI_CUDA(cudaMemcpyAsync(cmap2, c->cmap2 + F.base, per, cudaMemcpyDeviceToHost, s));
  if (ext)
    EPI_CUDA(cudaMemcpyAsync(ext, c->ext[c->ext_cur] + F.base, sizeof(double) * per,
                             cudaMemcpyDeviceToHost, s));
  if (zzmax)
    EPI_CUDA(cudaMemcpyAsync(zzmax, c->zzmax + tissue, sizeof(double), cudaMemcpyDeviceToHost, s));
  if ((rc = check_status(c))) return rc;
  // stored as index + 1 (0: none)
  if (cmap1)
    for (size_t v = 0; v < per; ++v) cmap1[v] -= 1;
  return EPI_OK;
  EPI_GUARD_END
}

int epi_field_set_ext(epi_ctx* c, int32_t tissue, const double* ext) {
  if (!c || tissue < 0 || !ext) return EPI_ERR_INVALID_ARG;
  if (!c->loaded || !c->field_on) return EPI_ERR_STATE;
  if (tissue >= c->ntissues) return EPI_ERR_INVALID_ARG;
  EPI_GUARD_BEGIN
  int rc = set_device(c);
  if (rc) return rc;
  const FieldDev& F = c->fd_h[tissue];
  const size_t per = (size_t)(F.nx + 1) * (F.ny + 1) * (F.nz + 1);
  for (int b = 0; b < 2; ++b)  // both buffers, as read_binary into first() and second()
    EPI_CUDA(cudaMemcpyAsync(c->ext[b] + F.base, ext, sizeof(double) * per,
                             cudaMemcpyHostToDevice, c->stream));
  return check_status(c);
  EPI_GUARD_END
}

int epi_connect(epi_ctx* c) {
  if (!c) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_connect");
  int rc = set_device(c);
  if (rc) return rc;
  return materialize(c);
  EPI_GUARD_END
}

int epi_interact_commit(epi_ctx* c) {
  if (!c) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_interact_commit");
  int rc = set_device(c);
  if (rc) return rc;
  enqueue_step(c, c->cur, nullptr);
  c->lists_fresh = false;
  return check_status(c);
  EPI_GUARD_END
}

int epi_step(epi_ctx* c, int32_t nsteps) {
  if (!c || nsteps < 0) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_step");
  int rc = set_device(c);
  if (rc) return rc;
  for (int32_t k = 0; k < nsteps; ++k) enqueue_step(c, c->cur, nullptr);
  if (nsteps > 0) c->lists_fresh = false;
  return check_status(c);
  EPI_GUARD_END
}

int epi_step_graph(epi_ctx* c, int32_t nsteps) {
  if (!c || nsteps < 0) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_step_graph");
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = enqueue_graph_steps(c, nsteps))) return rc;
  return check_status(c);
  EPI_GUARD_END
}

int epi_autotune(epi_ctx* c, int32_t trial_steps, double* skin_out, int32_t* variant_out,
                 double* ms_out) {
  if (!c || trial_steps < 2) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_autotune");
  int rc = set_device(c);
  if (rc) return rc;
  static const double kSkins[] = {0.05, 0.08, 0.1, 0.15, 0.2, 0.3};
  static const int32_t kVariants[] = {1, 2, 3, 4};
  constexpr int32_t kWarm = 4;  // the first step after a restore rebuilds every tissue
  const size_t pbytes = sizeof(double4) * (size_t)c->n;
  cudaStream_t s = c->stream;
  ScopedDeviceMemory mem;
  double4* saved = nullptr;
  if ((rc = mem.get(&saved, (size_t)c->n))) return rc;
  const int cur0 = c->cur;
  EPI_CUDA(cudaMemcpyAsync(saved, c->pos[cur0], pbytes, cudaMemcpyDeviceToDevice, s));
  cudaEvent_t ev[2];
  EPI_CUDA(cudaEventCreate(&ev[0]));
  EPI_CUDA(cudaEventCreate(&ev[1]));
  struct Events {
    cudaEvent_t* e;
    ~Events() {
      cudaEventDestroy(e[0]);
      cudaEventDestroy(e[1]);
    }
  } ev_guard{ev};
  // every trial starts from the saved positions with fresh candidates
  auto restore = [&]() -> int {
    EPI_CUDA(cudaMemcpyAsync(c->pos[cur0], saved, pbytes, cudaMemcpyDeviceToDevice, s));
    c->cur = cur0;
    c->posf_stale = true;
    launch_set_gates(make_state(c, c->cur), c->ntissues, s);
    c->lists_fresh = false;
    return EPI_OK;
  };
  auto apply = [&](double skin, int32_t variant, int32_t search_switch, int32_t gate) {
    apply_tuning(c, skin, variant, search_switch, gate);
  };
  // one trial: ms per trial (INFINITY when the rows overflowed)
  auto trial = [&](double* ms_out) -> int {
    int r;
    if ((r = restore())) return r;
    if ((r = enqueue_graph_steps(c, kWarm))) return r;
    EPI_CUDA(cudaEventRecord(ev[0], s));
    if ((r = enqueue_graph_steps(c, trial_steps))) return r;
    EPI_CUDA(cudaEventRecord(ev[1], s));
    *ms_out = INFINITY;
    // a skin whose candidate rows overflow max_cand fails here: skip it
    if (check_status(c) != EPI_OK) return EPI_OK;
    float ms = 0;
    EPI_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    *ms_out = ms;
    return EPI_OK;
  };
  double best = INFINITY, best_skin = c->cfg.skin;
  int32_t best_variant = c->cfg.variant;
  const int32_t switch0 = c->cfg.search_switch, form0 = c->cfg.rebuild_gate;
  for (double skin : kSkins) {
    for (int32_t variant : kVariants) {
      apply(skin, variant, switch0, form0);
      double ms;
      if ((rc = trial(&ms))) return rc;
      if (ms < best) {
        best = ms;
        best_skin = skin;
        best_variant = variant;
      }
    }
  }
  // then the rebuild in a conditional graph node or not, and the candidate
  // search's switch from a warp to a thread per particle
  int32_t best_form = form0, best_switch = switch0;
  if (std::isfinite(best)) {
    for (int32_t form : {1, 2}) {
      apply(best_skin, best_variant, switch0, form);
      double ms;
      if ((rc = trial(&ms))) return rc;
      if (ms < best) {
        best = ms;
        best_form = form;
      }
    }
    static const int32_t kSwitches[] = {8192, 16384, 49152, 131072};
    for (int32_t sw : kSwitches) {
      apply(best_skin, best_variant, sw, best_form);
      double ms;
      if ((rc = trial(&ms))) return rc;
      if (ms < best) {
        best = ms;
        best_switch = sw;
      }
    }
  }
  apply(best_skin, best_variant, best_switch, best_form);
  if ((rc = restore())) return rc;
  if ((rc = check_status(c))) return rc;
  if (skin_out) *skin_out = best_skin;
  if (variant_out) *variant_out = best_variant;
  if (ms_out) *ms_out = std::isfinite(best) ? best / trial_steps : -1.0;
  return std::isfinite(best) ? EPI_OK : EPI_ERR_LIST_OVERFLOW;
  EPI_GUARD_END
}

int epi_get_config(epi_ctx* c, epi_config* out) {
  if (!c || !out) return EPI_ERR_INVALID_ARG;
  *out = c->cfg;
  return EPI_OK;
}

int epi_set_tuning(epi_ctx* c, double skin, int32_t variant, int32_t search_switch,
                   int32_t rebuild_gate) {
  if (!c || !(skin > 0) || skin > 2.0 || variant < 0 || variant > 4 || search_switch < 0 ||
      rebuild_gate < 0 || rebuild_gate > 2)
    return EPI_ERR_INVALID_ARG;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_set_tuning");
  int rc = set_device(c);
  if (rc) return rc;
  apply_tuning(c, skin, variant, search_switch, rebuild_gate);
  if (c->loaded) {
    // candidates were built for the old skin: rebuild every tissue's
    launch_set_gates(make_state(c, c->cur), c->ntissues, c->stream);
    c->lists_fresh = false;
    return check_status(c);
  }
  return EPI_OK;
  EPI_GUARD_END
}

int epi_step_per_tissue(epi_ctx* c, int32_t nsteps) {
  if (!c || nsteps < 0) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_step_per_tissue");
  int rc = set_device(c);
  if (rc) return rc;
  ensure_posf(c);
  for (int32_t k = 0; k < nsteps; ++k) {
    for (int t = 0; t < c->ntissues; ++t) {
      const Range r = tissue_range(c, t);
      const DevState S = make_state(c, c->cur);
      launch_rebuild(S, r, c->scan, c->lc, c->stream, nullptr);
      prepass_tissue(c, c->cur, t);
      launch_step(S, r, c->cfg.precision, c->lc, c->stream, nullptr);
    }
    c->cur ^= 1;
  }
  if (nsteps > 0) c->lists_fresh = false;
  return check_status(c);
  EPI_GUARD_END
}

int epi_sync(epi_ctx* c) {
  if (!c) return EPI_ERR_INVALID_ARG;
  EPI_GUARD_BEGIN
  int rc = set_device(c);
  if (rc) return rc;
  // outbound copies of host steps run on their own stream
  if (c->copy_out) EPI_CUDA(cudaStreamSynchronize(c->copy_out));
  return check_status(c);
  EPI_GUARD_END
}

int epi_num_particles(const epi_ctx* c, int64_t* n) {
  if (!c || !n) return EPI_ERR_INVALID_ARG;
  *n = c->loaded ? c->n : 0;
  return EPI_OK;
}

int epi_download_positions(epi_ctx* c, double* x, double* y, double* z) {
  if (!c || !x || !y || !z) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_download_positions");
  int rc = set_device(c);
  if (rc) return rc;
  const int64_t n = c->n;
  double* d = c->stage;
  launch_unpack_positions(make_state(c, c->cur), d, d + n, d + 2 * n, (int32_t)n, c->stream);
  EPI_CUDA(cudaMemcpyAsync(x, d, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  EPI_CUDA(cudaMemcpyAsync(y, d + n, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  EPI_CUDA(cudaMemcpyAsync(z, d + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream));
  return check_status(c);
  EPI_GUARD_END
}

int epi_upload_positions(epi_ctx* c, const double* x, const double* y, const double* z) {
  if (!c || !x || !y || !z) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_upload_positions");
  int rc = set_device(c);
  if (rc) return rc;
  const int64_t n = c->n;
  double* d = c->stage;
  EPI_CUDA(cudaMemcpyAsync(d, x, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  EPI_CUDA(cudaMemcpyAsync(d + n, y, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  EPI_CUDA(cudaMemcpyAsync(d + 2 * n, z, sizeof(double) * n, cudaMemcpyHostToDevice, c->stream));
  const DevState S = make_state(c, c->cur);
  launch_pack_positions(S, d, d + n, d + 2 * n, (int32_t)n, c->stream);
  // a tissue re-derives its candidates once one of its particles is skin/2
  // from its last candidate build (the test the step itself applies)
  launch_gate_check(S, c->lc, c->stream);
  c->lists_fresh = false;
  launch_rebuild(S, whole(c), c->scan, c->lc, c->stream, nullptr);
  return check_status(c);
  EPI_GUARD_END
}

// One step of a batch whose positions live in host memory: what
// epi_upload_positions + epi_interact_commit + epi_download_positions do,
// split into groups of whole tissues of about equal particle count. A
// group's inbound copies, its kernels and its outbound copies run on three
// streams, so one group's copies overlap the next group's copies in the
// other direction and the compute between them. Tissues never interact, so
// the result equals the three calls'. Successive calls pipeline: a group's
// inbound copy and its unpack into the outbound staging wait only for the
// previous call's outbound copy of the same group (the host arrays may be
// the same for input and output, and the staging regions are reused).
static int enqueue_host_step(epi_ctx* c, bool chained, const double* x_in, const double* y_in,
                             const double* z_in, double* x_out, double* y_out, double* z_out) {
  const int64_t n = c->n;
  int rc;
  if (!c->copy_in)
    EPI_CUDA(cudaStreamCreateWithFlags(&c->copy_in, cudaStreamNonBlocking));
  if (!c->copy_out)
    EPI_CUDA(cudaStreamCreateWithFlags(&c->copy_out, cudaStreamNonBlocking));
  if (!c->stage_out && (rc = dev_alloc(&c->stage_out, 3 * (size_t)n))) return rc;
  // groups: whole tissues, split at multiples of n / K particles
  const int K = std::min(kHostStepGroups, c->ntissues);
  while ((int)c->ev_in.size() < K) {
    cudaEvent_t a, b, d;
    EPI_CUDA(cudaEventCreateWithFlags(&a, cudaEventDisableTiming));
    EPI_CUDA(cudaEventCreateWithFlags(&b, cudaEventDisableTiming));
    EPI_CUDA(cudaEventCreateWithFlags(&d, cudaEventDisableTiming));
    c->ev_in.push_back(a);
    c->ev_done.push_back(b);
    c->ev_d2h.push_back(d);
  }
  std::vector<int> split{0};
  for (int t = 0, k = 1; t < c->ntissues && k < K; ++t) {
    const TissueDev& T = c->tissues_h[t];
    if ((int64_t)(T.pbase + T.n) * K >= (int64_t)k * n && t + 1 < c->ntissues) {
      split.push_back(t + 1);
      ++k;
    }
  }
  split.push_back(c->ntissues);
  double* in = c->stage;
  double* out = c->stage_out;
  // other earlier work on the compute stream (an upload through the same
  // inbound staging, a step) precedes this step's inbound copies; after a
  // host step the per-group waits below are enough
  if (!chained) {
    EPI_CUDA(cudaEventRecord(c->ev_done[0], c->stream));
    EPI_CUDA(cudaStreamWaitEvent(c->copy_in, c->ev_done[0], 0));
  }
  const int cur = c->cur;
  const DevState S = make_state(c, cur);
  const DevState Snew = make_state(c, cur ^ 1);
  for (size_t g = 0; g + 1 < split.size(); ++g) {
    const int t0 = split[g], t1 = split[g + 1];
    const TissueDev& A = c->tissues_h[t0];
    const TissueDev& B = c->tissues_h[t1 - 1];
    const int32_t p0 = A.pbase, p1 = B.pbase + B.n;
    const size_t off = (size_t)p0, bytes = sizeof(double) * (size_t)(p1 - p0);
    const double* src[3] = {x_in, y_in, z_in};
    // the previous call's outbound copy of this group may still write the
    // host arrays this copy reads
    EPI_CUDA(cudaStreamWaitEvent(c->copy_in, c->ev_d2h[g], 0));
    {
      Nvtx r("host step: positions in");
      for (int k = 0; k < 3; ++k)
        EPI_CUDA(cudaMemcpyAsync(in + k * n + off, src[k] + off, bytes, cudaMemcpyHostToDevice,
                                 c->copy_in));
    }
    EPI_CUDA(cudaEventRecord(c->ev_in[g], c->copy_in));
    EPI_CUDA(cudaStreamWaitEvent(c->stream, c->ev_in[g], 0));
    launch_pack_gate(S, in, in + n, in + 2 * n, p0, p1, c->lc, c->stream);
    const Range r{p0, p1, A.binbase, B.binbase + B.anx * B.any * B.anz + 1, t0, t1};
    launch_rebuild(S, r, c->scan, c->lc, c->stream, nullptr);
    const TissueHost& HA = c->thost[t0];
    const TissueHost& HB = c->thost[t1 - 1];
    launch_prepass(S, HA.prep_m, HB.prep_m + B.nmemb, c->nprep_memb + HA.prep_f,
                   c->nprep_memb + HB.prep_f + HB.nfm, c->cfg.precision, c->lc, c->stream,
                   nullptr);
    launch_step(S, r, c->cfg.precision, c->lc, c->stream, nullptr);
    // ... and may still read this group's outbound staging
    EPI_CUDA(cudaStreamWaitEvent(c->stream, c->ev_d2h[g], 0));
    launch_unpack_range(Snew, out, out + n, out + 2 * n, p0, p1, c->lc, c->stream);
    EPI_CUDA(cudaEventRecord(c->ev_done[g], c->stream));
    EPI_CUDA(cudaStreamWaitEvent(c->copy_out, c->ev_done[g], 0));
    double* dst[3] = {x_out, y_out, z_out};
    {
      Nvtx r("host step: positions out");
      for (int k = 0; k < 3; ++k)
        EPI_CUDA(cudaMemcpyAsync(dst[k] + off, out + k * n + off, bytes, cudaMemcpyDeviceToHost,
                                 c->copy_out));
    }
    EPI_CUDA(cudaEventRecord(c->ev_d2h[g], c->copy_out));
  }
  c->cur ^= 1;
  c->posf_stale = false;
  c->lists_fresh = false;
  c->after_host_step = true;
  return EPI_OK;
}

int epi_step_host(epi_ctx* c, const double* x_in, const double* y_in, const double* z_in,
                  double* x_out, double* y_out, double* z_out) {
  if (!c || !x_in || !y_in || !z_in || !x_out || !y_out || !z_out) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_step_host");
  const bool chained = c->after_host_step;
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = enqueue_host_step(c, chained, x_in, y_in, z_in, x_out, y_out, z_out))) return rc;
  EPI_CUDA(cudaStreamSynchronize(c->copy_out));
  return check_status(c);
  EPI_GUARD_END
}

int epi_step_host_async(epi_ctx* c, const double* x_in, const double* y_in, const double* z_in,
                        double* x_out, double* y_out, double* z_out) {
  if (!c || !x_in || !y_in || !z_in || !x_out || !y_out || !z_out) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_step_host_async");
  const bool chained = c->after_host_step;
  int rc = set_device(c);
  if (rc) return rc;
  return enqueue_host_step(c, chained, x_in, y_in, z_in, x_out, y_out, z_out);
  EPI_GUARD_END
}

int epi_get_connections(epi_ctx* c, int32_t* offsets, int32_t* idx, int64_t cap,
                        int64_t* total) {
  if (!c || !offsets || cap < 0 || (cap > 0 && !idx)) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_get_connections");
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = materialize(c))) return rc;
  const int32_t n = (int32_t)c->n;
  ScanScratch sc;
  sc.capacity = (n + kScanTile - 1) / kScanTile + 1;
  if (c->x_n != c->n || !c->x_rowlen) {
    free_export(c);
    if ((rc = dev_alloc(&c->x_rowlen, n)) || (rc = dev_alloc(&c->x_rowoff, (size_t)n + 1)) ||
        (rc = dev_alloc(&c->x_partial, sc.capacity))) {
      free_export(c);
      return rc;
    }
    c->x_n = c->n;
  }
  sc.partial = c->x_partial;
  const DevState S = make_state(c, c->cur);
  launch_rowlen(S, c->x_rowlen, n, c->stream);
  launch_scan(c->x_rowlen, c->x_rowoff, n, 0, sc, nullptr, c->lc, c->stream);
  EPI_CUDA(cudaMemcpyAsync(offsets, c->x_rowoff, sizeof(int32_t) * ((size_t)n + 1),
                           cudaMemcpyDeviceToHost, c->stream));
  EPI_CUDA(cudaStreamSynchronize(c->stream));
  const int64_t tot = offsets[n];
  if (total) *total = tot;
  if (cap >= tot && tot > 0) {
    if (c->x_idx_cap < tot) {
      if (c->x_idx) cudaFree(c->x_idx);
      c->x_idx = nullptr;
      c->x_idx_cap = 0;
      // room for the lists to grow by a quarter before the next reallocation
      const int64_t want = tot + tot / 4;
      if ((rc = dev_alloc(&c->x_idx, (size_t)want))) return rc;
      c->x_idx_cap = want;
    }
    launch_fill_csr(S, c->x_rowoff, c->x_idx, n, c->stream);
    EPI_CUDA(cudaMemcpyAsync(idx, c->x_idx, sizeof(int32_t) * tot, cudaMemcpyDeviceToHost,
                             c->stream));
  }
  if (cap < tot && cap > 0) {
    EPI_CUDA(cudaStreamSynchronize(c->stream));
    return EPI_ERR_INVALID_ARG;
  }
  return check_status(c);
  EPI_GUARD_END
}

int epi_get_dermis(epi_ctx* c, int32_t* dermis) {
  if (!c || !dermis) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_get_dermis");
  int rc = set_device(c);
  if (rc) return rc;
  if ((rc = materialize(c))) return rc;
  if (c->x_n != c->n || !c->x_rowlen) {
    free_export(c);
    const int32_t n = (int32_t)c->n;
    if ((rc = dev_alloc(&c->x_rowlen, n)) || (rc = dev_alloc(&c->x_rowoff, (size_t)n + 1)) ||
        (rc = dev_alloc(&c->x_partial, (n + kScanTile - 1) / kScanTile + 1))) {
      free_export(c);
      return rc;
    }
    c->x_n = c->n;
  }
  // the row-length buffer holds the local dermis indices (n entries)
  launch_dermis_local(make_state(c, c->cur), c->x_rowlen, (int32_t)c->n, c->stream);
  EPI_CUDA(cudaMemcpyAsync(dermis, c->x_rowlen, sizeof(int32_t) * c->n, cudaMemcpyDeviceToHost,
                           c->stream));
  return check_status(c);
  EPI_GUARD_END
}

int epi_error_info(epi_ctx* c, int32_t* tissue, int32_t* particle, int32_t* other,
                   double* value) {
  if (!c) return EPI_ERR_INVALID_ARG;
  int32_t t = -1, a = c->last.a, b = c->last.b;
  if (c->last.code != 0 && a >= 0) {
    for (int k = 0; k < c->ntissues; ++k) {
      const TissueDev& T = c->tissues_h[k];
      if (a >= T.pbase && a < T.pbase + T.n) {
        t = k;
        a -= T.pbase;
        if (b >= T.pbase && b < T.pbase + T.n) b -= T.pbase;
        else if (c->last.code != EPI_ERR_BIN_OVERFLOW) b = -1;
        break;
      }
    }
  }
  if (tissue) *tissue = t;
  if (particle) *particle = a;
  if (other) *other = b;
  if (value) *value = c->last.v;
  return c->last.code;
}

void* epi_stream(epi_ctx* c) { return c ? (void*)c->stream : nullptr; }

int epi_rebuild_count(epi_ctx* c, int64_t* count) {
  if (!c || !count) return EPI_ERR_INVALID_ARG;
  EPI_GUARD_BEGIN
  int rc = set_device(c);
  if (rc) return rc;
  unsigned long long v = 0;
  EPI_CUDA(cudaMemcpyAsync(&v, c->rebuilds, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
  EPI_CUDA(cudaStreamSynchronize(c->stream));
  *count = (int64_t)v;
  return EPI_OK;
  EPI_GUARD_END
}

int epi_launch_count(epi_ctx* c, int64_t* count) {
  if (!c || !count) return EPI_ERR_INVALID_ARG;
  EPI_GUARD_BEGIN
  int rc = set_device(c);
  if (rc) return rc;
  unsigned long long v = 0;
  EPI_CUDA(cudaMemcpyAsync(&v, c->launches, sizeof(v), cudaMemcpyDeviceToHost, c->stream));
  EPI_CUDA(cudaStreamSynchronize(c->stream));
  *count = (int64_t)v;
  return EPI_OK;
  EPI_GUARD_END
}

int epi_time_kernels(epi_ctx* c, int32_t nsteps, int32_t max_classes, double* ms,
                     int32_t* launches, const char** names, int32_t* nclasses) {
  if (!c || nsteps < 0 || !ms || !launches || max_classes < KC_COUNT) return EPI_ERR_INVALID_ARG;
  if (!c->loaded) return EPI_ERR_STATE;
  EPI_GUARD_BEGIN
  Nvtx nvtx_range("epi_time_kernels");
  int rc = set_device(c);
  if (rc) return rc;
  Timer tm;
  for (int32_t k = 0; k < nsteps; ++k) enqueue_step(c, c->cur, &tm);
  if (nsteps > 0) c->lists_fresh = false;
  rc = check_status(c);
  for (int k = 0; k < KC_COUNT; ++k) {
    double sum = 0;
    for (auto& p : tm.ev[k]) {
      float f = 0;
      cudaEventElapsedTime(&f, p.a, p.b);
      sum += f;
    }
    ms[k] = sum;
    launches[k] = (int32_t)tm.ev[k].size();
    if (names) names[k] = kKernelClassNames[k];
  }
  if (nclasses) *nclasses = KC_COUNT;
  return rc;
  EPI_GUARD_END
}

}  // extern "C"
