// connect_cell for one tissue without any device allocation.
//
// Some callers cannot let this library call cudaMalloc: applications whose
// device memory all belongs to another allocator (a framework's caching
// allocator, or a pool sized once at start-up against a fixed memory budget)
// and loops that must not allocate once they run. For them,
// epi_connect_noalloc reads caller-owned device inputs, writes caller-owned
// device outputs, and keeps its working storage in one file-scope device
// array of fixed size. That array exists on every GPU that loads the
// library, from load until process exit.
//
// The scratch holds the bin counts, bin offsets and the sorted particle
// indices of the counting sort. It is shared by every call on a device and
// keeps the last call's contents; each call clears the counts it uses before
// binning. Two calls whose work overlaps on the GPU (different streams, or
// different host threads) race on it.
#include "epi_mech.h"
#include "epi_common.cuh"

#include <cuda_runtime.h>
#include <algorithm>
#include <mutex>

namespace {

using namespace epi;

constexpr int32_t kMaxP = EPI_NOALLOC_MAX_PARTICLES;
constexpr int32_t kMaxB = EPI_NOALLOC_MAX_BINS;
// scratch layout, in int32 words, each part 64-word aligned
constexpr int32_t kOffCounts = 0;
constexpr int32_t kOffStarts = kOffCounts + kMaxB;
constexpr int32_t kOffBin = kOffStarts + ((kMaxB + 1 + 63) / 64) * 64;
constexpr int32_t kOffRank = kOffBin + kMaxP;
constexpr int32_t kOffSorted = kOffRank + kMaxP;
constexpr int32_t kScratchWords = kOffSorted + kMaxP;

static __device__ __align__(256) int32_t g_noalloc_scratch[kScratchWords];

struct Args {
  const double* x;
  const double* y;
  const double* z;
  const double* r;
  int32_t n, nmemb, nmx, nmy;
  double lx, ly, lz, lt;
  int32_t anx, any, anz;
  int32_t max_conn;
  int32_t* conn;
  int32_t* count;
  int32_t* scratch;  // device address of g_noalloc_scratch
};

constexpr int kThreads = 256;

// Row heads: membrane rows start with their four lattice links in the order
// _memb_init pushes them (cellmanager.cpp:160-163); other rows are empty.
// Also clears the bin counts this call uses.
__global__ void na_init(Args A) {
  const int32_t nb = A.anx * A.any * A.anz;
  for (int32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x)
    A.scratch[kOffCounts + b] = 0;
  for (int32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < A.n; i += gridDim.x * blockDim.x) {
    if (i < A.nmemb) {
      const Lattice L = lattice_of(i, A.nmx, A.nmy);
      int32_t* row = A.conn + (int64_t)i * A.max_conn;
      const int32_t links[4] = {L.l, L.r, L.b, L.u};
      for (int k = 0; k < kMembAdj && k < A.max_conn; ++k) row[k] = links[k];
      A.count[i] = kMembAdj;
    } else {
      A.count[i] = 0;
    }
  }
}

// grid_init's bin (cell_connection.cpp:44-53); -1 marks the range assert.
__global__ void na_bin(Args A) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const double x = A.x[i], y = A.y[i], z = A.z[i];
  // Coordinates are converted to bin numbers only once they are finite and
  // within a few boxes of the grid, so every conversion is in int32 range.
  const double big = 4.0 * (A.lx + A.ly + A.lz);
  bool bad = !isfinite(x) || !isfinite(y) || !isfinite(z) || fabs(x) > big || fabs(y) > big ||
             fabs(z) > big;
  int32_t aix = 0, aiy = 0, aiz = 0;
  if (!bad) {
    aix = (int32_t)((0.5 * A.lx - pdiff(0.5 * A.lx, x, A.lx)) / kAreaGrid);
    aiy = (int32_t)((0.5 * A.ly - pdiff(0.5 * A.ly, y, A.ly)) / kAreaGrid);
    aiz = (int32_t)(fmax(z, 0.0) / kAreaGrid);
    bad = aix >= A.anx || aiy >= A.any || aiz >= A.anz || aix < 0 || aiy < 0 || aiz < 0;
  }
  if (!bad && i >= A.nmemb) {  // connect_proc's assert for the searching cells (:95-99)
    const int32_t cx = (int32_t)(x / kAreaGrid), cy = (int32_t)(y / kAreaGrid),
                  cz = (int32_t)(z / kAreaGrid);
    bad = cx >= A.anx || cy >= A.any || cz >= A.anz || cx < 0 || cy < 0 || cz < 0;
  }
  if (bad) {
    A.scratch[kOffBin + i] = -1;
    A.count[i] = -1;  // the range assert of grid_init / connect_proc
    return;
  }
  const int32_t b = (aix * A.any + aiy) * A.anz + aiz;
  A.scratch[kOffBin + i] = b;
  A.scratch[kOffRank + i] = atomicAdd(&A.scratch[kOffCounts + b], 1);
}

// One block: exclusive scan of the bin counts into the bin offsets.
__global__ void na_scan(Args A) {
  __shared__ int32_t wsum[kThreads / 32];
  const int32_t nb = A.anx * A.any * A.anz;
  const int32_t* in = A.scratch + kOffCounts;
  int32_t* out = A.scratch + kOffStarts;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int32_t carry = 0;
  for (int32_t base = 0; base < nb; base += kThreads) {
    const int32_t b = base + threadIdx.x;
    const int32_t v = b < nb ? in[b] : 0;
    int32_t incl = v;
    for (int o = 1; o < 32; o <<= 1) {
      const int32_t t = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += t;
    }
    if (lane == 31) wsum[wid] = incl;
    __syncthreads();
    int32_t before = 0, tot = 0;
    for (int w = 0; w < kThreads / 32; ++w) {
      if (w < wid) before += wsum[w];
      tot += wsum[w];
    }
    if (b < nb) out[b] = carry + before + incl - v;
    carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) out[nb] = carry;
}

__global__ void na_scatter(Args A) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int32_t b = A.scratch[kOffBin + i];
  if (b < 0) return;
  A.scratch[kOffSorted + A.scratch[kOffStarts + b] + A.scratch[kOffRank + i]] = i;
}

__device__ __forceinline__ void push(const Args& A, int32_t row, int32_t v) {
  const int32_t k = atomicAdd(&A.count[row], 1);
  if (k < A.max_conn) A.conn[(int64_t)row * A.max_conn + k] = v;
}

// connect_proc (cell_connection.cpp:70-129): every non-membrane cell scans
// the 5x5x5 bins around (int)(x/AREA_GRID) with wrap in x, y and z and
// connects to each lower-index particle within LJ_THRESH*(r_c+r_o),
// pushing each into the other's row.
__global__ void na_connect(Args A) {
  const int32_t c = A.nmemb + blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= A.n) return;
  if (A.scratch[kOffBin + c] < 0) return;
  const double x = A.x[c], y = A.y[c], z = A.z[c], r = A.r[c];
  const int32_t anx = (int32_t)(x / kAreaGrid), any = (int32_t)(y / kAreaGrid),
                anz = (int32_t)(z / kAreaGrid);
  for (int32_t j = anx - 2 + A.anx; j <= anx + 2 + A.anx; ++j) {
    const int32_t aix = j % A.anx;
    for (int32_t k = any - 2 + A.any; k <= any + 2 + A.any; ++k) {
      const int32_t aiy = k % A.any;
      for (int32_t l = anz - 2 + A.anz; l <= anz + 2 + A.anz; ++l) {
        const int32_t b = (aix * A.any + aiy) * A.anz + l % A.anz;
        const int32_t s1 = A.scratch[kOffStarts + b + 1];
        for (int32_t s = A.scratch[kOffStarts + b]; s < s1; ++s) {
          const int32_t o = A.scratch[kOffSorted + s];
          if (c <= o) continue;
          const double d2 = dist_sq_exact(pdiff(x, A.x[o], A.lx), pdiff(y, A.y[o], A.ly), z - A.z[o]);
          if (connected_pred(d2, A.lt, r, A.r[o])) {
            push(A, c, o);
            push(A, o, c);
          }
        }
      }
    }
  }
}

// Each row sorted ascending (the rows' push order depends on thread timing).
__global__ void na_sort_rows(Args A) {
  const int32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.n) return;
  const int32_t c = A.count[i];
  const int32_t m = c < 0 ? 0 : (c < A.max_conn ? c : A.max_conn);
  int32_t* row = A.conn + (int64_t)i * A.max_conn;
  for (int32_t s = 1; s < m; ++s) {
    const int32_t v = row[s];
    int32_t k = s - 1;
    while (k >= 0 && row[k] > v) {
      row[k + 1] = row[k];
      --k;
    }
    row[k + 1] = v;
  }
}

// Launches kernel k with `grid` blocks of kThreads threads on stream s and
// returns that launch's own status.
cudaError_t launch(void (*k)(Args), int grid, cudaStream_t s, const Args& A) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)kThreads);
  cfg.stream = s;
  return cudaLaunchKernelEx(&cfg, k, A);
}

// Device address of the scratch array, looked up once per device.
constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
int32_t* g_scratch_addr[kMaxDevices] = {};

int scratch_of_current_device(int32_t** out) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return EPI_ERR_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return EPI_ERR_UNSUPPORTED;
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) return EPI_ERR_CUDA;
    g_scratch_addr[dev] = static_cast<int32_t*>(p);
  }
  *out = g_scratch_addr[dev];
  return EPI_OK;
}

}  // namespace

extern "C" int epi_connect_noalloc(const double* x, const double* y, const double* z,
                                   const double* radius, int32_t n, int32_t nmemb, int32_t nmx,
                                   int32_t nmy, double lx, double ly, double lz,
                                   double lj_thresh, int32_t max_conn, int32_t* conn,
                                   int32_t* count, void* stream) {
  try {
    if (n < 0 || nmemb < 0 || nmemb > n || max_conn < kMembAdj) return EPI_ERR_INVALID_ARG;
    if (n > 0 && (!x || !y || !z || !radius || !conn || !count))
      return EPI_ERR_INVALID_ARG;
    if (!(lx > 0) || !(ly > 0) || !(lz > 0) || !(lj_thresh > 0)) return EPI_ERR_INVALID_ARG;
    if (nmemb != nmx * nmy || (nmemb > 0 && (nmx < 3 || nmy < 3))) return EPI_ERR_UNSUPPORTED;
    Args A;
    A.anx = (int32_t)(lx / 2.0 + 0.5);  // ANX / ANY / ANZ, cell_connection.cpp:22-26
    A.any = (int32_t)(ly / 2.0 + 0.5);
    A.anz = (int32_t)(lz / 2.0);
    // a window of 5 bins that wrapped onto itself would push pairs twice
    if (A.anx < 5 || A.any < 5 || A.anz < 5) return EPI_ERR_UNSUPPORTED;
    // the fixed scratch bounds every call
    if (n > kMaxP || (int64_t)A.anx * A.any * A.anz > kMaxB) return EPI_ERR_INVALID_ARG;
    if (n == 0) return EPI_OK;
    int rc = scratch_of_current_device(&A.scratch);
    if (rc != EPI_OK) return rc;
    A.x = x;
    A.y = y;
    A.z = z;
    A.r = radius;
    A.n = n;
    A.nmemb = nmemb;
    A.nmx = nmx;
    A.nmy = nmy;
    A.lx = lx;
    A.ly = ly;
    A.lz = lz;
    A.lt = lj_thresh;
    A.max_conn = max_conn;
    A.conn = conn;
    A.count = count;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int nb = A.anx * A.any * A.anz;
    const int g = (std::max(n, nb) + kThreads - 1) / kThreads;
    const int gp = (n + kThreads - 1) / kThreads;
    // Each launch reports its own status, so an error that earlier, unrelated
    // work left pending on this thread is neither reported here nor cleared.
    cudaError_t e = launch(na_init, g, s, A);
    if (e == cudaSuccess) e = launch(na_bin, gp, s, A);
    if (e == cudaSuccess) e = launch(na_scan, 1, s, A);
    if (e == cudaSuccess) e = launch(na_scatter, gp, s, A);
    if (e == cudaSuccess && n > nmemb)
      e = launch(na_connect, (n - nmemb + kThreads - 1) / kThreads, s, A);
    if (e == cudaSuccess) e = launch(na_sort_rows, gp, s, A);
    return e == cudaSuccess ? EPI_OK : EPI_ERR_CUDA;
  } catch (...) {
    return EPI_ERR_CUDA;
  }
}
