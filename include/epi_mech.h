/* epi_mech.h -- C ABI of the B200 cell-mechanics library (libepi_mech.so).
 *
 * The library replaces the per-step mechanics of the epi5_MT epidermis model:
 *   connect_cell(CellManager&)          epi5_MT/cell_connection.h:3,
 *                                       epi5_MT/cell_connection.cpp:191-203
 *   cell_interaction(CellManager&)      epi5_MT/cell_interaction.h:5,
 *                                       epi5_MT/cell_interaction.cpp:648-685
 *   pos_copy(CellManager&)              epi5_MT/cellmanager.h:117,
 *                                       epi5_MT/cellmanager.cpp:19-26
 *   cell_pos_periodic_fix(CellManager&) epi5_MT/cellmanager.h:111,
 *                                       epi5_MT/cellmanager.cpp:395-414
 * for the square- and the triangular-membrane (TRI_MEMB) builds, on one
 * GPU, for one tissue or a batch of independent tissues, and the cell maps
 * and external-stimulus diffusion that follow them in the reference's loop
 * (setup_map_lat, calc_ext_stim); it adds gradients (epi_adjoint) and an
 * autotuner. A tissue is what one epi5_MT CellManager holds:
 * particles in the reference's index layout (membrane [0,nmemb), dermis
 * [nmemb,nmemb+nder), every other cell after), a periodic box LX x LY and an
 * open height LZ.
 *
 * Conventions: every call returns an epi_status (0 = EPI_OK); no exception
 * crosses the ABI. Pointers are host pointers unless stated otherwise. A
 * context is bound to one device and one stream and must not be used from two
 * threads at once. Work is stream-ordered; calls that return data to the host
 * synchronise the context's stream. Errors raised inside kernels are sticky
 * until the call that reports them returns.
 */
#ifndef EPI_MECH_H
#define EPI_MECH_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. Kernel-side conditions mirror the reference's aborts. */
typedef enum epi_status {
  EPI_OK = 0,
  EPI_ERR_INVALID_ARG = 1,      /* bad pointer, size or tissue description */
  EPI_ERR_NO_DEVICE = 2,        /* no usable CUDA device */
  EPI_ERR_CUDA = 3,             /* a CUDA runtime call failed */
  EPI_ERR_OOM = 4,              /* device allocation failed */
  EPI_ERR_BIN_RANGE = 5,        /* particle outside the grid: cell_connection.cpp:48-53, :99 */
  EPI_ERR_BIN_OVERFLOW = 6,     /* more than 199 particles in one 2.0 grid bin: cell_connection.cpp:59 */
  EPI_ERR_LIST_OVERFLOW = 7,    /* connection list capacity exceeded: cell_connection.cpp:122 */
  EPI_ERR_COEF_RANGE = 8,       /* |pair coefficient| > 1000: cell_interaction.cpp:51-55 */
  EPI_ERR_MEMB_COEF_RANGE = 9,  /* |membrane coefficient| > 100: cell_interaction.cpp:200-231 */
  EPI_ERR_NONFINITE = 10,       /* a position became NaN or infinite */
  EPI_ERR_TIMEOUT = 11,         /* a bounded device-side wait gave up */
  EPI_ERR_STATE = 12,           /* call out of order (e.g. step before upload) */
  EPI_ERR_UNSUPPORTED = 13,     /* geometry outside what the library implements */
  EPI_ERR_CHECK = 14            /* an index check of the bounds-checked build failed
                                   (libepi_mech_check.so, built with -DEPI_CHECK) */
} epi_status;

/* Force-law constants of one tissue. Defaults (epi_params_default) are the
 * reference's compile-time constants: epi5_MT/cell_interaction.cpp:21-45
 * (eps_m, P_MEMB, DER_DER_CONST, K_TOTAL, K_DESMOSOME, Kspring, Kspring_d,
 * KBEND, delta_R, para_ljp2, Kspring_division) and epi5_MT/define.h:86,132,135
 * (DT_Cell, THRESH_SP, LJ_THRESH). */
typedef struct epi_params {
  double dt;
  double eps_m;
  double p_memb;
  double der_der_const;
  double k_total;
  double k_desmosome;
  double kspring;
  double kspring_d;
  double kbend;
  double delta_r;
  double para_ljp2;
  double kspring_division;
  double lj_thresh;
  double thresh_sp;
} epi_params;

/* Membrane lattices of epi5_MT (define.h:66, TRI_MEMB). */
typedef enum epi_lattice {
  EPI_LATTICE_SQUARE = 0,     /* TRI_MEMB undefined: 4 links, cellmanager.cpp:114-166 */
  EPI_LATTICE_TRIANGULAR = 1  /* TRI_MEMB (the reference's default): 6 links,
                                 cellmanager.cpp:70-111; nmy = rows, even */
} epi_lattice;

/* One tissue in structure-of-arrays form: what epi5_MT's Cell objects hold for
 * the mechanics (epi5_MT/cell.h:101-247). Indices (pair) are tissue-local,
 * -1 for none; pairs must be mutual. nmemb must equal nmx * nmy; the
 * membrane particles come first, row by row, wired as `lattice` says. */
typedef struct epi_tissue_view {
  int32_t n, nmemb, nder;
  int32_t nmx, nmy;
  double lx, ly, lz;
  const double* x;
  const double* y;
  const double* z;
  const double* radius;
  const double* agek;
  const double* spr_nat_len;
  const uint8_t* state;          /* CELL_STATE, epi5_MT/define.h:36-47 */
  const int32_t* pair;
  const int32_t* rest_div_times;
  int32_t lattice;               /* epi_lattice (0 = square) */
  int32_t reserved;              /* must be 0 */
} epi_tissue_view;

typedef enum epi_precision {
  EPI_PREC_FP64 = 0,  /* every force in FP64 */
  EPI_PREC_MIXED = 1  /* pair and bending forces in FP32, sums and positions in FP64 */
} epi_precision;

/* Connection lists are exact every step, as connect_cell's are. Internally a
 * tissue keeps a candidate list of every partner within
 * LJ_THRESH*(r_i+r_j) + skin, rebuilt once any of its particles has moved
 * skin/2 since the last rebuild; the reference's predicate is evaluated on
 * the candidates at every step. skin trades rebuild frequency for candidate
 * count and never changes results. */
typedef struct epi_config {
  int32_t device;     /* CUDA device ordinal */
  int32_t precision;  /* epi_precision */
  int32_t max_conn;   /* connections per particle (membrane lattice links are
                         extra); the reference allows 400 (define.h:80) */
  int32_t max_cand;   /* candidates per particle (>= max_conn) */
  double skin;        /* candidate margin, > 0 (default 0.1) */
  int32_t variant;    /* step-kernel form: 0 = default (3); 1, 2 = the
                         neighbours' positions copied asynchronously into
                         shared memory, 8 / 15 per thread at once (FP64: 4 /
                         8); 3, 4 = gathered into registers four at a time
                         (FP64: two), 3 / 4 resident 256-thread blocks per SM
                         (FP64: 3 / 2). Same formulas; the compiler may fuse
                         multiply-adds differently, so results agree to
                         rounding. */
  int32_t search_switch; /* candidate search: rebuilds of at least this many
                         particles take one thread per particle, smaller ones
                         one warp per particle; 0 = default (49152) */
  int32_t rebuild_gate; /* step graph: 0 = default (1 for a single tissue,
                         2 for a batch); 1 = the candidate rebuild's kernels
                         sit in a conditional node that skips them on steps
                         with nothing to rebuild; 2 = they are always launched
                         (and exit at once when nothing is listed) */
  int32_t reserved;   /* must be 0 */
} epi_config;

typedef struct epi_ctx epi_ctx;

void epi_params_default(epi_params* p);
void epi_config_default(epi_config* c);
const char* epi_strerror(int status);

/* Context lifetime. */
int epi_create(epi_ctx** out, const epi_config* cfg);
void epi_destroy(epi_ctx* ctx);

/* Loads ntissues tissues (one CellManager each) and their constants, then runs
 * the first connect, as cman_init does (epi5_MT/cell_init.cpp:132-137).
 * Replaces any previous contents. params may be NULL (defaults). */
int epi_upload(epi_ctx* ctx, int32_t ntissues, const epi_tissue_view* tissues,
               const epi_params* params);

/* connect_cell over every tissue: bins, connection lists, dermis. */
int epi_connect(epi_ctx* ctx);
/* cell_interaction + pos_copy + cell_pos_periodic_fix over every tissue,
 * using the lists of the last connect. */
int epi_interact_commit(epi_ctx* ctx);
/* nsteps of the reference's cell_dynamics mechanics (epi5_MT/proc.cpp:22-32
 * without cell_state_renew): interact+commit, then connect. */
int epi_step(epi_ctx* ctx, int32_t nsteps);
/* Same as epi_step, replayed from a CUDA graph captured on first use. */
int epi_step_graph(epi_ctx* ctx, int32_t nsteps);
/* Same as epi_step, but one kernel sequence per tissue and no graph: the
 * unbatched launch pattern, kept as the comparison point for batching. */
int epi_step_per_tissue(epi_ctx* ctx, int32_t nsteps);
/* Waits for queued work and reports any kernel-side error. */
int epi_sync(epi_ctx* ctx);

/* Total particles over all tissues (positions are concatenated by tissue). */
int epi_num_particles(const epi_ctx* ctx, int64_t* n);
int epi_download_positions(epi_ctx* ctx, double* x, double* y, double* z);
/* Overwrites positions (both buffers, like dual_double::_set) and re-connects. */
int epi_upload_positions(epi_ctx* ctx, const double* x, const double* y, const double* z);
/* One mechanics step of a batch whose positions live in host memory: the
 * loop body the drop-in runs per step (connect_cell, then cell_interaction,
 * pos_copy and cell_pos_periodic_fix; epi5_MT/proc.cpp:22-32), equal to
 * epi_upload_positions(in) + epi_interact_commit + epi_download_positions(out).
 * The batch is split into groups of whole tissues whose host copies in both
 * directions overlap the other groups' kernels. Blocks until the new
 * positions are in the out arrays; in and out may be the same arrays. Host
 * memory should be pinned (page-locked) for the copies to overlap. */
int epi_step_host(epi_ctx* ctx, const double* x_in, const double* y_in, const double* z_in,
                  double* x_out, double* y_out, double* z_out);
/* epi_step_host without waiting: returns once the step is queued. Successive
 * calls pipeline (a call's first copies overlap the previous call's last
 * ones); the out arrays hold the new positions, and the in arrays may be
 * reused, only after epi_sync (which also reports errors of queued steps). */
int epi_step_host_async(epi_ctx* ctx, const double* x_in, const double* y_in,
                        const double* z_in, double* x_out, double* y_out, double* z_out);
/* Connection lists as CSR over all particles (offsets has n+1 entries). Each
 * row holds tissue-local indices sorted ascending; membrane rows include their
 * four lattice links, as connected_cell does (epi5_MT/cell.h:132). Writes at
 * most cap indices and always the exact total to *total. */
int epi_get_connections(epi_ctx* ctx, int32_t* offsets, int32_t* idx, int64_t cap,
                        int64_t* total);
/* Nearest connected membrane particle of each FIX / MUSUME cell
 * (find_dermis, epi5_MT/cell_connection.cpp:158-172), tissue-local, -1 where
 * none or not applicable. */
int epi_get_dermis(epi_ctx* ctx, int32_t* dermis);
/* Details of the last kernel-side error: particle and partner (tissue-local
 * where known, else -1) and the offending value. */
int epi_error_info(epi_ctx* ctx, int32_t* tissue, int32_t* particle, int32_t* other,
                   double* value);

/* The cudaStream_t the context launches on (as void*). */
void* epi_stream(epi_ctx* ctx);
/* Tissue candidate-list rebuilds since the context was created (the count
 * the skin trades against candidate-list length). */
int epi_rebuild_count(epi_ctx* ctx, int64_t* count);
/* Kernels of the step sequence (rebuild, membrane prepass, dermis, step, and
 * the graph's condition and loop kernels) executed on the device since the
 * context was created, counted by the kernels themselves; kernels a graph's
 * conditional node skipped are not counted. */
int epi_launch_count(epi_ctx* ctx, int64_t* count);
/* Per-kernel timing: runs nsteps (not graph-captured) recording CUDA events
 * around each kernel class on the context stream. ms receives the summed
 * milliseconds per class, launches the launch count per class, names the
 * class names; returns the number of classes (<= max_classes). */
int epi_time_kernels(epi_ctx* ctx, int32_t nsteps, int32_t max_classes, double* ms,
                     int32_t* launches, const char** names, int32_t* nclasses);

/* Autotuner. Times short graph-replayed trials of the uploaded batch for
 * every candidate skin in {0.05, 0.08, 0.1, 0.15, 0.2, 0.3} and step-kernel
 * variant 1..4 (4 warm-up steps, then trial_steps timed with CUDA events),
 * then, for the fastest pair, the rebuild in a conditional graph node or
 * not, and the candidate search's switch from a warp to a thread per
 * particle in {8192, 16384, 49152, 131072} rebuilt particles, and keeps the
 * fastest choice in the context's configuration. Skins whose candidate rows would overflow
 * max_cand are skipped. The simulation state is left as it was (positions
 * are restored after every trial), and no choice changes results beyond
 * multiply-add rounding (connection sets are exact for every skin, and both
 * search forms emit candidates in the same order). Writes the skin, variant
 * and the best trial's time per step (any output may be NULL);
 * epi_get_config returns the whole choice. No counterpart in the
 * reference. */
int epi_autotune(epi_ctx* ctx, int32_t trial_steps, double* skin, int32_t* variant,
                 double* ms_per_step);

/* The context's configuration (after epi_autotune: its choice). */
int epi_get_config(epi_ctx* ctx, epi_config* out);

/* Applies a tuning chosen earlier (for instance a cached epi_autotune
 * result for the same batch shape): skin, variant, search switch and
 * rebuild node, with epi_config's ranges. Every tissue's candidates are rebuilt before the
 * next step. No counterpart in the reference. */
int epi_set_tuning(epi_ctx* ctx, double skin, int32_t variant, int32_t search_switch,
                   int32_t rebuild_gate);

/* ---- cell maps and external-stimulus diffusion -----------------------------
 * The rest of the reference's per-step loop before its chemistry
 * (epi5_MT/proc.cpp:152-157): calc_zzmax, setup_map_lat (map.cpp:24-167) and
 * calc_ext_stim (ext_stim.cpp:18-69), per tissue on an (nx+1) x (ny+1) x
 * (nz+1) grid over its box (define.h NX, NY, NZ; z fastest, the layout of
 * FArr3D). Results equal the reference's bit for bit on the same positions.
 *
 * epi_field_init allocates the grids of every tissue of the batch and zeroes
 * the stimulus (ext_stim_init, define.h:180); the grids survive uploads that
 * keep the tissue count. */
int epi_field_init(epi_ctx* ctx, int32_t nx, int32_t ny, int32_t nz);
/* nsteps of: zzmax, cell maps, one stimulus update, from the current positions. */
int epi_field_step(epi_ctx* ctx, int32_t nsteps);
/* Tissue `tissue`'s grids: cmap1 (tissue-local cell index, -1 none; the
 * reference's cell pointers), cmap2 (the ALIVE / FIX / MUSUME mask), ext
 * (the current stimulus) and the last zzmax; each output may be NULL. */
int epi_field_get(epi_ctx* ctx, int32_t tissue, int32_t* cmap1, uint8_t* cmap2, double* ext,
                  double* zzmax);
/* Sets tissue `tissue`'s stimulus (both buffers, as the reference's
 * read_binary of saved field data does, proc.cpp:106-109). */
int epi_field_set_ext(epi_ctx* ctx, int32_t tissue, const double* ext);

/* ---- gradients: reverse-mode adjoint of the step --------------------------
 * No counterpart in the reference, which has no gradients. The loss of
 * tissue t is L_t = mean over its loss set of |x_i(T) - x*_i|^2, x_i(T) the
 * positions after nsteps steps from the current state (minimum image in x
 * and y); the loss set is every particle (cells_only = 0) or every
 * non-membrane particle (cells_only = 1). Targets are n_total doubles each,
 * concatenated by tissue like the positions. */
typedef struct epi_loss {
  const double* target_x;
  const double* target_y;
  const double* target_z;
  int32_t cells_only;
  int32_t reserved;  /* must be 0 */
} epi_loss;
/* Runs nsteps steps (the context ends at the positions epi_step(ctx, nsteps)
 * reaches) and returns, per tissue t, loss[t] and the gradient of L_t with
 * respect to three multipliers of the tissue's force constants, at 1:
 *   grad[3t + 0]  every spring constant (der_der_const, k_total,
 *                 k_desmosome, kspring, kspring_d, kspring_division),
 *   grad[3t + 1]  eps_m (Lennard-Jones depth),
 *   grad[3t + 2]  kbend (membrane bending).
 * d L_t / d eps_m is grad[3t + 1] / eps_m, and so on. Reverse mode: the
 * positions are checkpointed every `checkpoint_every` steps and each segment
 * is recomputed before it is differentiated, so the device holds
 * ceil(nsteps / checkpoint_every) + checkpoint_every position sets.
 * Derivatives are evaluated in FP64 along the trajectory of the context's
 * precision. Square and triangular membranes and every cell state of the
 * path (DER, FIX, MUSUME with their dermis springs, ALIVE / DEAD / AIR, pair
 * springs). loss or grad may be NULL. */
int epi_adjoint(epi_ctx* ctx, int32_t nsteps, int32_t checkpoint_every, const epi_loss* loss,
                double* loss_out, double* grad);

/* ---- connect_cell of one tissue without any device allocation ------------
 * No counterpart in the reference: it exists for callers that cannot let this
 * library call cudaMalloc — applications whose device memory all belongs to
 * another allocator (a framework's caching allocator, or a pool sized once at
 * start-up against a fixed memory budget) and loops that must not allocate
 * once they run. The caller owns every buffer; the working storage is one
 * fixed file-scope device array (about 0.75 MB) that exists on every GPU
 * that loads the library until the process exits.
 *
 * Inputs x, y, z, radius (n doubles each) and outputs conn (n * max_conn
 * int32, row i at conn + i * max_conn) and count (n int32) are device memory.
 * Particles [0, nmemb) are the square membrane (nmemb = nmx * nmy). On return
 * the work is queued on `stream` (a cudaStream_t; NULL = the default stream)
 * and nothing is synchronised. When the stream reaches it: count[i] is the
 * length of connected_cell for particle i (membrane rows include their four
 * lattice links) and, when count[i] <= max_conn, row i holds its partner
 * indices sorted ascending. count[i] > max_conn means the row overflowed:
 * the row then holds an unspecified subset of max_conn partners (which ones
 * depends on thread timing); treat it as an error, as the context API's
 * EPI_ERR_LIST_OVERFLOW. count[i] = -1 means particle i is outside the grid
 * (the reference's range assert); no searched connection lists it (membrane
 * rows still list their lattice links). The connection set is connect_proc's (cell_connection.cpp:70-129).
 *
 * Limits: n <= EPI_NOALLOC_MAX_PARTICLES and ANX*ANY*ANZ <=
 * EPI_NOALLOC_MAX_BINS (ANX = (int)(lx/2 + 0.5), ANY likewise, ANZ =
 * (int)(lz/2)); larger calls return EPI_ERR_INVALID_ARG and queue nothing.
 * It calls no allocating routine. The first call on each device looks up the
 * device address of the working array (cudaGetSymbolAddress); make that first
 * call before any stream capture. Every call on a device shares the array and
 * it keeps the last call's contents (each call clears what it needs); calls
 * whose work overlaps on the GPU — on different streams or from different
 * host threads — race on it. */
#define EPI_NOALLOC_MAX_PARTICLES 40960
#define EPI_NOALLOC_MAX_BINS 32768
int epi_connect_noalloc(const double* x, const double* y, const double* z,
                        const double* radius, int32_t n, int32_t nmemb, int32_t nmx,
                        int32_t nmy, double lx, double ly, double lz, double lj_thresh,
                        int32_t max_conn, int32_t* conn, int32_t* count, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* EPI_MECH_H */
