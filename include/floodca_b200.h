/*
 * floodca_b200 -- B200-native (sm_100a) weighted cellular-automata flood step.
 *
 * Two C-ABI surfaces:
 *
 * 1. The drop-in: the entry points of FloodCA's CUDA backend
 *    (src/cuda/cuda_backend.h:14-32) with the same names, argument meaning,
 *    return codes and struct layouts (src/common/fca_types.h:34-159), so the
 *    reference's unmodified src/cuda/main_cuda.c and
 *    src/hybrid/main_ens_mpi_cuda.c link against this library in place of
 *    src/cuda/kernels.cu. Build the caller and this library with the same
 *    FCA_DOUBLE setting (libfloodca_b200.so: float `real`;
 *    libfloodca_b200_f64.so: double `real`). The struct block below uses the
 *    reference's include guard, so including both headers is harmless.
 *
 * 2. The extended API (fcab_*): device-resident sessions for callers that keep
 *    the state on the GPU (benchmarks, ensembles, the surrogate pipeline).
 *    Plain pointers and sizes; no `real`, so it is the same in both builds and
 *    lives in libfloodca_b200_core.so.
 */
#ifndef FLOODCA_B200_H
#define FLOODCA_B200_H

#include <stddef.h>
#include <stdint.h>

/* ------------------------------------------------------------------------ */
/* Reference ABI types (layout-identical to FloodCA src/common/fca_types.h).  */
/* ------------------------------------------------------------------------ */
#ifndef FCA_TYPES_H
#define FCA_TYPES_H

#ifdef FCA_DOUBLE
typedef double real;
#else
typedef float real;
#endif

enum { FCA_LAND = 0, FCA_SEA = 1, FCA_WALL = 2 };
enum { FCA_BND_OPEN = 0, FCA_BND_CLOSED = 1 };
enum { FCA_HYETO_TRIANGLE = 0, FCA_HYETO_UNIFORM = 1 };

#define FCA_MAX_FORCE_DAYS 64
#define FCA_DAY_S 86400.0

/* Physical parameters (fca_types.h:34-49). */
typedef struct FcaPhys {
    real dx, A, g, alpha, tau_h, tau_l, z_sea, dt_max, dt_min, S_bnd, h_flood;
    int U, K, boundary;
} FcaPhys;

/* Run configuration (fca_types.h:51-86). */
typedef struct FcaRunCfg {
    FcaPhys phys;
    real T_sim, out_every;
    int diag_every, progress_every, hyeto;
    real D_h, phi, lambda;
    int steps, no_output, neigh;
    char config_path[512], grid_dir[512], scenario[128], scenario_file[512];
    char warmstart[512], rain_file[512], out_dir[512], csv_path[512], exp_id[32];
    int repeat, threads, ranks, gpus, block_x, block_y;
    char halo_mode[16], reduce_impl[16], gpu_model[64], backend[32], forcing_csv[512];
    int n_force_days;
    char force_files[FCA_MAX_FORCE_DAYS][768];
} FcaRunCfg;

struct FcaGrid;

/* Distributed-memory hooks (fca_types.h:91-98); ignored by this library. */
typedef struct FcaComm {
    void *ctx;
    int rank;
    void (*halo)(struct FcaGrid *g, real *arr, void *ctx);
    real (*min_real)(real v, void *ctx);
    double (*sum_double)(double v, void *ctx);
    int (*load_rday)(struct FcaGrid *g, const char *path, void *ctx);
} FcaComm;

/* Row-major host grid (fca_types.h:100-126). */
typedef struct FcaGrid {
    int nrows, ncols;
    int r0, r1, c0, c1;
    int edge_n, edge_s, edge_w, edge_e;
    FcaComm *comm;
    real dx, x0, y0;
    real *z, *h, *n, *C;
    uint8_t *mask;
    real *Rday, *hmax, *tmax, *s, *out, *Qx, *Qy, *Qd1, *Qd2, *Qopen;
} FcaGrid;

/* Run accumulators (fca_types.h:128-142). */
typedef struct FcaAcc {
    double V, V0, V_rain, V_sea, V_bnd, clamp_err;
    long cap_active, cap_total, dt_min_hits;
    double t;
    int step;
    real dt_base;
    int force_day;
} FcaAcc;

/* Phase timers (fca_types.h:144-159). */
typedef struct FcaTimers {
    double wall_total, t_init, t_flux, t_limiter, t_update, t_dt, t_io;
    double t_h2d, t_d2h, t_halo, t_allreduce, bytes_per_step;
    long active_cells;
} FcaTimers;

#endif /* FCA_TYPES_H */

#if defined(__GNUC__)
#define FCAB_API __attribute__((visibility("default")))
#else
#define FCAB_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Drop-in entry points (FloodCA src/cuda/cuda_backend.h:14-32).             */
/* ------------------------------------------------------------------------ */

/* Replaces fca_cuda_run (src/cuda/kernels.cu:617-776). Runs the whole
 * simulation on the current device and returns with g->h, g->hmax, g->tmax
 * downloaded and acc/tm filled as the reference does. Differences: every edge
 * flag g->edge_{n,s,w,e} is honoured (the reference CUDA path treats all four
 * edges as open); a CUDA failure returns -2 instead of exit(1); a fixed-step
 * run (cfg->steps > 0) whose step would have dt <= 0 stops instead of
 * looping forever; run parameters the step cannot use (see fcab_sim_create)
 * and a non-finite z, h, n, C or Rday on a LAND cell are refused with -2.
 * A forcing-day file that is missing or short ends the run where that day
 * begins, with acc->t = T_sim and h, hmax, tmax downloaded as the reference
 * leaves them, but returns -3 (the reference returns 0, and its CLI then
 * writes a truncated run as if complete). Returns 0, -1 on a bad block shape
 * (same check as the reference), -2 on a refused input or a device error,
 * -3 on a forcing file that failed to load. The run's device buffers stay
 * cached for later runs (fcab_release_cached_memory frees them). */
FCAB_API int fca_cuda_run(FcaGrid *g, FcaRunCfg *cfg, FcaAcc *acc, FcaTimers *tm);

/* Replaces fca_cuda_device_name (src/cuda/kernels.cu:606-615). */
FCAB_API void fca_cuda_device_name(char *name, size_t n);

/* Replaces fca_cuda_select_device (src/cuda/kernels.cu:778-788): binds device
 * local_rank % count and returns its index, or -1. */
FCAB_API int fca_cuda_select_device(int local_rank);

/* Ensemble session (src/cuda/kernels.cu:790-1043). Static fields stay on the
 * device; each run uploads h, hmax, tmax and Rday, runs like fca_cuda_run and
 * adds hmax >= thr[j] on LAND into uint16 counts kept on the device. */
typedef struct FcaCudaEns FcaCudaEns;
FCAB_API FcaCudaEns *fca_cuda_ens_open(const FcaGrid *g, FcaRunCfg *cfg, int nthr, const double *thr);
FCAB_API int fca_cuda_ens_run(FcaCudaEns *e, FcaGrid *g, const FcaRunCfg *cfg, FcaAcc *acc,
                     FcaTimers *tm, long *flooded, double *max_depth, void (*poll)(void *),
                     void *pctx, int poll_every);
FCAB_API int fca_cuda_ens_counts(FcaCudaEns *e, uint16_t *host);
FCAB_API void fca_cuda_ens_close(FcaCudaEns *e);

/* ------------------------------------------------------------------------ */
/* Extended API (libfloodca_b200_core.so). No reference counterpart.          */
/* ------------------------------------------------------------------------ */

enum {
    FCAB_PREC_F32 = 0,     /* FP32 stencil, FP64 volume and time (reference float build) */
    FCAB_PREC_F32_ALL = 1, /* FP32 stencil, FP32 accumulators and simulated time */
    FCAB_PREC_F64 = 2      /* FP64 everywhere (reference FCA_DOUBLE build) */
};

enum {
    FCAB_MATH_EXACT = 0,   /* every float op rounded as in the reference parity build */
    FCAB_MATH_FAST = 1     /* hardware approximations for cbrt/sqrt/divide */
};

typedef struct FcabConfig {
    int nrows, ncols;
    int precision;            /* FCAB_PREC_* */
    int math;                 /* FCAB_MATH_* */
    int K, U, boundary;       /* neighbours 4|8, dt reuse, FCA_BND_* */
    int edge_n, edge_s, edge_w, edge_e; /* open-boundary edges when boundary is open */
    int hyeto;                /* FCA_HYETO_* */
    int max_steps;            /* > 0: fixed step count (reference `steps`) */
    double dx, g, alpha, tau_h, tau_l, z_sea, dt_max, dt_min, S_bnd;
    double T_sim, out_every, D_h, phi;
    double rain_end;          /* > 0: no rain for steps starting at t >= rain_end (an event) */
    long long inflow_cell;    /* row*ncols+col of a LAND cell, or -1 */
    double inflow_peak;       /* triangular hydrograph: 0 at t=0, peak (m^3/s) at */
    double inflow_t_peak;     /*   inflow_t_peak, 0 at inflow_t_end; added after  */
    double inflow_t_end;      /*   the clamp, before hmax                         */
    int cols_per_lane;        /* 0 = autotuned (1 or 2); else 1, 2 or 4 (FP32 all-LAND
                                 grids: 2 runs the packed pair sweep, 4 with K = 4 two
                                 pairs per lane; padded fields beyond 2^31 elements run 1) */
    int seg_rows;             /* 0 = autotuned; rows per warp segment */
} FcabConfig;

typedef struct FcabStats {
    double t, dt_base;
    int step, done;
    double V, V0, V_rain, V_sea, V_bnd, clamp_err, V_in;
    long long cap_active, cap_total, dt_min_hits;
    double E_mass;            /* |V+V_sea+V_bnd-V_rain-V_in-V0-clamp| / (V_rain+V_in+V0) */
    long long dt_full_passes; /* steps whose dt needed the full velocity pass (seed missed) */
} FcabStats;

/* Error codes returned by the fcab_* calls (fcab_last_error() has the text). */
enum {
    FCAB_OK = 0,
    FCAB_ERR_ARG = -1,     /* invalid argument or unsupported combination */
    FCAB_ERR_CUDA = -2,    /* a CUDA call failed */
    FCAB_ERR_STATE = -3,   /* call out of order (e.g. advance before upload) */
    FCAB_ERR_IO = -4       /* file read failed */
};

/* Snapshot of the device step control, for host loops. */
typedef struct FcabPoll {
    double t, dt_base;
    int step, done, pause, force_day;
} FcabPoll;

/* Launch shape chosen for a session. */
typedef struct FcabInfo {
    int cols_per_lane, grid, warps, ctas_per_sm, rain_field, land_only;
    long long land_cells, faces_per_step, pitch;
    int tma_rows;             /* 1: the pair sweep reads rows by TMA (FCAB_ROW_SOURCE=tma) */
} FcabInfo;

typedef struct FcabSim FcabSim;

/* Fills cfg with the reference defaults (src/common/config.c:8-45) for an
 * nrows x ncols grid. */
FCAB_API void fcab_config_defaults(FcabConfig *cfg, int nrows, int ncols);

/* Creates a session on the current device. stream is a cudaStream_t (NULL:
 * the session creates its own). Returns 0 or a negative code. Before any
 * CUDA call it refuses (FCAB_ERR_ARG, message in fcab_last_error) an empty
 * or too large grid, K other than 4 or 8, U < 1, unknown precision, math,
 * boundary or hyetograph, non-positive or non-finite dx, g, alpha, dt_max
 * or dt_min, negative or non-finite tau_h / tau_l, non-finite z_sea, S_bnd,
 * T_sim, out_every, D_h, phi or rain_end, negative max_steps or seg_rows,
 * cols_per_lane other than 0, 1, 2 or 4, and a non-finite inflow
 * hydrograph. fcab_sim_upload refuses a non-finite z, h, n, C or Rday on a
 * LAND cell. */
FCAB_API int fcab_sim_create(FcabSim **out, const FcabConfig *cfg, void *stream);

/* Uploads row-major host fields of nrows*ncols values (float, or double for
 * FCAB_PREC_F64). n, C, Rday, hmax and tmax may be NULL: n = 0.03, C = Rday = 0,
 * hmax = h, tmax = 0 (FloodCA src/common/grid.c:197-235). Resets time,
 * step and accumulators; V0 is the LAND volume of h. */
FCAB_API int fcab_sim_upload(FcabSim *s, const void *z, const void *h, const void *n, const void *C,
                    const void *Rday, const uint8_t *mask, const void *hmax, const void *tmax);

/* Same, from device pointers with the session's element type. */
FCAB_API int fcab_sim_upload_device(FcabSim *s, const void *z, const void *h, const void *n,
                           const void *C, const void *Rday, const uint8_t *mask,
                           const void *hmax, const void *tmax);

/* Replaces the rain field C*Rday (host arrays; either may be NULL = unchanged). */
FCAB_API int fcab_sim_set_rain(FcabSim *s, const void *C, const void *Rday);

/* Enqueues up to nsteps steps on the session stream without waiting. Steps
 * after the end of the run (T_sim or max_steps) do nothing. */
FCAB_API int fcab_sim_advance(FcabSim *s, int nsteps);

/* Runs to the end of the run (T_sim or max_steps) and waits. */
FCAB_API int fcab_sim_run(FcabSim *s);

/* Sets the run clock (time, step count, held dt of the U-step reuse and the
 * loaded forcing day, -1 for none), recomputes V0 and the first step's dt.
 * fcab_sim_upload calls it with zeros. */
FCAB_API int fcab_sim_reset_time(FcabSim *s, double t, int step, double dt_base, int force_day);

/* Waits for the queued steps and reads the device step control. */
FCAB_API int fcab_sim_poll(FcabSim *s, FcabPoll *p);

/* Clears a pause (forcing day changed, or a progress point), recording the
 * forcing day now loaded. */
FCAB_API int fcab_sim_resume(FcabSim *s, int force_day);

/* Launch shape (strip width, grid) and grid statistics of the session. */
FCAB_API int fcab_sim_info(FcabSim *s, FcabInfo *info);

/* Changes the run parameters of a session (not its grid size, precision or
 * K); takes effect at the next fcab_sim_reset_time. */
FCAB_API int fcab_sim_set_config(FcabSim *s, const FcabConfig *cfg);

/* Pause the run every nsteps steps (0: never) and whenever the forcing day
 * index floor(t/86400) (clamped to n_force_days-1) differs from the loaded
 * one (n_force_days 0: no forcing days). */
FCAB_API int fcab_sim_set_pause_every(FcabSim *s, int nsteps, int n_force_days);

/* Uploads the dynamic state only (h; hmax = h when NULL; tmax = 0 when NULL);
 * the static fields stay resident. Call fcab_sim_reset_time afterwards. */
FCAB_API int fcab_sim_upload_state(FcabSim *s, const void *h, const void *hmax, const void *tmax);

/* Adds hmax >= thr[j] on LAND cells into the device array counts[j*N + a]
 * (uint16, N = nrows*ncols, at most 4 thresholds; NULL: no raster) and
 * returns the flooded cell counts and the largest LAND hmax (at least 0). */
FCAB_API int fcab_sim_count_flooded(FcabSim *s, int nthr, const double *thr, uint16_t *counts,
                           long long *flooded, double *max_depth);

/* The session's cudaStream_t. */
FCAB_API void *fcab_sim_stream(FcabSim *s);

/* Session buffers freed by fcab_sim_destroy (and by fca_cuda_run, which
 * destroys its session on return) are kept on their device for the next
 * session of about the same size, up to FCAB_CACHE_BYTES (environment;
 * default a quarter of the device memory; 0 disables). This frees them. */
FCAB_API void fcab_release_cached_memory(void);

/* ---- Slabs of a row-split domain (the reference's distributed run:
 * owned rows [r0, r1) of FcaGrid, src/common/fca_types.h:103-104, with
 * comm->halo and comm->min_real, src/common/model.c:143-144,359-360,
 * 507-508). A slab session holds its own rows (FcabConfig.nrows) plus up
 * to FCAB_SLAB_HALO rows of each neighbour; its step leaves the dt decision
 * pending until the velocity maximum has been max-reduced over all slabs. */
#define FCAB_SLAB_HALO 3

/* Before the upload: makes the session a slab with halo_n / halo_s halo
 * rows above / below (0..FCAB_SLAB_HALO; 0 on a domain edge). Every array
 * uploaded afterwards (fcab_sim_upload*, fcab_sim_set_rain,
 * fcab_sim_upload_state) carries halo_n + nrows + halo_s rows, and
 * FcabConfig.inflow_cell indexes such an array. Internal edges must be
 * closed in FcabConfig.edge_*. Slabs step only through fcab_sim_slab_*. */
FCAB_API int fcab_sim_set_slab(FcabSim *s, int halo_n, int halo_s);

/* One step on the slab's own rows; the next step's dt stays pending. */
FCAB_API int fcab_sim_slab_step(FcabSim *s);

/* The full velocity pass over the slab's own rows, when the last
 * fcab_sim_slab_finalize deferred dt (the reduced maximum of the seed-pruned
 * step fell below the seed; every slab defers alike); otherwise it returns at
 * once. The next step's dt is then pending again. */
FCAB_API int fcab_sim_slab_vfull(FcabSim *s);

/* Device address of the pending velocity maximum (an unsigned 64-bit
 * integer holding the bits of a non-negative float or double, so that an
 * integer max over slabs is the maximum velocity). */
FCAB_API int fcab_sim_slab_vmax(FcabSim *s, unsigned long long **vmax);

/* Prepares the next step from the (reduced) pending maximum; does nothing
 * when no decision is pending. */
FCAB_API int fcab_sim_slab_finalize(FcabSim *s);

/* Copies rows [row0, row0 + nrows) of the current depth (rows -halo_n ..
 * nrows + halo_s - 1) to a dense nrows x ncols device buffer, or back, in
 * the session's element type, on the session's stream. */
FCAB_API int fcab_sim_rows_get(FcabSim *s, int row0, int nrows, void *dst);
FCAB_API int fcab_sim_rows_put(FcabSim *s, int row0, int nrows, const void *src);

/* ---- Batched ensembles (no reference counterpart; the reference runs
 * members one at a time, src/hybrid/main_ens_mpi_cuda.c:69-120). ---- */
typedef struct FcabBatch FcabBatch;

typedef struct FcabBatchInfo {
    int members, cols_per_lane, seg_rows, grid, total_units;
    long long launches, windows, graph_replays;
} FcabBatchInfo;

/* Groups uploaded sessions into one batch. Members must share FP32
 * precision, K, math mode, rain form (uniform or field), mask form and
 * device; sizes, parameters, rain and time differ freely. cols_per_lane
 * (1, 2, 4; 0 = 2) sets the strip width of every member; a member's work
 * units are strips of member_seg_rows[i] rows (NULL: seg_rows for every
 * member; values <= 0 mean 64). stream: cudaStream_t or NULL (the first
 * member's). */
FCAB_API int fcab_batch_create(FcabBatch **out, FcabSim *const *members, int n,
                               int cols_per_lane, int seg_rows, const int *member_seg_rows,
                               void *stream);

/* Runs every member to the end of its run. One launch advances every active
 * member by one step. Each output window is one CUDA graph launch: the graph
 * opens the window and loops on the device (a conditional while node, passes
 * of graph_steps steps) until no member is active, so the host waits only at
 * window ends; without conditional graph support the host replays graphs of
 * graph_steps steps instead. window_s > 0 paces the members by output
 * windows: a window lasts until every member reaches its end (window_s
 * seconds of simulated time past the previous one; steps land on window ends
 * when out_every divides window_s), then the next window opens; max_windows
 * > 0 stops after that many windows.
 * window_s <= 0 runs every member freely to its end. Pacing never changes a
 * member's steps: they are those of its own session run alone. Members with
 * forcing days or progress pauses are refused at fcab_batch_create. Member
 * results are read with fcab_sim_stats / fcab_sim_download. */
FCAB_API int fcab_batch_run(FcabBatch *b, double window_s, int graph_steps, int max_windows);

FCAB_API int fcab_batch_info(FcabBatch *b, FcabBatchInfo *info);

FCAB_API void fcab_batch_destroy(FcabBatch *b);

/* Runs cfg->max_steps steps of the FP32 WCA step (the same fused kernel as
 * the sessions) on caller-owned device arrays, allocating nothing. No
 * counterpart in the reference. For callers that cannot call cudaMalloc:
 * processes whose device memory belongs to another allocator (a framework's
 * pool, an arena sized at start-up), or pipelines that must not allocate once
 * running, since cudaMalloc/cudaFree synchronise the device and stall other
 * streams. The working memory is one library-global device array of 2^19
 * padded cells (about 15 MB, held on every GPU that loads the library until
 * exit): (nrows + 16) * round_up(ncols + 132, 32) must not exceed 524288
 * (e.g. 512 x 768), else FCAB_ERR_ARG. Inputs z, n, mask (row-major
 * nrows*ncols, device), optional C and Rday (NULL: no rain); h and hmax are
 * read as the initial state and overwritten with the final state, tmax too
 * (NULL: start at 0, not written back); h, hmax and tmax must be distinct.
 * cfg->cols_per_lane and cfg->seg_rows set the launch shape as for sessions.
 * An inflow cell that is not LAND receives nothing (checked on the device).
 * stream: cudaStream_t, NULL for the legacy stream; without stats the call
 * only enqueues work on it and returns. stats (host, may be NULL) receives
 * the run totals after a stream synchronisation, cap_total and
 * dt_full_passes included. The first call on each device looks up the
 * array's device address; make that first call before any stream capture.
 * Calls share the array: calls that overlap on the GPU (other streams, other
 * host threads) race and corrupt each other. */
FCAB_API int fcab_run_noalloc(const FcabConfig *cfg, const float *z, const float *n,
                              const float *C, const float *Rday, const uint8_t *mask, float *h,
                              float *hmax, float *tmax, void *stream, FcabStats *stats);

/* Test hook: evaluates a device math helper on n host inputs and writes n
 * host outputs. which = 0: RN(cbrt(x*x)) as the exact mode computes
 * hf^(2/3); 1: min(x, RN(sqrt(g*y))); 2: the fast-mode hf^(2/3); 4/5/6: the
 * branch-free reciprocal, square root and Markstein quotient x/y; 7/8/9: the
 * IEEE reciprocal, square root and quotient they must equal; 10: the packed
 * pair sweep's hf^(2/3), NaN where it defers to the exact evaluation; 11: the
 * pair sweep's product then packed sum, RN(RN(x*y) + g), rounded twice. */
FCAB_API int fcab_math_probe(int which, const float *x, const float *y, float *out, long long n,
                             float g);

/* Waits, then fills st (computes the LAND volume V). */
FCAB_API int fcab_sim_stats(FcabSim *s, FcabStats *st);

/* Downloads h, hmax, tmax (any may be NULL) to host arrays. */
FCAB_API int fcab_sim_download(FcabSim *s, void *h, void *hmax, void *tmax);

/* Device pointers of the padded state, for zero-copy consumers: element
 * (r, c) is at base + (r + pad_rows) * pitch + c + pad_cols. */
FCAB_API int fcab_sim_layout(FcabSim *s, void **h, void **hmax, void **tmax, long long *pitch,
                    int *pad_rows, int *pad_cols);

/* Number of kernels the session has launched so far. */
FCAB_API long long fcab_sim_launches(FcabSim *s);

FCAB_API void fcab_sim_destroy(FcabSim *s);

/* Last error message of the calling thread ("" if none). */
FCAB_API const char *fcab_last_error(void);

/* Library build identification (e.g. "floodca_b200 sm_100a"). */
FCAB_API const char *fcab_version(void);

/* ---- Flood-depth surrogate layers (no reference counterpart: FloodCA has
 * no surrogate). Activations are bf16 matrices [N*(H+2)*(W+2)][C] of NHWC
 * images with a one-pixel zero border (C a multiple of 16); kernels write
 * interior pixels only, so borders stay zero once the buffer is zeroed.
 * Weights are [Cout][9][Cin] bf16 (tap = ky*3 + kx). All calls are
 * asynchronous on `stream` (cudaStream_t or NULL) and return 0 or an
 * FCAB_ERR_* code with fcab_last_error(). ---- */

/* y = conv3x3(x, w) (+ bias[Cout] fp32, ReLU when relu != 0). Cin % 16 == 0,
 * Cout % 32 == 0. tcgen05 tensor cores, FP32 accumulation. */
FCAB_API int fcab_unet_conv_fwd(const void *x, int N, int H, int W, int Cin, const void *w,
                                int Cout, const float *bias, int relu, void *y, void *stream);
/* dx[.][Cin] = data gradient of the convolution given dy[.][Cout] and the
 * flipped, transposed weights wt[Cin][9][Cout] (fcab_unet_prep_weights). */
FCAB_API int fcab_unet_conv_dgrad(const void *dy, int N, int H, int W, int Cout, const void *wt,
                                  int Cin, void *dx, void *stream);
/* dw[Cout][9][Cin] (fp32) += weight gradient from dy[.][Cout] and x[.][Cin]. */
FCAB_API int fcab_unet_conv_wgrad(const void *dy, const void *x, int N, int H, int W, int Cin,
                                  int Cout, float *dw, void *stream);
/* 2x2 max pooling of an (H, W) image; idx[N][H/2][W/2][C] records the arg max. */
FCAB_API int fcab_unet_maxpool2(const void *x, void *y, uint8_t *idx, int N, int H, int W, int C,
                                void *stream);
FCAB_API int fcab_unet_maxpool2_bwd(const void *dy, const uint8_t *idx, void *dx, int N, int H,
                                    int W, int C, void *stream);
/* The same plus add[.][add_off .. add_off+C) (row width Cadd): the skip
 * connection's share of a concatenation's gradient, added in one pass. */
FCAB_API int fcab_unet_maxpool2_bwd_add(const void *dy, const uint8_t *idx, const void *add,
                                        int Cadd, int add_off, void *dx, int N, int H, int W,
                                        int C, void *stream);
/* Nearest 2x upsampling of an (H, W) image; the backward sums 2x2 children. */
FCAB_API int fcab_unet_upsample2(const void *x, void *y, int N, int H, int W, int C, void *stream);
FCAB_API int fcab_unet_upsample2_bwd(const void *dy, void *dx, int N, int H, int W, int C,
                                     void *stream);
/* y = [a | b] along channels (backward != 0: split y into a and b). */
FCAB_API int fcab_unet_concat(const void *a, int Ca, const void *b, int Cb, void *y, int N, int H,
                              int W, int backward, void *stream);
/* y = [upsample2(coarse) | skip] for an (H, W) output in one pass, and the
 * gradient of its upsampled part: gcoarse, an (H/2, W/2) image, sums the
 * 2x2 children of gy[.][0..C1) (gy row width C1 + C2). */
FCAB_API int fcab_unet_upcat(const void *coarse, int C1, const void *skip, int C2, void *y, int N,
                             int H, int W, void *stream);
FCAB_API int fcab_unet_upcat_bwd(const void *gy, int C1, int C2, void *gcoarse, int N, int H,
                                 int W, void *stream);
/* y += x, n bf16 elements. */
FCAB_API int fcab_unet_add(void *y, const void *x, long long n, void *stream);
/* g *= (y > 0), n elements. */
FCAB_API int fcab_unet_relu_bwd(void *g, const void *y, long long n, void *stream);
/* In-place inverted dropout with a hashed mask of (seed, element). */
FCAB_API int fcab_unet_dropout(void *x, long long n, float p, uint32_t seed, void *stream);
/* db[c] += sum over the P rows of g[.][C]. */
FCAB_API int fcab_unet_bias_grad(const void *g, long long P, int C, float *db, void *stream);
/* 1x1 output head C -> 1 (C = 32 or 64): out[N][H][W] fp32. */
FCAB_API int fcab_unet_head_fwd(const void *x, const float *w, const float *b, float *out, int N,
                                int H, int W, int C, void *stream);
/* Mean squared error of out against target: dx (bf16), dw, db, loss sum
 * (accumulated). */
FCAB_API int fcab_unet_head_bwd(const void *x, const float *w, const float *out,
                                const float *target, void *dx, float *dw, float *db, float *loss,
                                int N, int H, int W, int C, void *stream);
/* fp32 master weights -> bf16 forward weights wb and dgrad weights wt. */
FCAB_API int fcab_unet_prep_weights(const float *w, void *wb, void *wt, int Cout, int Cin,
                                    void *stream);
/* Adam step t (>= 1) with decoupled-free L2 term wd. */
FCAB_API int fcab_unet_adam(float *w, const float *g, float *m, float *v, long long n, float lr,
                            float b1, float b2, float eps, int t, float wd, void *stream);
/* fp32 [N][H][W][Cs] -> bf16 bordered matrix with C >= Cs channels. */
FCAB_API int fcab_unet_pack_input(const float *in, int Cs, void *x, int C, int N, int H, int W,
                                  void *stream);
/* Returns and clears the device-side error code of these kernels (0: none;
 * nonzero: a pipeline wait gave up). */
FCAB_API int fcab_unet_device_error(void);
/* Failure-path probe: runs the kernels' bounded mbarrier wait on a barrier
 * that nothing completes, giving up after limit_cycles (1 to 2^32) SM
 * cycles; fcab_unet_device_error() then returns 10. */
FCAB_API int fcab_unet_wait_probe(long long limit_cycles, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* FLOODCA_B200_H */
