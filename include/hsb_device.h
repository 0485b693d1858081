/*
 * hsb_device.h -- the thin C-ABI between libhotspot_b200's C host code and
 * its sm_100a CUDA kernels.  Plain pointers, sizes and status codes only.
 *
 * The host side (grid_model.c) owns everything the reference computes once
 * per model -- layers, block<->grid maps, package R/C, per-cell detailed-3D
 * resistances, microchannel flow rates -- and hands the results to the device
 * model through these calls.  The device model keeps the grid state resident
 * in HBM and runs the hot loops that the reference runs on the CPU:
 *
 *   hsb_dev_transient  replaces compute_temp_grid's RK4 loop
 *                      (temperature_grid.c:3603-3704, RCutil.c:440-640,
 *                       slope_fn_grid/slope_fn_pack :3130-3601, :2857-3093)
 *   hsb_dev_steady     replaces steady_state_temp_grid's solver
 *                      (temperature_grid.c:2426-2851; the SuperLU-only
 *                       microchannel direct solve :5130-5194 becomes BiCGStab)
 *   b2g / g2b          xlate_vector_b2g / xlate_temp_g2b (:1888-2015) run on
 *                      the device inside the two calls above.
 *
 * Every function returns 0 on success or a negative HSB_E* code; the message
 * of the last failure on the calling thread is hsb_dev_last_error().
 */
#ifndef HSB_DEVICE_H
#define HSB_DEVICE_H

#ifdef __cplusplus
extern "C" {
#endif

#define HSB_OK            0
#define HSB_E_ARG        -1   /* invalid argument / state                */
#define HSB_E_CUDA       -2   /* CUDA runtime error                      */
#define HSB_E_NOMEM      -3   /* device allocation failed / over budget  */
#define HSB_E_NOCONV     -4   /* iteration cap reached without converging */
#define HSB_E_NODEV      -5   /* no CUDA device visible                  */

#define HSB_MAX_LAYERS   64

/* solver forms */
#define HSB_FORM_PARITY  0    /* FP64, replays the reference's operation order */
#define HSB_FORM_FAST    1    /* FP32 stencil work, FP64 state/refinement       */
#define HSB_FORM_FAST_STAGES 2  /* the fast transient evaluated stage by stage     */
#define HSB_FORM_FAST_PASSES 3  /* the fast transient with one grid-wide pass per Krylov
                                   vector (no temporal blocking); same arithmetic */
#define HSB_FORM_FP64_BLOCKED 4 /* transient: the temporally blocked Krylov form with every
                                   stencil pass in FP64 (per-layer models of 3..12 layers),
                                   within 1e-6 K of the FP64 replay; steady as HSB_FORM_PARITY */
#define HSB_FORM_FAST_BLOCKED 5 /* the fast transient on the temporally blocked kernel
                                   whatever the model's size (HSB_FORM_FAST takes it from
                                   2^21 cells up, the pass-by-pass kernel below) */

/* steady methods */
#define HSB_STEADY_AUTO       0  /* GS replay for FORM_PARITY; MG-PCG (or BiCGStab with advection) for FORM_FAST */
#define HSB_STEADY_GS_REPLAY  1  /* nested-iteration multigrid + exact-order Gauss-Seidel */
#define HSB_STEADY_MG         2  /* V-cycle preconditioned CG, FP32 inner, FP64 refinement */
#define HSB_STEADY_BICGSTAB   3  /* BiCGStab, FP32 inner, FP64 refinement (non-symmetric) */

typedef struct hsb_grid_desc {
  int nl, nr, nc;            /* layers, rows, cols (finest grid) */
  int n_extra;               /* 12, or 28 with the secondary path */
  int spidx, hsidx;          /* spreader / heat-sink layer indices */
  int subidx, solderidx, pcbidx;  /* secondary-path layers, -1 if absent */
  int field;                 /* 0: per-layer R/C (uniform); 1: per-cell arrays */
  int map_mode;              /* HSB_GRID_* block mapping for temperatures */
  int total_n_blocks;
  double ambient;
  double width, height;      /* die size (m): cell sizes of every multigrid level */
  double pcb_amb_num;        /* r_convec_sec * s_pcb^2, secondary path only */
  /* per layer (nl entries): the reference's layer_t rx, ry, rz, c */
  const double *layer_rx, *layer_ry, *layer_rz, *layer_c;
  const double *pack;        /* 52 doubles, package_RC_t field order */
} hsb_grid_desc;

typedef struct hsb_solver_opts {
  int form;                  /* HSB_FORM_* */
  int steady_method;         /* HSB_STEADY_* */
  double steady_tol;         /* FP64 residual target (K) for MG / BiCGStab */
  int max_iters;             /* cap on sweeps / cycles / Krylov iterations (0 = default) */
} hsb_solver_opts;

typedef struct hsb_stats {
  long long rk4_steps;       /* accepted RK4 steps */
  long long rk4_attempts;    /* RK4 attempts including rejected ones */
  long long slope_evals;     /* stencil evaluations */
  long long sweeps;          /* Gauss-Seidel sweeps, summed over levels */
  long long cycles;          /* V-cycles / Krylov iterations */
  long long refinements;     /* FP64 iterative-refinement passes */
  double residual;           /* final max |r| (W) of the FP64 residual, or last GS delta */
  double sim_time;           /* simulated seconds advanced */
  double device_ms;          /* device time of the call (CUDA events) */
  double kernel_ms;          /* device time of the solver kernels alone (CUDA events) */
  long long launches;        /* kernels this library launched during the call */
  long long fallbacks;       /* intervals the Krylov-form transient handed to the stage form */
} hsb_stats;

struct hsb_dev_model;
typedef struct hsb_dev_model hsb_dev_model;

int  hsb_dev_create(hsb_dev_model **out, const hsb_grid_desc *d);
void hsb_dev_destroy(hsb_dev_model *m);

/* per-layer values may change (populate_R_model re-called, natural convection) */
int hsb_dev_set_layers(hsb_dev_model *m, const double *rx, const double *ry,
                       const double *rz, const double *c, const double *pack52,
                       double ambient, double width, double height,
                       double pcb_amb_num);

/* per-cell detailed-3D coefficients; each array has nl*nr*nc entries.
 * r?[c] is the resistance between cell c and its N/S/W/E/above/below
 * neighbour exactly as find_res(neighbour, c) returns it (0 where absent). */
int hsb_dev_set_cells(hsb_dev_model *m, const double *rN, const double *rS,
                      const double *rW, const double *rE, const double *rA,
                      const double *rB, const double *cap);

/* microchannel advection per cell (nl*nr*nc each, zero outside channel
 * layers): aN..aE = Cv*flow(neighbour->cell) for fluid pairs, aO = outlet
 * self coefficient, qin = inlet source (W). */
int hsb_dev_set_advection(hsb_dev_model *m, const double *aN, const double *aS,
                          const double *aW, const double *aE, const double *aO,
                          const double *qin);

/* block->grid map: CSR over the nl*nr*nc cells, entries (block, occupancy,
 * block area); g2b: 5 ints per block (layer, i1, i2, j1, j2). */
int hsb_dev_set_maps(hsb_dev_model *m, const int *b2g_ptr, const int *b2g_blk,
                     const double *b2g_occ, const double *b2g_area,
                     double cell_area, const int *g2b);

int hsb_dev_transient(hsb_dev_model *m, const double *block_power,
                      const double *block_temp_in, double time_elapsed,
                      double *block_temp_out, const hsb_solver_opts *o,
                      hsb_stats *st);
int hsb_dev_steady(hsb_dev_model *m, const double *block_power,
                   double *block_temp_out, const hsb_solver_opts *o,
                   hsb_stats *st);
/* K consecutive sampling intervals (compute_temp_grid called K times,
 * temperature_grid.c:3603-3704) in one call: block_powers holds K block
 * power vectors (total_n_blocks + n_extra each, host), block_temp_in seeds
 * the state (or NULL), block_temp_out receives the block temperatures after
 * the last interval (or NULL).  With HSB_FORM_FAST the intervals run back
 * to back in one persistent launch, no host round trip between them; the
 * results equal K single-interval calls. */
int hsb_dev_transient_trace(hsb_dev_model *m, const double *block_powers, int K,
                            const double *block_temp_in, double time_elapsed,
                            double *block_temp_out, const hsb_solver_opts *o,
                            hsb_stats *st);

/* No counterpart in the reference.  For callers that may not allocate
 * device memory while they run (a simulator that reserves its GPU memory at
 * start-up and forbids later allocation, or a real-time loop that cannot
 * take cudaMalloc's implicit synchronisation): one sampling interval of the
 * fast transient form on a state y and a grid power vector pgrid that the
 * caller owns in device memory (nl*nr*nc + n_extra doubles each, y updated
 * in place), on the model's stream.  It calls no cudaMalloc/cudaFree: its
 * temporaries live in one static device array (about 2.8 MB, held by every
 * GPU that loads the library until exit) that fits models of at most
 * HSB_NOALLOC_MAX_CELLS cells, 4096 rows and 16384 columns, with per-layer
 * conductances; larger, more elongated or
 * per-cell (detailed 3-D, microchannel) models are rejected with
 * HSB_E_ARG.
 *   Ordering: y and pgrid are read on the model's stream, so whatever
 * wrote them must be complete before the call -- written on that stream, or
 * finished by a host synchronisation or an event the stream waited on.
 *   Blocking: the call waits on the host until the interval is done (it
 * reads the step counters back), so it must never be issued on a stream
 * that is being captured into a CUDA graph.
 *   The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress) and keeps it for the life of the process, so
 * cudaDeviceReset is not supported while the library is loaded.  All calls
 * share the array: calls that overlap on the GPU race.  Call with the
 * model's device current. */
#define HSB_NOALLOC_MAX_CELLS 65536
int hsb_dev_transient_noalloc(hsb_dev_model *m, double *y, const double *pgrid,
                              double time_elapsed, hsb_stats *st);

/* ---- batches: many models advanced together (no counterpart in the
 * reference, which simulates one chip per process; each chip's arithmetic is
 * the fast transient form of compute_temp_grid, temperature_grid.c:3603-3704).
 *
 * A batch references n existing device models (per-layer conductances, 3 to
 * 12 layers, primary or secondary heat path, one device);
 * hsb_batch_transient_trace advances all of them by K sampling intervals in
 * ONE persistent cooperative launch of the temporally blocked kernel,
 * replayed from a CUDA graph.  block_powers holds K rows, each row every
 * model's power vector (total_n_blocks + n_extra entries each, model after
 * model), or NULL to keep the grid powers of the last call (then K = 1).
 * Each model keeps its own adaptive step sequence; its state stays in its
 * own device model (hsb_dev_get_state, g2b through the model's entry
 * points).  hsb_batch_transient is the call with K = 1. */
struct hsb_batch;
typedef struct hsb_batch hsb_batch;
int  hsb_batch_create(hsb_batch **out, hsb_dev_model *const *models, int n);
void hsb_batch_destroy(hsb_batch *b);
int  hsb_batch_transient(hsb_batch *b, const double *block_power, double time_elapsed, hsb_stats *st);
int  hsb_batch_transient_trace(hsb_batch *b, const double *block_powers, int K, double time_elapsed,
                               hsb_stats *st);
/* schedule: tile policy (0: 16x64 tiles on chips of side >= 256, 16x32 on
 * 64..128, 32x32 below; 1: 32x32 tiles; 2: 16x32 tiles), and how finely big
 * models are split over CTA groups (1.0 = in proportion to their share of
 * the work) */
int  hsb_batch_set_schedule(hsb_batch *b, int policy, double split);
int  hsb_batch_info(hsb_batch *b, int *grid, long long *cells, int *policy, double *split);
/* accepted RK4 steps of each model in the last call (n entries) */
int  hsb_batch_chip_steps(hsb_batch *b, long long *steps);
/* at most `ctas` CTAs per launch (0: every co-resident CTA), so that other
 * work keeps SMs while a batch runs */
int  hsb_batch_set_ctas(hsb_batch *b, int ctas);
/* one launch advancing only the listed models (n indices) by K intervals;
 * block_powers: K rows, each the listed models' block vectors one after
 * another in list order; blocks until done */
int  hsb_batch_run_subset(hsb_batch *b, const int *chips, int n, const double *block_powers, int K,
                          double time_elapsed, hsb_stats *st);
/* where each model's block powers sit in a row: off[c] .. off[c + 1] (n + 1 entries) */
int  hsb_batch_offsets(hsb_batch *b, long long *off);
/* own-tile shape (rows x columns) of model c under the current schedule */
int  hsb_batch_chip_tile(hsb_batch *b, int c, int *rows, int *cols);
/* autotuner: when enabled, the next calls each run one candidate schedule
 * (tile policy, split) on the real work and the fastest per cell-step is
 * kept, and remembered for batches of the same shape in this process */
int  hsb_batch_autotune(hsb_batch *b, int enable);
/* the autotuner's measurements: 4 doubles per candidate (policy, split, 0,
 * ms per 1e9 cell-steps), up to n candidates; returns the count */
int  hsb_batch_tuning(hsb_batch *b, double *out, int n);

/* ---- serving (no counterpart in the reference): steady and transient
 * requests over resident models, admitted continuously.  Each request runs
 * on its model's stream, so the requests in flight overlap on the device; a
 * model serves one request at a time.  A request starts once it has arrived,
 * its model is idle, a worker is free and -- on the model's first request,
 * which allocates its solver workspace -- the device's free memory exceeds
 * that workspace plus the reserve; the least estimated work goes first. */
#define HSB_REQ_STEADY    0
#define HSB_REQ_TRANSIENT 1

typedef struct hsb_request {
  int model;                 /* index from hsb_server_add_model / _add_replica (its pool serves it) */
  int kind;                  /* HSB_REQ_STEADY or HSB_REQ_TRANSIENT */
  int steps;                 /* transient: sampling intervals */
  double dt;                 /* transient: interval length (s) */
  const double *power;       /* host block powers: 1 vector (steady) or `steps` vectors (transient) */
  const double *temp_in;     /* transient: initial block temperatures, or NULL to continue the state */
  double *out;               /* host block temperatures at the end (total_n_blocks + n_extra) */
  double arrival;            /* seconds after the start of hsb_server_run */
  double start, finish;      /* written by the server: seconds after the start */
  int status;                /* written by the server: HSB_OK or an HSB_E_* code */
  int worker;                /* written by the server */
} hsb_request;

struct hsb_server;
typedef struct hsb_server hsb_server;
int  hsb_server_create(hsb_server **out, int workers, long long reserve_bytes);
void hsb_server_destroy(hsb_server *s);
/* register a resident model; form HSB_FORM_*, steady_tol (K, 0 = default),
 * workspace_bytes = device memory its first solve allocates; returns its
 * index, which also names the model's pool */
int  hsb_server_add_model(hsb_server *s, hsb_dev_model *m, int form, double steady_tol,
                          long long workspace_bytes);
/* register m (same grid and block vector) as another member of `model`'s
 * pool, with its form, tolerance, workspace and priority; returns its index.
 * A request naming any member of a pool may be served by any idle member
 * (warm members first), except a transient request without temp_in, which
 * continues the state of the model it names and waits for that model. */
int  hsb_server_add_replica(hsb_server *s, int model, hsb_dev_model *m);
/* serve n requests (released at their arrival times); returns when all are done */
int  hsb_server_run(hsb_server *s, hsb_request *reqs, int n);
/* priority class of a registered model: its requests are dispatched before
 * normal ones and its kernels run on a high-priority stream (high = 1) */
int  hsb_server_set_priority(hsb_server *s, int model, int high);
/* continuous batching (on = 1): transient requests of normal-priority
 * fast-form models that the temporally blocked kernel takes are served by a
 * batch engine -- one launch advances every admitted transient of one
 * interval length by a few intervals (a tick); requests join and leave the
 * batch between ticks.  The batch is built at the next hsb_server_run over
 * the models registered then. */
int  hsb_server_set_batching(hsb_server *s, int on);
/* engine counters since the server was created: ticks (launches), the sum
 * over ticks of the requests each advanced, and of requests x intervals */
int  hsb_server_batch_stats(hsb_server *s, long long *ticks, long long *request_ticks,
                            long long *request_intervals);

/* run the model's work on a high-priority (high = 1) or normal stream; call
 * with no work of the model in flight */
int hsb_dev_set_priority(hsb_dev_model *m, int high);

/* own-tile shape (rows x columns) of the temporally blocked transient kernel
 * for this model (no counterpart in the reference): 0, 0 lets the library
 * choose by its cost model; otherwise rows x columns must be at most 1024
 * own cells (512 for more than six layers) and fit shared memory.  The
 * arithmetic of a cell does not depend on the tile; only the order of the
 * FP64 sums over grid edges does. */
int hsb_dev_set_tile(hsb_dev_model *m, int rows, int cols);

/* the temperature-leakage fixed point of the steady solve (temperature.c:
 * 706-746) on the device: height/width of each of the total_n_blocks blocks
 * (0 for blocks of layers without power), block_temp in: starting
 * temperatures, out: the result; *iterations: steady solves taken */
int hsb_dev_steady_leakage(hsb_dev_model *m, const double *block_power, const double *height,
                           const double *width, double *block_temp, const hsb_solver_opts *o,
                           int *iterations, hsb_stats *st);

/* which of the model's solver workspaces exist (no counterpart in the
 * reference): the fast transient, MG-PCG and BiCGStab solvers allocate
 * theirs on their first call; *mask = OR of HSB_WS_* */
#define HSB_WS_FAST_TRANSIENT 1
#define HSB_WS_MG             2
#define HSB_WS_BICGSTAB       4
int hsb_dev_workspaces(const hsb_dev_model *m, int *mask);

/* the kernel the fast transient form runs for this model (set at its first
 * fast interval): 0 none yet, or HSB_TK_* */
#define HSB_TK_BLOCKED      1   /* temporally blocked, FP32 passes */
#define HSB_TK_BLOCKED_FP64 2   /* temporally blocked, FP64 passes */
#define HSB_TK_PASSES       3   /* one grid-wide pass per Krylov vector */
int hsb_dev_transient_kernel(const hsb_dev_model *m, int *kind);

/* which: 0 = transient state (last_trans), 1 = steady state (last_steady);
 * n = nl*nr*nc + n_extra doubles */
int hsb_dev_get_state(hsb_dev_model *m, int which, double *out);
int hsb_dev_set_state(hsb_dev_model *m, int which, const double *in);

const char *hsb_dev_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
