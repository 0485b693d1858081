// dev_model.cuh -- device-resident grid model shared by all kernels.
//
// HBM layout (one model):
//   state vectors are the reference's dcuboid_tail layout (util.c:231-261):
//   [nl][nr][nc] doubles followed by the n_extra package nodes, so a whole
//   vector is one contiguous array of ncell + nx doubles and cell
//   c = (n*nr + i)*nc + j.  Per-cell coefficient arrays (detailed 3-D and
//   microchannel models) use the same cell indexing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

extern "C" {
#include "hotspot_b200_types.h"
#include "hsb_device.h"
}

namespace hsb {

// kinds of layers with package terms (temperature_grid.c:2474-2589, 3193-3254)
enum LayerKind { LK_PLAIN = 0, LK_SPREADER, LK_SINK, LK_SUB, LK_SOLDER, LK_PCB };

// Per-layer coefficients of one multigrid level.  All resistances are the
// exact doubles the reference divides by, precomputed on the host with the
// reference's arithmetic (e.g. rNS = rx/2.0 + rx/2.0, temperature_grid.c:126).
struct LayerCoef {
  double rNS, rEW;        // lateral neighbour resistance, N/S and E/W
  double rz;              // rz of this layer: R to the layer below; ambient R for the sink
  double cap;             // capacitance of one cell
  double edgeNS, edgeEW;  // R to the package node on the N/S and E/W edges
  double ramb;            // R to ambient per cell (sink: rz; PCB: r_convec_sec share)
  int kind;               // LayerKind
  int pad;
};

struct StencilArgs {
  int nl, nr, nc, nx;
  long long plane, ncell;
  int field;              // per-cell coefficient arrays in use
  int secondary;
  unsigned long long uchan_mask;   // bit n set: layer n has advection terms
  double ambient;
  const LayerCoef *L;     // nl entries (device)
  const package_RC_t *pk; // device copy of the package R/C
  const double *rN, *rS, *rW, *rE, *rA, *rB, *cap;
  const double *aN, *aS, *aW, *aE, *aO, *qin;
};

struct LevelBuf {
  int nr, nc;
  double *p;              // power at this level (ncell + nx)
  double *v;              // temperature at this level (ncell + nx)
  LayerCoef *L;           // device per-layer table for this level
  LayerCoef hostL[HSB_MAX_LAYERS];
};

}  // namespace hsb

struct hsb_dev_model {
  int nl, nr, nc, nx;
  long long plane, ncell, vlen;   // vlen = ncell + nx
  int spidx, hsidx, subidx, solderidx, pcbidx;
  int field, map_mode, total_n_blocks;
  double ambient, width, height, pcb_amb_num;
  double h_rx[HSB_MAX_LAYERS], h_ry[HSB_MAX_LAYERS], h_rz[HSB_MAX_LAYERS], h_c[HSB_MAX_LAYERS];
  package_RC_t h_pk;
  int device;
  cudaStream_t stream;

  // state and work vectors (FP64, vlen each)
  double *y;          // transient state (last_trans)
  double *ys;         // steady state (last_steady)
  double *pgrid;      // grid power
  double *k1, *k2, *k3, *ytemp, *t1, *t2;
  unsigned long long *errbits;   // device max-norm accumulator
  double *h_err;                 // pinned host mirror
  package_RC_t *pk;   // device package R/C
  hsb::LayerCoef *L0; // finest-level layer table (device)
  hsb::LayerCoef hostL0[HSB_MAX_LAYERS];

  // per-cell coefficients (field mode)
  double *rN, *rS, *rW, *rE, *rA, *rB, *cap;
  // advection
  double *aN, *aS, *aW, *aE, *aO, *qin;
  unsigned long long uchan_mask;

  // block <-> grid maps
  int *b2g_ptr, *b2g_blk;
  double *b2g_occ, *b2g_area;
  double cell_area;
  int *g2b;
  double *blk_in, *blk_out;      // device block vectors (total_n_blocks + nx)
  double *trace_buf;             // block powers of a multi-interval call (trace_cap doubles)
  long long trace_cap;
  double *h_blk;                 // pinned staging: [0, nb) block powers in, [nb, 2 nb) block temperatures out
  cudaEvent_t ev[2];             // call timing events
  // the fast-form interval as CUDA graphs, one per (state buffers in their
  // roles, step, output request, coefficient version, kernel, g2b mode)
  struct IvGraph {
    const double *y, *y2;          // the two state buffers, in their roles at capture
    double T;
    int out, version, mode;
    const void *fn;
    cudaGraphExec_t exec;
  } ivg[4];
  int ivg_next;
  int ivg_off;                   // capture refused once: launch by launch from then on

  // multigrid levels for the exact nested-iteration replay
  int n_levels;
  hsb::LevelBuf *levels;
  int *gs_status;                // device: [0]=converged flag, [1]=sweeps done
  double *gs_delta;              // device: last sweep's max change
  int *h_gs;                     // pinned host mirror of gs_status
  double *h_gsd;

  // fast-form workspaces (allocated lazily by those solvers); coef_version
  // counts coefficient uploads so derived FP32 tables are rebuilt when stale
  int coef_version;
  // the fast transient's kernel: 0 the temporally blocked one where it
  // applies (rk4_tb.cu), 1 one grid-wide pass per Krylov vector (rk4_krylov.cu),
  // 2 the temporally blocked one with FP64 passes
  int fast_passes;
  int tile_oi, tile_oj;          // the blocked kernel's own tile requested for this model (0: automatic)
  void *fast;
  void (*fast_free)(void *);
  void *mg;
  void (*mg_free)(void *);
  void *krylov;
  void (*krylov_free)(void *);
  // called by the steady solvers between refinement passes (a scheduler
  // may hold a background request there); null: never
  void (*yield_fn)(void *);
  void *yield_ctx;
};

namespace hsb {

StencilArgs make_args(const hsb_dev_model *m, const LayerCoef *L, int nr, int nc);
int set_error(int code, const std::string &msg);
int cuda_check(cudaError_t e, const char *what);
// HSB_OK on cudaSuccess, else the error recorded as cuda_check records it
inline int cuda_ok(cudaError_t e, const char *what) { return e == cudaSuccess ? 0 : cuda_check(e, what); }
// raise (never lower) a kernel's dynamic shared memory limit, thread-safe
int raise_smem_limit(const void *fn, size_t bytes);

// b2g / g2b on the device (temperature_grid.c:1888-2015)
// host-to-device copy ordered on stream s, complete on return (a plain
// cudaMemcpy from pageable memory is ordered on the legacy default stream
// only, which non-blocking streams do not wait for)
inline cudaError_t h2d_on(void *dst, const void *src, size_t bytes, cudaStream_t s) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s);
  return e == cudaSuccess ? cudaStreamSynchronize(s) : e;
}
int b2g(hsb_dev_model *m, const double *blk_dev, double *grid_dev, int type);
// the steady solve from the block powers in m->blk_in to m->ys and the block
// temperatures in m->blk_out, all on the device
int steady_core(hsb_dev_model *m, const hsb_solver_opts *o, hsb_stats *st);
int g2b(hsb_dev_model *m, const double *grid_dev, double *blk_dev);
// the same on a given stream
int b2g_on(hsb_dev_model *m, const double *blk_dev, double *grid_dev, int type, cudaStream_t s);
int g2b_on(hsb_dev_model *m, const double *grid_dev, double *blk_dev, cudaStream_t s);

// exact-replay solvers
int rk4_exact_interval(hsb_dev_model *m, double time_elapsed, hsb_stats *st);
// the exact replay over [0, T) starting from step size h0 (the rest of an
// interval another form could not finish)
int rk4_exact_run(hsb_dev_model *m, double T, double h0, hsb_stats *st);
int gs_exact_steady(hsb_dev_model *m, const hsb_solver_opts *o, hsb_stats *st);

// fast-form solvers
int rk4_fast_stages_interval(hsb_dev_model *m, double time_elapsed, hsb_stats *st);
// one interval of the fast form in two halves (rk4_fast.cu)
int rk4_fast_interval_begin(hsb_dev_model *m, double time_elapsed, hsb_stats *st, void **work,
                            const double *bpow_dev);
int rk4_fast_interval_end(hsb_dev_model *m, void *work, double time_elapsed, hsb_stats *st, int *fell_back);
int rk4_fast_ready(hsb_dev_model *m, void **work, const void **kernel);
void fast_state_buffers(hsb_dev_model *m, void *work, double **second, const long long **which);
// g2b of whichever of two grid vectors *which selects (read on the device)
int g2b_select(hsb_dev_model *m, const double *g0, const double *g1, const long long *which, double *blk_dev);
// K consecutive intervals of the fast form from K block-power vectors in device memory
int rk4_fast_trace(hsb_dev_model *m, const double *bpow_dev, int K, double time_elapsed, hsb_stats *st);

// the fast transient kernel on caller-provided state, power and scratch
struct FastBuffers {
  double *y;                 // state, ncell + nx (in/out)
  const double *pgrid;       // grid power, ncell + nx
  float *pf, *k1, *k2, *k3;  // ncell each
  double *ytemp, *t1, *t2;   // ncell + nx each
  void *layer_table;         // rk4_fast_layer_table_bytes()
  void *pack_table;          // rk4_fast_pack_table_bytes()
  double *part;              // rk4_fast_part_bytes(m): per-tile edge partial sums
  unsigned long long *err;   // 2
  long long *cnt;            // 4
};
size_t rk4_fast_layer_table_bytes();
size_t rk4_fast_pack_table_bytes();
size_t rk4_fast_part_bytes(const hsb_dev_model *m);
int rk4_fast_on_buffers(hsb_dev_model *m, const FastBuffers &b, double time_elapsed, hsb_stats *st);
int mg_steady(hsb_dev_model *m, const hsb_solver_opts *o, hsb_stats *st);
int bicgstab_steady(hsb_dev_model *m, const hsb_solver_opts *o, hsb_stats *st);

}  // namespace hsb

#define HSB_CUDA(call)                                              \
  do {                                                              \
    cudaError_t _e = (call);                                        \
    if (_e != cudaSuccess) return hsb::cuda_check(_e, #call);       \
  } while (0)
