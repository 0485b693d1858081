// mg_steady.cu -- converged steady state (HSB_STEADY_MG, the fast form).
//
// Solves the steady system of the grid model, G T = P (the fixed point the
// reference's Gauss-Seidel approaches, i.e. the system that
// build_transient_grid_matrix / build_transient_power_vector define,
// temperature_grid.c:5196-6694), to FP64 accuracy:
//
//   outer loop (FP64):  r = P - G T;  solve G e = r approximately;  T += e
//   inner solver (FP32): conjugate gradients preconditioned by one V-cycle
//
// V-cycle: cell-centred geometric multigrid that halves rows and columns
// (layers are kept), like the reference's own coarsening; coarse operators
// sum vertical/ambient/edge conductances over the 2x2 children and average
// the two lateral faces crossing a coarse face, so a uniform model gets
// exactly the reference's coarse R values (rz/4, rx and ry unchanged).
// Smoother: red-black z-line Gauss-Seidel -- every (i,j) column is solved
// exactly along z with a tridiagonal (Thomas) solve, which handles the thin,
// highly conductive TIM layers -- followed by an exact dense solve of the
// 12 package nodes given the grid.  Pre-smoothing runs red, black, package;
// post-smoothing package, black, red, so the preconditioner is symmetric.
// Restriction sums the 2x2 children, prolongation injects (its transpose).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dev_model.cuh"

namespace hsb {

#define MGT 256
#define NXP (HSB_EXTRA + HSB_EXTRA_SEC)   // package node slots of either path; the primary path uses 12
#ifndef MG_SWEEPS
#define MG_SWEEPS 1  // smoothing sweeps before and after each coarse-grid correction
#endif
#ifndef MG_INNER
#define MG_INNER 6   // PCG iterations of the first FP64 refinement pass
#endif
#ifndef MG_INNER_NEXT
#define MG_INNER_NEXT 3   // ... and of the later ones, which start from a small residual
#endif
// background solves of at least this many cells yield between PCG iterations
#define MG_YIELD_SPLIT_CELLS (1LL << 18)

struct PackSys {               // the 12 package nodes' equations
  float D[NXP];                // diagonal (edge cells + links + ambient) at level 0
  float link[NXP][NXP];        // conductance between package nodes
  float gamb[NXP];             // conductance to ambient
  int elayer[NXP], eside[NXP]; // attached edge: layer, side (0 N,1 S,2 W,3 E), -1 none
  float ge0[NXP];              // per-cell edge conductance at level 0
  int nx;                      // the model's nodes (12 or 28); the solves touch only these
};

struct MgLevelDev {
  int nr, nc, nl;
  long long plane, ncell;
  const float *gE, *gS, *gB;   // face conductances: (i,j)->(i,j+1), (i,j)->(i+1,j), n->n+1
  const float *diag;
  const float *gAmbL;          // per layer ambient conductance per cell
  const float *gEdgeNS, *gEdgeEW;  // per layer edge conductance per cell
  int el[5];                   // layers of the edge groups: sink, spreader, PCB, solder, substrate (-1 absent)
  float scale;                 // 2^level: edge conductances per coarse cell
  const float *pinv;           // NXP x NXP inverse of the package block
};

struct MgLevel {
  int nr, nc;
  long long plane, ncell, n;
  float *gE, *gS, *gB, *diag, *gAmbL, *gEdgeNS, *gEdgeEW;
  float *x, *f, *r;
  float *pinv;                 // NXP x NXP inverse of the package block at this level
};

struct MgWork {
  int nlev, coef_version;
  std::vector<MgLevel> lv;
  PackSys ps;
  PackSys *d_ps;
  // FP64 fine-level operator for the refinement residual
  double *gE64, *gS64, *gB64, *gAmb64, *gEdgeNS64, *gEdgeEW64;  // per cell (faces) / per layer
  double *r64, *b64;             // residual, right-hand side (vlen)
  // PCG vectors (fine level, FP32, n = ncell + 12)
  float *p, *q, *z, *e, *rr;
  double *red;                   // reduction scratch
  double *h_red;
  // one refinement pass (FP64 residual, inner PCG, correction) as a graph
  cudaGraphExec_t pass_exec, pass_exec_next;   // the first refinement pass; the later ones
  const double *pass_T;
  int pass_version;
  // the same pass in pieces (head + first iteration, one further iteration,
  // tail), for solves that yield between iterations
  cudaGraphExec_t piece_exec[3];
  const double *piece_T;
  int piece_version;
  // exact solve of the coarsest level: its dense FP64 inverse (cn x cn), or
  // none when the level is too large (then smoothing sweeps stand in)
  double *cinv;
  int cn;
  // levels fuse .. nlev-1 run as one single-CTA kernel in shared memory
  // (mg_cycle_fused); -1: every level kernel by kernel
  int fuse;
  size_t fuse_smem;
  unsigned *dot_ticket;          // last-block counter of dot_one (returns to 0 after each launch)
};

// ---------------------------------------------------------------------------
// operator application helpers
// ---------------------------------------------------------------------------
// the package node an edge of a layer couples to (side 0 N, 1 S, 2 W, 3 E):
// each edge group's nodes are numbered W, E, N, S from its W node
__host__ __device__ __forceinline__ int edge_node(int layer, int side, const int *el) {
  const int wnode[5] = {HSB_SINK_C_W, HSB_SP_W, HSB_PCB_C_W, HSB_SOLDER_W, HSB_SUB_W};
  for (int g = 0; g < 5; g++)
    if (layer == el[g]) return wnode[g] + ((side + 2) & 3);
  return -1;
}
__host__ __device__ __forceinline__ bool edge_layer(int layer, const int *el) {
  return layer == el[0] || layer == el[1] || layer == el[2] || layer == el[3] || layer == el[4];
}

// y = A x on level L (cells; the package rows by apply_pack_rows),
// written in difference form, gAmb x + sum g (x - x_nbr): the system is
// nearly singular (the overall temperature level is tied to ambient only
// through weak convection), and diag*x - sum g*x_nbr would cancel most FP32
// digits of smooth vectors
__device__ void apply_pack_rows(const MgLevelDev &L, const PackSys *__restrict__ ps, const float *__restrict__ x,
                                float *__restrict__ y, const float *__restrict__ f, int mode);

// ps != null: the grid has one more CTA, which applies the package rows
// (apply_pack_rows, in the same launch)
__global__ void mg_apply_cells(MgLevelDev L, const float *__restrict__ x, float *__restrict__ y,
                               const float *__restrict__ f, int mode, const PackSys *__restrict__ ps) {
  // mode 0: y = A x ; mode 1: y = f - A x
  if (ps && blockIdx.x == gridDim.x - 1) {
    apply_pack_rows(L, ps, x, y, f, mode);
    return;
  }
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.ncell) return;
  const int n = (int)(c / L.plane);
  const long long r = c - n * L.plane;
  const int i = (int)(r / L.nc), j = (int)(r - (long long)i * L.nc);
  const float xc = x[c];
  float s = L.gAmbL[n] * xc;
  if (j < L.nc - 1) s += L.gE[c] * (xc - x[c + 1]);
  if (j > 0) s += L.gE[c - 1] * (xc - x[c - 1]);
  if (i < L.nr - 1) s += L.gS[c] * (xc - x[c + L.nc]);
  if (i > 0) s += L.gS[c - L.nc] * (xc - x[c - L.nc]);
  if (n < L.nl - 1) s += L.gB[c] * (xc - x[c + L.plane]);
  if (n > 0) s += L.gB[c - L.plane] * (xc - x[c - L.plane]);
  const float *xp = x + L.ncell;
  if (edge_layer(n, L.el)) {
    if (i == 0) s += L.gEdgeNS[n] * (xc - xp[edge_node(n, 0, L.el)]);
    if (i == L.nr - 1) s += L.gEdgeNS[n] * (xc - xp[edge_node(n, 1, L.el)]);
    if (j == 0) s += L.gEdgeEW[n] * (xc - xp[edge_node(n, 2, L.el)]);
    if (j == L.nc - 1) s += L.gEdgeEW[n] * (xc - xp[edge_node(n, 3, L.el)]);
  }
  y[c] = mode ? f[c] - s : s;
}

// package rows (one CTA), difference form: ge sum_edge (x_k - x_c) +
// gamb x_k + sum link (x_k - x_o)
__device__ void apply_pack_rows(const MgLevelDev &L, const PackSys *__restrict__ ps, const float *__restrict__ x,
                                float *__restrict__ y, const float *__restrict__ f, int mode) {
  __shared__ float esum[NXP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const float *xp = x + L.ncell;
  for (int k = w; k < ps->nx; k += blockDim.x >> 5) {
    float s = 0.f;
    const int layer = ps->elayer[k], side = ps->eside[k];
    if (layer >= 0) {
      const int len = side < 2 ? L.nc : L.nr;
      const long long base = (long long)layer * L.plane +
                             (side == 0 ? 0 : side == 1 ? (long long)(L.nr - 1) * L.nc : side == 2 ? 0 : L.nc - 1);
      const long long st = side < 2 ? 1 : L.nc;
      const float xk = xp[k];
      for (int q = lane; q < len; q += 32) s += xk - x[base + q * st];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if (lane == 0) esum[k] = s;
  }
  __syncthreads();
  if (threadIdx.x < NXP) {   // the slots the model has no node for stay zero
    const int k = threadIdx.x;
    float v = 0.f;
    if (k < ps->nx) {
      const float ge = ps->ge0[k] * L.scale;
      float s = ge * esum[k] + ps->gamb[k] * xp[k];
      for (int o = 0; o < ps->nx; o++) s += ps->link[k][o] * (xp[k] - xp[o]);
      v = mode ? f[L.ncell + k] - s : s;
    }
    y[L.ncell + k] = v;
  }
}

// exact z-line solve of column `col` of level L (tridiagonal, Thomas)
__device__ __forceinline__ void zline_col(const MgLevelDev &L, float *__restrict__ x, const float *__restrict__ f,
                                          long long col) {
  const int i = (int)(col / L.nc), j = (int)(col - (long long)i * L.nc);
  const int nl = L.nl;
  float cp[HSB_MAX_LAYERS], dp[HSB_MAX_LAYERS];
  const float *xp = x + L.ncell;
  float prev_c = 0.f, prev_d = 0.f;
  for (int n = 0; n < nl; n++) {
    const long long c = (long long)n * L.plane + col;
    float rhs = f[c];
    if (j < L.nc - 1) rhs += L.gE[c] * x[c + 1];
    if (j > 0) rhs += L.gE[c - 1] * x[c - 1];
    if (i < L.nr - 1) rhs += L.gS[c] * x[c + L.nc];
    if (i > 0) rhs += L.gS[c - L.nc] * x[c - L.nc];
    if (edge_layer(n, L.el)) {
      if (i == 0) rhs += L.gEdgeNS[n] * xp[edge_node(n, 0, L.el)];
      if (i == L.nr - 1) rhs += L.gEdgeNS[n] * xp[edge_node(n, 1, L.el)];
      if (j == 0) rhs += L.gEdgeEW[n] * xp[edge_node(n, 2, L.el)];
      if (j == L.nc - 1) rhs += L.gEdgeEW[n] * xp[edge_node(n, 3, L.el)];
    }
    const float a = n > 0 ? -L.gB[c - L.plane] : 0.f;   // sub-diagonal
    const float cc = n < nl - 1 ? -L.gB[c] : 0.f;        // super-diagonal
    const float bd = L.diag[c];
    // Thomas forward elimination
    const float den = bd - a * prev_c;
    const float cn = cc / den;
    const float dn = (rhs - a * prev_d) / den;
    cp[n] = cn;
    dp[n] = dn;
    prev_c = cn;
    prev_d = dn;
  }
  float v = dp[nl - 1];
  x[(long long)(nl - 1) * L.plane + col] = v;
  for (int n = nl - 2; n >= 0; n--) {
    v = dp[n] - cp[n] * v;
    x[(long long)n * L.plane + col] = v;
  }
}

// the same for models of at most MAXL layers: every layer's loads are issued
// before the elimination starts (the arrays live in registers), so a column
// costs one memory round trip instead of one per layer.  x and f may be
// global or shared memory.
// ZERO: x is zero on entry (the first half sweep of a V-cycle level), so the
// right-hand side is f alone -- the neighbour and package terms all vanish
template <int MAXL, bool EXACT = false, bool ZERO = false>
__device__ __forceinline__ void zline_colT(const MgLevelDev &L, float *x, const float *f, int col) {
  const int nc = L.nc, nr = L.nr;
  const int i = col / nc, j = col - i * nc;
  const int nl = EXACT ? MAXL : L.nl;   // EXACT: the layer count is MAXL, every layer test is static
  const float *xp = x + L.ncell;
  // neighbour columns clamped to this one at the boundary, where the face
  // conductance is zero: every load is unconditional and can be in flight
  // at once; a zero weight adds exactly nothing
  const int dE = j < nc - 1 ? 1 : 0, dW = j > 0 ? 1 : 0;
  const int dS = i < nr - 1 ? nc : 0, dN = i > 0 ? nc : 0;
  float rhs[MAXL], gb[MAXL], bd[MAXL];
#pragma unroll
  for (int n = 0; n < MAXL; n++) {
    if (n < nl) {
      const long long c = (long long)n * L.plane + col;
      float r = f[c];
      if (!ZERO) {
        const float wE = dE ? L.gE[c] : 0.f, wW = dW ? L.gE[c - dW] : 0.f;
        const float wS = dS ? L.gS[c] : 0.f, wN = dN ? L.gS[c - dN] : 0.f;
        r += wE * x[c + dE];
        r += wW * x[c - dW];
        r += wS * x[c + dS];
        r += wN * x[c - dN];
      }
      if (!ZERO && edge_layer(n, L.el)) {
        if (i == 0) r += L.gEdgeNS[n] * xp[edge_node(n, 0, L.el)];
        if (i == nr - 1) r += L.gEdgeNS[n] * xp[edge_node(n, 1, L.el)];
        if (j == 0) r += L.gEdgeEW[n] * xp[edge_node(n, 2, L.el)];
        if (j == nc - 1) r += L.gEdgeEW[n] * xp[edge_node(n, 3, L.el)];
      }
      rhs[n] = r;
      gb[n] = n < nl - 1 ? L.gB[c] : 0.f;
      bd[n] = L.diag[c];
    }
  }
  float cp[MAXL], dp[MAXL];
  float prev_c = 0.f, prev_d = 0.f;
#pragma unroll
  for (int n = 0; n < MAXL; n++) {
    if (n < nl) {
      const float a = n > 0 ? -gb[n - 1] : 0.f;   // sub-diagonal
      const float cc = -gb[n];                     // super-diagonal (0 on the last layer)
      const float inv = 1.f / (bd[n] - a * prev_c);
      const float cn = cc * inv;
      const float dn = (rhs[n] - a * prev_d) * inv;
      cp[n] = cn;
      dp[n] = dn;
      prev_c = cn;
      prev_d = dn;
    }
  }
  float v = 0.f;
#pragma unroll
  for (int n = MAXL - 1; n >= 0; n--) {
    if (n < nl) {
      v = n == nl - 1 ? dp[n] : dp[n] - cp[n] * v;
      x[(long long)n * L.plane + col] = v;
    }
  }
}

// one colour of z-lines for models of exactly NL layers (columns < 2^31,
// checked at set-up)
// first: x holds no defined values yet and counts as zero -- this colour is
// solved from f alone and the other colour and the package nodes are set to
// zero (what a zeroing pass followed by this half sweep gives)
template <int NL>
__global__ void __launch_bounds__(MGT) mg_zline_t(MgLevelDev L, float *__restrict__ x, const float *__restrict__ f,
                                                  int color, int first) {
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= L.plane) return;
  const int i = col / L.nc, j = col - i * L.nc;
  if (first && blockIdx.x == 0 && threadIdx.x < NXP) x[L.ncell + threadIdx.x] = 0.f;
  if (((i + j) & 1) == color) {
    if (first) zline_colT<NL, true, true>(L, x, f, col);
    else zline_colT<NL, true>(L, x, f, col);
  } else if (first) {
#pragma unroll
    for (int n = 0; n < NL; n++) x[(long long)n * L.plane + col] = 0.f;
  }
}

// red-black z-line Gauss-Seidel half sweep on level L: solve A x = f
__global__ void mg_zline(MgLevelDev L, float *__restrict__ x, const float *__restrict__ f, int color) {
  long long col = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= L.plane) return;
  const int i = (int)(col / L.nc), j = (int)(col - (long long)i * L.nc);
  if (((i + j) & 1) != color) return;
  zline_col(L, x, f, col);
}

// exact solve of the package nodes with the grid fixed: x_pk = M^-1 (f_pk +
// ge * edge sums), M^-1 precomputed per level
__global__ void mg_pack_solve(MgLevelDev L, const PackSys *__restrict__ ps, float *__restrict__ x,
                              const float *__restrict__ f) {
  __shared__ float esum[NXP], rhs[NXP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = w; k < ps->nx; k += blockDim.x >> 5) {
    float s = 0.f;
    const int layer = ps->elayer[k], side = ps->eside[k];
    if (layer >= 0) {
      const int len = side < 2 ? L.nc : L.nr;
      const long long base = (long long)layer * L.plane +
                             (side == 0 ? 0 : side == 1 ? (long long)(L.nr - 1) * L.nc : side == 2 ? 0 : L.nc - 1);
      const long long st = side < 2 ? 1 : L.nc;
      for (int q = lane; q < len; q += 32) s += x[base + q * st];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if (lane == 0) esum[k] = s;
  }
  __syncthreads();
  if (threadIdx.x < ps->nx) {
    const int k = threadIdx.x;
    rhs[k] = f[L.ncell + k] + ps->ge0[k] * L.scale * esum[k];
  }
  __syncthreads();
  if (threadIdx.x < NXP) {
    const int k = threadIdx.x;
    float s = 0.f;
    if (k < ps->nx)
      for (int o = 0; o < ps->nx; o++) s += L.pinv[k * NXP + o] * rhs[o];
    x[L.ncell + k] = s;
  }
}

// the coarsest level in one CTA, from x = 0: `sweeps` pre-smoothing sweeps
// (red, black z-lines, package) then `sweeps` post-smoothing sweeps
// (package, black, red), the symmetric pattern of the per-kernel smoother
__global__ void __launch_bounds__(1024) mg_coarse_solve(MgLevelDev L, const PackSys *__restrict__ ps,
                                                        float *__restrict__ x, const float *__restrict__ f,
                                                        int sweeps) {
  __shared__ float esum[NXP], rhs[NXP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto zl = [&](int color) {
    for (long long col = threadIdx.x; col < L.plane; col += blockDim.x) {
      const int i = (int)(col / L.nc), j = (int)(col - (long long)i * L.nc);
      if (((i + j) & 1) == color) zline_col(L, x, f, col);
    }
    __syncthreads();
  };
  auto pk = [&]() {
    for (int k = w; k < ps->nx; k += blockDim.x >> 5) {
      float sm = 0.f;
      const int layer = ps->elayer[k], side = ps->eside[k];
      if (layer >= 0) {
        const int len = side < 2 ? L.nc : L.nr;
        const long long base = (long long)layer * L.plane +
                               (side == 0 ? 0 : side == 1 ? (long long)(L.nr - 1) * L.nc : side == 2 ? 0 : L.nc - 1);
        const long long st = side < 2 ? 1 : L.nc;
        for (int q = lane; q < len; q += 32) sm += x[base + q * st];
        for (int o = 16; o > 0; o >>= 1) sm += __shfl_down_sync(0xffffffffu, sm, o);
      }
      if (lane == 0) esum[k] = sm;
    }
    __syncthreads();
    if (threadIdx.x < ps->nx) rhs[threadIdx.x] = f[L.ncell + threadIdx.x] + ps->ge0[threadIdx.x] * L.scale * esum[threadIdx.x];
    __syncthreads();
    if (threadIdx.x < NXP) {
      float v = 0.f;
      if ((int)threadIdx.x < ps->nx)
        for (int o = 0; o < ps->nx; o++) v += L.pinv[threadIdx.x * NXP + o] * rhs[o];
      x[L.ncell + threadIdx.x] = v;
    }
    __syncthreads();
  };
  __syncthreads();
  for (int s = 0; s < sweeps; s++) {
    zl(0);
    zl(1);
    pk();
  }
  for (int s = 0; s < sweeps; s++) {
    pk();
    zl(1);
    zl(0);
  }
}

// exact solve of the coarsest level, x = A^-1 f, with its dense FP64 inverse
// (one CTA; the level has at most MG_COARSE_MAX unknowns)
#define MG_COARSE_MAX 2048
// x = inv f for the rows of warp w: four rows at a time, so that each lane
// has the loads of four rows in flight; per row the lane-strided partial
// sums and the shuffle tree are those of a one-row-per-warp loop
template <typename FV>
__device__ __forceinline__ void coarse_rows(const double *__restrict__ inv, int n, const FV *fv, float *x, int w,
                                            int nw, int lane) {
  for (int r0 = 4 * w; r0 < n; r0 += 4 * nw) {
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int c = lane; c < n; c += 32) {
      const double v = (double)fv[c];
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (r0 + q < n) acc[q] += inv[(long long)(r0 + q) * n + c] * v;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
      double sacc = acc[q];
      for (int o = 16; o > 0; o >>= 1) sacc += __shfl_down_sync(0xffffffffu, sacc, o);
      if (lane == 0 && r0 + q < n) x[r0 + q] = (float)sacc;
    }
  }
}
__global__ void __launch_bounds__(1024) mg_coarse_direct(const double *__restrict__ inv, int n,
                                                         float *__restrict__ x, const float *__restrict__ f) {
  __shared__ double fs[MG_COARSE_MAX];
  for (int k = threadIdx.x; k < n; k += blockDim.x) fs[k] = (double)f[k];
  __syncthreads();
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  coarse_rows(inv, n, fs, x, w, nw, lane);
}

// Transfers: cell-centred bilinear prolongation (each fine cell takes 9/16 of
// its parent, 3/16 of the two nearest coarse neighbours and 1/16 of the
// diagonal one, the pattern of the reference's multigrid_prolong_temp,
// temperature_grid.c:2616-2715; a neighbour outside the grid is replaced by
// the parent) and its transpose as restriction, so the V-cycle stays a
// symmetric preconditioner.  Layers are not coarsened; package values are
// carried over unchanged.

// 1-D weight with which fine index f contributes to coarse index c
__device__ __forceinline__ float bl_w(int f, int c, int cn) {
  const int par = f >> 1;
  int nb = par + ((f & 1) ? 1 : -1);
  nb = nb < 0 ? 0 : nb >= cn ? cn - 1 : nb;
  return (par == c ? 0.75f : 0.f) + (nb == c ? 0.25f : 0.f);
}

// coarse f = P^T r (each coarse cell gathers the 4x4 fine cells around it)
__global__ void mg_restrict_f(const float *__restrict__ rf, float *__restrict__ fc, int nl, int cnr,
                              int cnc, int nx) {
  const long long cpl = (long long)cnr * cnc, ncell = cpl * nl;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int fnr = 2 * cnr, fnc = 2 * cnc;
  const long long fpl = 4 * cpl;
  if (t < ncell) {
    const int n = (int)(t / cpl);
    const long long r = t - n * cpl;
    const int i = (int)(r / cnc), j = (int)(r - (long long)i * cnc);
    const float *s = rf + n * fpl;
    float acc = 0.f;
    for (int fi = 2 * i - 1; fi <= 2 * i + 2; fi++) {
      if (fi < 0 || fi >= fnr) continue;
      const float wi = bl_w(fi, i, cnr);
      if (wi == 0.f) continue;
      float row = 0.f;
      for (int fj = 2 * j - 1; fj <= 2 * j + 2; fj++) {
        if (fj < 0 || fj >= fnc) continue;
        const float wj = bl_w(fj, j, cnc);
        if (wj != 0.f) row += wj * s[(long long)fi * fnc + fj];
      }
      acc += wi * row;
    }
    fc[t] = acc;
  } else if (t < ncell + nx) {
    fc[t] = rf[fpl * nl + (t - ncell)];
  }
}

// fine x += P xc
__global__ void mg_prolong_add(const float *__restrict__ xc, float *__restrict__ xf, int nl, int cnr,
                               int cnc, int nx) {
  const int fnr = 2 * cnr, fnc = 2 * cnc;
  const long long fpl = (long long)fnr * fnc, cpl = (long long)cnr * cnc;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < fpl * nl) {
    const int n = (int)(t / fpl);
    const long long r = t - n * fpl;
    const int fi = (int)(r / fnc), fj = (int)(r - (long long)fi * fnc);
    const int ci = fi >> 1, cj = fj >> 1;
    int ci2 = ci + ((fi & 1) ? 1 : -1), cj2 = cj + ((fj & 1) ? 1 : -1);
    ci2 = ci2 < 0 ? 0 : ci2 >= cnr ? cnr - 1 : ci2;
    cj2 = cj2 < 0 ? 0 : cj2 >= cnc ? cnc - 1 : cj2;
    const float *c = xc + n * cpl;
    xf[t] += 0.5625f * c[(long long)ci * cnc + cj] + 0.1875f * c[(long long)ci2 * cnc + cj] +
             0.1875f * c[(long long)ci * cnc + cj2] + 0.0625f * c[(long long)ci2 * cnc + cj2];
  } else if (t < fpl * nl + nx) {
    xf[t] += xc[cpl * nl + (t - fpl * nl)];
  }
}

__global__ void mg_zero(float *x, long long n) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) x[t] = 0.f;
}

// ---------------------------------------------------------------------------
// The coarse end of the V-cycle in one CTA.  Below some size every level
// kernel is a few microseconds of launch and memory latency for very little
// work; levels fuse .. nlev-1 (planes of at most 16 x 16 columns) instead run
// here, with their x, f, r and coefficients in shared memory, in the order of the
// kernel-by-kernel cycle: zero x, MG_SWEEPS pre-smoothing sweeps (red z-lines,
// black z-lines, package nodes), r = f - A x, restriction, the coarser
// level, prolongation, MG_SWEEPS post-smoothing sweeps (package, black, red); the
// coarsest level by its dense FP64 inverse (read from global memory).
// ---------------------------------------------------------------------------
#define MG_FUSE_MAXLEV 8
#define MG_FUSE_THREADS 512
#define MG_FUSE_SMEM (200 * 1024)
#define MG_FUSE_PLANE 256

struct FusedArgs {
  MgLevelDev L[MG_FUSE_MAXLEV];
  int off[MG_FUSE_MAXLEV];   // float offset of level k's block in shared memory (fused_block_floats)
  int nf;                    // fused levels; the last is the coarsest
  const PackSys *ps;
  const double *cinv;        // coarsest level inverse (cn x cn)
  int cn;
  const float *f_in;         // right-hand side of the first fused level (global)
  float *x_out;              // its solution (global)
};

// a fused level's block of shared memory, in floats: x, f, r (n each), then
// its coefficients gE, gS, gB, diag (ncell each), the package inverse
// (NXP x NXP) and the per-layer ambient and edge conductances (3 x nl)
__host__ __device__ inline long long fused_block_floats(long long ncell, int nl) {
  const long long n = ncell + NXP;
  return (3 * n + 4 * ncell + NXP * NXP + 3 * nl + 3) / 4 * 4;
}

// phases of the fused coarse cycle (one CTA; each ends with a block barrier),
// kept out of line so the kernel's code stays small
// the z-lines of one colour (non-coarsest levels have an even column count)
template <int MAXL>
__device__ __noinline__ void fz_zl(const MgLevelDev &L, float *x, const float *f, int color) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int half = L.nc >> 1, ncol = (int)(L.plane >> 1);
  for (int k = tid; k < ncol; k += nt) {
    const int i = k / half, jj = k - i * half;
    const int j = 2 * jj + ((i + color) & 1);
    zline_colT<MAXL>(L, x, f, i * L.nc + j);
  }
  __syncthreads();
}

// package nodes with the grid fixed (mg_pack_solve)
__device__ __noinline__ void fz_pk(const MgLevelDev &L, const PackSys *ps, float *x, const float *f, float *esum,
                                   float *prhs) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int w = tid >> 5, lane = tid & 31, nw = nt >> 5;
  for (int k = w; k < ps->nx; k += nw) {
    float sm = 0.f;
    const int layer = ps->elayer[k], side = ps->eside[k];
    if (layer >= 0) {
      const int len = side < 2 ? L.nc : L.nr;
      const long long base = (long long)layer * L.plane +
                             (side == 0 ? 0 : side == 1 ? (long long)(L.nr - 1) * L.nc : side == 2 ? 0 : L.nc - 1);
      const long long st = side < 2 ? 1 : L.nc;
      for (int q = lane; q < len; q += 32) sm += x[base + q * st];
      for (int o = 16; o > 0; o >>= 1) sm += __shfl_down_sync(0xffffffffu, sm, o);
    }
    if (lane == 0) esum[k] = sm;
  }
  __syncthreads();
  if (tid < ps->nx) prhs[tid] = f[L.ncell + tid] + ps->ge0[tid] * L.scale * esum[tid];
  __syncthreads();
  if (tid < NXP) {   // the slots the model has no node for stay zero
    float v = 0.f;
    if (tid < ps->nx)
      for (int o = 0; o < ps->nx; o++) v += L.pinv[tid * NXP + o] * prhs[o];
    x[L.ncell + tid] = v;
  }
  __syncthreads();
}

// r = f - A x (mg_apply_cells with its package rows, mode 1)
__device__ __noinline__ void fz_resid(const MgLevelDev &L, const PackSys *ps, const float *x, const float *f, float *r,
                                      float *esum) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int w = tid >> 5, lane = tid & 31, nw = nt >> 5;
  const float *xp = x + L.ncell;
  const int plane = (int)L.plane, ncl = (int)L.ncell;
  for (int c = tid; c < ncl; c += nt) {
    const int n = c / plane;
    const int q = c - n * plane;
    const int i = q / L.nc, j = q - i * L.nc;
    const float xc = x[c];
    float s = L.gAmbL[n] * xc;
    if (j < L.nc - 1) s += L.gE[c] * (xc - x[c + 1]);
    if (j > 0) s += L.gE[c - 1] * (xc - x[c - 1]);
    if (i < L.nr - 1) s += L.gS[c] * (xc - x[c + L.nc]);
    if (i > 0) s += L.gS[c - L.nc] * (xc - x[c - L.nc]);
    if (n < L.nl - 1) s += L.gB[c] * (xc - x[c + L.plane]);
    if (n > 0) s += L.gB[c - L.plane] * (xc - x[c - L.plane]);
    if (edge_layer(n, L.el)) {
      if (i == 0) s += L.gEdgeNS[n] * (xc - xp[edge_node(n, 0, L.el)]);
      if (i == L.nr - 1) s += L.gEdgeNS[n] * (xc - xp[edge_node(n, 1, L.el)]);
      if (j == 0) s += L.gEdgeEW[n] * (xc - xp[edge_node(n, 2, L.el)]);
      if (j == L.nc - 1) s += L.gEdgeEW[n] * (xc - xp[edge_node(n, 3, L.el)]);
    }
    r[c] = f[c] - s;
  }
  for (int k = w; k < ps->nx; k += nw) {
    float sm = 0.f;
    const int layer = ps->elayer[k], side = ps->eside[k];
    if (layer >= 0) {
      const int len = side < 2 ? L.nc : L.nr;
      const long long base = (long long)layer * L.plane +
                             (side == 0 ? 0 : side == 1 ? (long long)(L.nr - 1) * L.nc : side == 2 ? 0 : L.nc - 1);
      const long long st = side < 2 ? 1 : L.nc;
      const float xk = xp[k];
      for (int q = lane; q < len; q += 32) sm += xk - x[base + q * st];
      for (int o = 16; o > 0; o >>= 1) sm += __shfl_down_sync(0xffffffffu, sm, o);
    }
    if (lane == 0) esum[k] = sm;
  }
  __syncthreads();
  if (tid < NXP) {   // the slots the model has no node for stay zero (shared memory is not)
    const int k = tid;
    float v = 0.f;
    if (k < ps->nx) {
      const float ge = ps->ge0[k] * L.scale;
      float s = ge * esum[k] + ps->gamb[k] * xp[k];
      for (int o = 0; o < ps->nx; o++) s += ps->link[k][o] * (xp[k] - xp[o]);
      v = f[L.ncell + k] - s;
    }
    r[L.ncell + k] = v;
  }
  __syncthreads();
}

// coarse f = P^T r (mg_restrict_f)
__device__ __noinline__ void fz_restrict(const MgLevelDev &F, const float *rf, const MgLevelDev &C, float *fc) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int cnr = C.nr, cnc = C.nc, fnr = F.nr, fnc = F.nc;
  const int cpl = (int)C.plane, fpl = (int)F.plane, cncell = (int)C.ncell;
  for (int t = tid; t < cncell + NXP; t += nt) {
    if (t < cncell) {
      const int n = t / cpl;
      const int q = t - n * cpl;
      const int i = q / cnc, j = q - i * cnc;
      const float *src = rf + n * fpl;
      float acc = 0.f;
      for (int fi = 2 * i - 1; fi <= 2 * i + 2; fi++) {
        if (fi < 0 || fi >= fnr) continue;
        const float wi = bl_w(fi, i, cnr);
        if (wi == 0.f) continue;
        float row = 0.f;
        for (int fj = 2 * j - 1; fj <= 2 * j + 2; fj++) {
          if (fj < 0 || fj >= fnc) continue;
          const float wj = bl_w(fj, j, cnc);
          if (wj != 0.f) row += wj * src[(long long)fi * fnc + fj];
        }
        acc += wi * row;
      }
      fc[t] = acc;
    } else {
      fc[t] = rf[F.ncell + (t - cncell)];
    }
  }
  __syncthreads();
}

// fine x += P xc (mg_prolong_add)
__device__ __noinline__ void fz_prolong(const MgLevelDev &C, const float *xc, const MgLevelDev &F, float *xf) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int cnr = C.nr, cnc = C.nc, fnc = F.nc;
  const int cpl = (int)C.plane, fpl = (int)F.plane, fncell = (int)F.ncell;
  for (int t = tid; t < fncell + NXP; t += nt) {
    if (t < fncell) {
      const int n = t / fpl;
      const int q = t - n * fpl;
      const int fi = q / fnc, fj = q - fi * fnc;
      const int ci = fi >> 1, cj = fj >> 1;
      int ci2 = ci + ((fi & 1) ? 1 : -1), cj2 = cj + ((fj & 1) ? 1 : -1);
      ci2 = ci2 < 0 ? 0 : ci2 >= cnr ? cnr - 1 : ci2;
      cj2 = cj2 < 0 ? 0 : cj2 >= cnc ? cnc - 1 : cj2;
      const float *c = xc + n * cpl;
      xf[t] += 0.5625f * c[(long long)ci * cnc + cj] + 0.1875f * c[(long long)ci2 * cnc + cj] +
               0.1875f * c[(long long)ci * cnc + cj2] + 0.0625f * c[(long long)ci2 * cnc + cj2];
    } else {
      xf[t] += xc[C.ncell + (t - fncell)];
    }
  }
  __syncthreads();
}

template <int MAXL>
__global__ void __launch_bounds__(MG_FUSE_THREADS) mg_cycle_fused(const __grid_constant__ FusedArgs A) {
  extern __shared__ __align__(16) float smf[];
  __shared__ float esum[NXP], prhs[NXP];
  __shared__ MgLevelDev SL[MG_FUSE_MAXLEV];   // the levels with their coefficients in shared memory
  __shared__ PackSys sps;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int w = tid >> 5, lane = tid & 31, nw = nt >> 5;
  const PackSys *ps = &sps;

  // stage every read-only table in shared memory: each phase below is then a
  // few shared-memory round trips instead of global-memory ones
  for (int q = tid; q < (int)(sizeof(PackSys) / 4); q += nt) ((int *)&sps)[q] = ((const int *)A.ps)[q];
  for (int k = 0; k < A.nf; k++) {
    const MgLevelDev &G = A.L[k];
    const long long n = G.ncell + NXP, nc = G.ncell;
    float *blk = smf + A.off[k];
    float *gE = blk + 3 * n, *gS = gE + nc, *gB = gS + nc, *dg = gB + nc, *pinv = dg + nc;
    float *amb = pinv + NXP * NXP, *ens = amb + G.nl, *eew = ens + G.nl;
    for (long long q = tid; q < nc; q += nt) {
      gE[q] = G.gE[q];
      gS[q] = G.gS[q];
      gB[q] = G.gB[q];
      dg[q] = G.diag[q];
    }
    for (int q = tid; q < NXP * NXP; q += nt) pinv[q] = G.pinv[q];
    for (int q = tid; q < G.nl; q += nt) {
      amb[q] = G.gAmbL[q];
      ens[q] = G.gEdgeNS[q];
      eew[q] = G.gEdgeEW[q];
    }
    if (tid == 0) {
      MgLevelDev L = G;
      L.gE = gE; L.gS = gS; L.gB = gB; L.diag = dg; L.pinv = pinv;
      L.gAmbL = amb; L.gEdgeNS = ens; L.gEdgeEW = eew;
      SL[k] = L;
    }
  }
  __syncthreads();


  const int nf = A.nf;
  {
    const long long n0 = SL[0].ncell + NXP;
    float *f0 = smf + A.off[0] + n0;
    for (long long q = tid; q < n0; q += nt) f0[q] = A.f_in[q];
  }
  __syncthreads();
  for (int k = 0; k < nf - 1; k++) {
    const MgLevelDev &L = SL[k];
    const long long n = L.ncell + NXP;
    float *x = smf + A.off[k], *f = x + n, *r = f + n;
    for (long long q = tid; q < n; q += nt) x[q] = 0.f;
    __syncthreads();
    for (int sw = 0; sw < MG_SWEEPS; sw++) {
      fz_zl<MAXL>(L, x, f, 0);
      fz_zl<MAXL>(L, x, f, 1);
      fz_pk(L, ps, x, f, esum, prhs);
    }
    fz_resid(L, ps, x, f, r, esum);
    const MgLevelDev &C = SL[k + 1];
    fz_restrict(L, r, C, smf + A.off[k + 1] + (C.ncell + NXP));
  }
  {   // coarsest: x = A^-1 f, one warp per row
    const MgLevelDev &C = SL[nf - 1];
    const long long n = C.ncell + NXP;
    float *x = smf + A.off[nf - 1], *f = x + n;
    coarse_rows(A.cinv, A.cn, f, x, w, nw, lane);
    __syncthreads();
  }
  for (int k = nf - 2; k >= 0; k--) {
    const MgLevelDev &L = SL[k], &C = SL[k + 1];
    const long long n = L.ncell + NXP;
    float *x = smf + A.off[k], *f = x + n;
    fz_prolong(C, smf + A.off[k + 1], L, x);
    for (int sw = 0; sw < MG_SWEEPS; sw++) {
      fz_pk(L, ps, x, f, esum, prhs);
      fz_zl<MAXL>(L, x, f, 1);
      fz_zl<MAXL>(L, x, f, 0);
    }
  }
  {
    const long long n0 = SL[0].ncell + NXP;
    const float *x0 = smf + A.off[0];
    for (long long q = tid; q < n0; q += nt) A.x_out[q] = x0[q];
  }
}

// coarse-level face conductances from the fine level
__global__ void mg_coarsen(const float *__restrict__ gEf, const float *__restrict__ gSf,
                           const float *__restrict__ gBf, float *__restrict__ gEc, float *__restrict__ gSc,
                           float *__restrict__ gBc, int nl, int cnr, int cnc) {
  const long long cpl = (long long)cnr * cnc;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cpl * nl) return;
  const int n = (int)(t / cpl);
  const long long r = t - n * cpl;
  const int i = (int)(r / cnc), j = (int)(r - (long long)i * cnc);
  const int fnc = 2 * cnc;
  const long long fo = (long long)n * 4 * cpl;
  const long long f00 = fo + (2 * i) * fnc + 2 * j, f10 = f00 + fnc;
  gEc[t] = j < cnc - 1 ? 0.5f * (gEf[f00 + 1] + gEf[f10 + 1]) : 0.f;
  gSc[t] = i < cnr - 1 ? 0.5f * (gSf[f10] + gSf[f10 + 1]) : 0.f;
  gBc[t] = gBf[f00] + gBf[f00 + 1] + gBf[f10] + gBf[f10 + 1];
}

// diagonal of level L from its faces, ambient and edge conductances
__global__ void mg_diag(MgLevelDev L, float *__restrict__ diag) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= L.ncell) return;
  const int n = (int)(c / L.plane);
  const long long r = c - n * L.plane;
  const int i = (int)(r / L.nc), j = (int)(r - (long long)i * L.nc);
  float d = L.gAmbL[n];
  if (j < L.nc - 1) d += L.gE[c];
  if (j > 0) d += L.gE[c - 1];
  if (i < L.nr - 1) d += L.gS[c];
  if (i > 0) d += L.gS[c - L.nc];
  if (n < L.nl - 1) d += L.gB[c];
  if (n > 0) d += L.gB[c - L.plane];
  if (edge_layer(n, L.el)) {
    if (i == 0) d += L.gEdgeNS[n];
    if (i == L.nr - 1) d += L.gEdgeNS[n];
    if (j == 0) d += L.gEdgeEW[n];
    if (j == L.nc - 1) d += L.gEdgeEW[n];
  }
  diag[c] = d;
}

// FP64 residual of the finest level: r = b - G T, returns max |r| via atomics
__global__ void fine_residual64(const hsb::StencilArgs S, const double *__restrict__ gE,
                                const double *__restrict__ gS, const double *__restrict__ gB,
                                const double *__restrict__ gAmb, const double *__restrict__ gENS,
                                const double *__restrict__ gEEW, const double *__restrict__ T,
                                const double *__restrict__ b, double *__restrict__ r, float *__restrict__ r32,
                                unsigned long long *maxbits) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double res = 0.0;
  if (c < S.ncell) {
    const int n = (int)(c / S.plane);
    const long long q = c - n * S.plane;
    const int i = (int)(q / S.nc), j = (int)(q - (long long)i * S.nc);
    const double Tc = T[c];
    double s = gAmb[n] * Tc;
    if (j < S.nc - 1) s += gE[c] * (Tc - T[c + 1]);
    if (j > 0) s += gE[c - 1] * (Tc - T[c - 1]);
    if (i < S.nr - 1) s += gS[c] * (Tc - T[c + S.nc]);
    if (i > 0) s += gS[c - S.nc] * (Tc - T[c - S.nc]);
    if (n < S.nl - 1) s += gB[c] * (Tc - T[c + S.plane]);
    if (n > 0) s += gB[c - S.plane] * (Tc - T[c - S.plane]);
    const double *x = T + S.ncell;
    const hsb::LayerCoef &Ln = S.L[n];
    // the edge group's W node (its nodes are W, E, N, S)
    const int k = Ln.kind;
    const int wn = k == hsb::LK_SINK ? HSB_SINK_C_W : k == hsb::LK_SPREADER ? HSB_SP_W
                   : k == hsb::LK_PCB ? HSB_PCB_C_W : k == hsb::LK_SOLDER ? HSB_SOLDER_W
                   : k == hsb::LK_SUB ? HSB_SUB_W : -1;
    if (wn >= 0) {
      if (i == 0) s += gENS[n] * (Tc - x[wn + 2]);
      if (i == S.nr - 1) s += gENS[n] * (Tc - x[wn + 3]);
      if (j == 0) s += gEEW[n] * (Tc - x[wn + 0]);
      if (j == S.nc - 1) s += gEEW[n] * (Tc - x[wn + 1]);
    }
    res = b[c] - s;
    r[c] = res;
    r32[c] = (float)res;
  }
  for (int o = 16; o > 0; o >>= 1) res = fmax(fabs(res), fabs(__shfl_down_sync(0xffffffffu, res, o)));
  if ((threadIdx.x & 31) == 0) atomicMax(maxbits, (unsigned long long)__double_as_longlong(fabs(res)));
}

// package rows of the FP64 residual (one CTA)
__global__ void pack_residual64(const hsb::StencilArgs S, const PackSys *__restrict__ ps,
                                const double *__restrict__ ge64, const double *__restrict__ link64,
                                const double *__restrict__ gamb64, const double *__restrict__ T,
                                const double *__restrict__ b, double *__restrict__ r,
                                float *__restrict__ r32, unsigned long long *maxbits) {
  __shared__ double esum[NXP];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int k = w; k < S.nx; k += blockDim.x >> 5) {
    double s = 0.0;
    const int layer = ps->elayer[k], side = ps->eside[k];
    if (layer >= 0) {
      const int len = side < 2 ? S.nc : S.nr;
      const long long base = (long long)layer * S.plane +
                             (side == 0 ? 0 : side == 1 ? (long long)(S.nr - 1) * S.nc : side == 2 ? 0 : S.nc - 1);
      const long long st = side < 2 ? 1 : S.nc;
      for (int q = lane; q < len; q += 32) s += T[S.ncell + k] - T[base + q * st];
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    }
    if (lane == 0) esum[k] = s;
  }
  __syncthreads();
  if (threadIdx.x < NXP) {   // the model's nodes; the state has no entries for inert ones (residual 0)
    const int k = threadIdx.x;
    double res = 0.0;
    if (k < S.nx) {
      const double *x = T + S.ncell;
      double s = ge64[k] * esum[k] + gamb64[k] * x[k];
      for (int o = 0; o < S.nx; o++) s += link64[k * NXP + o] * (x[k] - x[o]);
      res = b[S.ncell + k] - s;
    }
    r[S.ncell + k] = res;
    r32[S.ncell + k] = (float)res;
    atomicMax(maxbits, (unsigned long long)__double_as_longlong(fabs(res)));
  }
}

// ---------------------------------------------------------------------------
// PCG vector kernels (FP32 data, FP64 reductions in a fixed order)
// ---------------------------------------------------------------------------
// dot product in one launch: each block writes its partial, and the last
// block to finish (ticket counter, no waiting) adds the partials in block
// order; shift: the previous value of *out is first moved there (the PCG
// keeps rz_old beside rz)
__global__ void dot_one(const float *__restrict__ a, const float *__restrict__ b, long long n,
                        double *__restrict__ part, unsigned *__restrict__ ticket, double *out, double *shift) {
  __shared__ double sm[MGT / 32];
  __shared__ int last;
  double s = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
    s += (double)a[k] * (double)b[k];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < MGT / 32; w++) t += sm[w];
    part[blockIdx.x] = t;
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  s = 0.0;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) s += __ldcg(part + k);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < MGT / 32; w++) t += sm[w];
    if (shift) *shift = *out;
    *out = t;
    *ticket = 0u;
  }
}

// x += alpha p; r -= alpha q   with alpha = rz / pq  (sc[2] rz, sc[1] pq)
__global__ void pcg_update_xr(float *__restrict__ x, float *__restrict__ r, const float *__restrict__ p,
                              const float *__restrict__ q, const double *__restrict__ sc, long long n) {
  const double alpha = sc[2] / sc[1];
  const float a = (float)alpha;
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) {
    x[k] += a * p[k];
    r[k] -= a * q[k];
  }
}

// p = z + beta p with beta = rz_new / rz_old; the first iteration sets p = z
// without reading p (whatever the buffer held, NaN bit patterns included)
__global__ void pcg_update_p(float *__restrict__ p, const float *__restrict__ z, const double *__restrict__ sc,
                             long long n, int first) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  if (first) {
    p[k] = z[k];
    return;
  }
  const float beta = (float)(sc[2] / sc[0]);
  p[k] = z[k] + beta * p[k];
}

// T += e; the max |e| (K) into *emax_bits (zeroed by the caller)
__global__ void add_correction(double *__restrict__ T, const float *__restrict__ e, long long n,
                               unsigned long long *emax_bits) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double a = 0.0;
  if (k < n) {
    T[k] += (double)e[k];
    a = fabs((double)e[k]);
  }
  for (int o = 16; o > 0; o >>= 1) a = fmax(a, __shfl_down_sync(0xffffffffu, a, o));
  if ((threadIdx.x & 31) == 0 && a > 0.0) atomicMax(emax_bits, (unsigned long long)__double_as_longlong(a));
}

__global__ void copy_f(const float *__restrict__ a, float *__restrict__ b, long long n) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) b[k] = a[k];
}

// right-hand side in FP64: P + ambient conductances * ambient
__global__ void build_rhs64(const hsb::StencilArgs S, const double *__restrict__ pgrid,
                            const double *__restrict__ gAmb, const double *__restrict__ gamb64,
                            double *__restrict__ b) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c < S.ncell) {
    const int n = (int)(c / S.plane);
    b[c] = pgrid[c] + gAmb[n] * S.ambient;
  } else if (c < S.ncell + S.nx) {
    b[c] = gamb64[c - S.ncell] * S.ambient;
  }
}

// heuristic start in FP64 (set_heuristic_temp semantics, any precision)
__global__ void heuristic_start(const hsb::StencilArgs S, const double *__restrict__ p, double *__restrict__ v) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < S.plane) {
    double sum = 0.0;
    for (int n = 0; n < S.nl; n++) sum += p[n * S.plane + t];
    v[(S.nl - 1) * S.plane + t] = S.ambient + sum * S.L[S.nl - 1].rz;
    sum -= p[(S.nl - 1) * S.plane + t];
    for (int n = S.nl - 2; n >= 0; n--) {
      v[n * S.plane + t] = v[(n + 1) * S.plane + t] + S.L[n].rz * sum;
      sum -= p[n * S.plane + t];
    }
  }
  if (t < S.nx) v[S.ncell + t] = S.ambient;
}

// fine FP64 face conductances for a uniform model (1/R of the layer)
__global__ void uniform_faces64(const hsb::StencilArgs S, double *gE, double *gS, double *gB) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= S.ncell) return;
  const int n = (int)(c / S.plane);
  const long long q = c - n * S.plane;
  const int i = (int)(q / S.nc), j = (int)(q - (long long)i * S.nc);
  gE[c] = j < S.nc - 1 ? 1.0 / S.L[n].rEW : 0.0;
  gS[c] = i < S.nr - 1 ? 1.0 / S.L[n].rNS : 0.0;
  gB[c] = n < S.nl - 1 ? 1.0 / S.L[n].rz : 0.0;
}

// fine FP64 face conductances from per-cell resistances (detailed 3-D)
__global__ void field_faces64(const hsb::StencilArgs S, double *gE, double *gS, double *gB) {
  long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= S.ncell) return;
  const int n = (int)(c / S.plane);
  const long long q = c - n * S.plane;
  const int i = (int)(q / S.nc), j = (int)(q - (long long)i * S.nc);
  gE[c] = j < S.nc - 1 ? 1.0 / S.rE[c] : 0.0;
  gS[c] = i < S.nr - 1 ? 1.0 / S.rS[c] : 0.0;
  gB[c] = n < S.nl - 1 ? 1.0 / S.rB[c] : 0.0;
}

__global__ void d2f(const double *__restrict__ a, float *__restrict__ b, long long n) {
  long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) b[k] = (float)a[k];
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
static inline unsigned nb(long long n) { return (unsigned)((n + MGT - 1) / MGT); }

// the layers of the edge groups (sink, spreader, PCB, solder, substrate), -1 absent
static void edge_layers(const hsb_dev_model *m, int el[5]) {
  for (int g = 0; g < 5; g++) el[g] = -1;
  for (int n = 0; n < m->nl; n++) {
    const int k = m->hostL0[n].kind;
    const int g = k == LK_SINK ? 0 : k == LK_SPREADER ? 1 : k == LK_PCB ? 2 : k == LK_SOLDER ? 3 : k == LK_SUB ? 4 : -1;
    if (g >= 0) el[g] = n;
  }
}

static MgLevelDev dev_level(const hsb_dev_model *m, const MgLevel &L, int lvl) {
  MgLevelDev d;
  d.nr = L.nr; d.nc = L.nc; d.nl = m->nl;
  d.plane = L.plane; d.ncell = L.ncell;
  d.gE = L.gE; d.gS = L.gS; d.gB = L.gB; d.diag = L.diag;
  d.gAmbL = L.gAmbL; d.gEdgeNS = L.gEdgeNS; d.gEdgeEW = L.gEdgeEW;
  edge_layers(m, d.el);
  d.scale = (float)(1 << lvl);
  d.pinv = L.pinv;
  return d;
}

static void free_mg(void *p);

// workspace arrays start zeroed: no kernel of the solver depends on what an
// earlier allocation left in the memory it reuses.  The zeroing is ordered
// on the model's stream (a non-blocking stream does not wait for work on the
// legacy default stream: a plain cudaMemset there could land after the
// coefficients the solver's set-up kernels write)
template <typename Tp>
static cudaError_t mg_alloc(Tp **p, size_t bytes, cudaStream_t s) {
  cudaError_t e = cudaMalloc((void **)p, bytes);
  if (e == cudaSuccess) e = cudaMemsetAsync(*p, 0, bytes, s);
  return e;
}

static int mg_setup(hsb_dev_model *m, MgWork **out) {
  MgWork *w = new MgWork();
  w->coef_version = -1;
  const int nl = m->nl, nx = m->nx;
  // levels: halve while both sides are even and >= 4 (keep >= 2x2 columns)
  int nr = m->nr, nc = m->nc;
  while (true) {
    MgLevel L{};
    L.nr = nr; L.nc = nc;
    L.plane = (long long)nr * nc;
    L.ncell = L.plane * nl;
    L.n = L.ncell + nx;
    w->lv.push_back(L);
    if (nr < 8 || nc < 8 || (nr & 1) || (nc & 1) || L.plane <= 16) break;
    nr /= 2; nc /= 2;
  }
  w->nlev = (int)w->lv.size();
  for (int l = 0; l < w->nlev; l++) {
    MgLevel &L = w->lv[l];
    HSB_CUDA(mg_alloc(&L.gE, sizeof(float) * L.ncell, m->stream));
    HSB_CUDA(mg_alloc(&L.gS, sizeof(float) * L.ncell, m->stream));
    HSB_CUDA(mg_alloc(&L.gB, sizeof(float) * L.ncell, m->stream));
    HSB_CUDA(mg_alloc(&L.diag, sizeof(float) * L.ncell, m->stream));
    HSB_CUDA(mg_alloc(&L.gAmbL, sizeof(float) * HSB_MAX_LAYERS, m->stream));
    HSB_CUDA(mg_alloc(&L.gEdgeNS, sizeof(float) * HSB_MAX_LAYERS, m->stream));
    HSB_CUDA(mg_alloc(&L.gEdgeEW, sizeof(float) * HSB_MAX_LAYERS, m->stream));
    HSB_CUDA(mg_alloc(&L.x, sizeof(float) * L.n, m->stream));
    HSB_CUDA(mg_alloc(&L.f, sizeof(float) * L.n, m->stream));
    HSB_CUDA(mg_alloc(&L.r, sizeof(float) * L.n, m->stream));
    HSB_CUDA(mg_alloc(&L.pinv, sizeof(float) * NXP * NXP, m->stream));
  }
  const long long n0 = w->lv[0].n, ncell = m->ncell;
  HSB_CUDA(mg_alloc(&w->gE64, sizeof(double) * ncell, m->stream));
  HSB_CUDA(mg_alloc(&w->gS64, sizeof(double) * ncell, m->stream));
  HSB_CUDA(mg_alloc(&w->gB64, sizeof(double) * ncell, m->stream));
  HSB_CUDA(mg_alloc(&w->gAmb64, sizeof(double) * (HSB_MAX_LAYERS + 3 * NXP + NXP * NXP), m->stream));
  HSB_CUDA(mg_alloc(&w->gEdgeNS64, sizeof(double) * HSB_MAX_LAYERS, m->stream));
  HSB_CUDA(mg_alloc(&w->gEdgeEW64, sizeof(double) * HSB_MAX_LAYERS, m->stream));
  HSB_CUDA(mg_alloc(&w->r64, sizeof(double) * n0, m->stream));
  HSB_CUDA(mg_alloc(&w->b64, sizeof(double) * n0, m->stream));
  HSB_CUDA(mg_alloc(&w->p, sizeof(float) * n0, m->stream));
  HSB_CUDA(mg_alloc(&w->q, sizeof(float) * n0, m->stream));
  HSB_CUDA(mg_alloc(&w->z, sizeof(float) * n0, m->stream));
  HSB_CUDA(mg_alloc(&w->e, sizeof(float) * n0, m->stream));
  HSB_CUDA(mg_alloc(&w->rr, sizeof(float) * n0, m->stream));
  HSB_CUDA(mg_alloc(&w->red, sizeof(double) * 4096, m->stream));
  HSB_CUDA(mg_alloc(&w->d_ps, sizeof(PackSys), m->stream));
  HSB_CUDA(mg_alloc(&w->dot_ticket, sizeof(unsigned), m->stream));
  if (w->lv[0].plane >= (1LL << 31) - MGT) return set_error(HSB_E_ARG, "multigrid: more than 2^31 columns per layer");

  HSB_CUDA(cudaMallocHost(&w->h_red, sizeof(double) * 8));
  *out = w;
  return HSB_OK;
}

static void free_mg(void *p) {
  MgWork *w = (MgWork *)p;
  if (!w) return;
  for (auto &L : w->lv) {
    float *b[] = {L.gE, L.gS, L.gB, L.diag, L.gAmbL, L.gEdgeNS, L.gEdgeEW, L.x, L.f, L.r, L.pinv};
    for (float *q : b)
      if (q) cudaFree(q);
  }
  void *b2[] = {w->gE64, w->gS64, w->gB64, w->gAmb64, w->gEdgeNS64, w->gEdgeEW64, w->r64, w->b64,
                w->p, w->q, w->z, w->e, w->rr, w->red, w->d_ps, w->cinv, w->dot_ticket};
  for (void *q : b2)
    if (q) cudaFree(q);
  if (w->h_red) cudaFreeHost(w->h_red);
  if (w->pass_exec) cudaGraphExecDestroy(w->pass_exec);
  if (w->pass_exec_next) cudaGraphExecDestroy(w->pass_exec_next);
  for (auto &e : w->piece_exec)
    if (e) cudaGraphExecDestroy(e);
  delete w;
}

// build level operators from the device model's current conductances
static int mg_build(hsb_dev_model *m, MgWork *w) {
  const StencilArgs S = make_args(m, m->L0, m->nr, m->nc);
  const int nl = m->nl;
  const package_RC_t &pk = m->h_pk;
  // FP64 fine faces
  if (m->field) field_faces64<<<nb(m->ncell), MGT, 0, m->stream>>>(S, w->gE64, w->gS64, w->gB64);
  else uniform_faces64<<<nb(m->ncell), MGT, 0, m->stream>>>(S, w->gE64, w->gS64, w->gB64);
  // per-layer ambient and edge conductances (FP64 and per level FP32): the
  // sink's and, on the secondary path, the PCB's cells to ambient; the edge
  // cells of every edge group's layer to its package nodes
  double gamb[HSB_MAX_LAYERS] = {0}, gens[HSB_MAX_LAYERS] = {0}, geew[HSB_MAX_LAYERS] = {0};
  int el[5];
  edge_layers(m, el);
  for (int n = 0; n < nl; n++) {
    const LayerCoef &c = m->hostL0[n];
    if (c.kind == LK_SINK || c.kind == LK_PCB) gamb[n] = 1.0 / c.ramb;   // ramb is rz on the other layers
    if (edge_layer(n, el)) {
      gens[n] = 1.0 / c.edgeNS;
      geew[n] = 1.0 / c.edgeEW;
    }
  }
  // package system: the steady package equations of temperature_grid.c:
  // 2123-2379 (primary nodes, and the secondary path's PCB, solder and
  // substrate nodes), one row per node; nodes the model does not have are
  // inert (unit diagonal, no coupling, zero right-hand side)
  PackSys ps;
  memset(&ps, 0, sizeof(ps));
  double link64[NXP * NXP] = {0}, gamb_p[NXP] = {0}, ge_p[NXP] = {0};
  for (int k = 0; k < NXP; k++) ps.elayer[k] = -1;
  for (int k = m->nx; k < NXP; k++) gamb_p[k] = 1.0;
  auto link = [&](int a, int b, double r) {
    link64[a * NXP + b] += 1.0 / r;
    link64[b * NXP + a] += 1.0 / r;
  };
  auto edge = [&](int node, int layer, int side) {
    ps.elayer[node] = layer;
    ps.eside[node] = side;
    ge_p[node] = side < 2 ? gens[layer] : geew[layer];
  };
  const int nodesC[4] = {HSB_SINK_C_N, HSB_SINK_C_S, HSB_SINK_C_W, HSB_SINK_C_E};
  const int nodesO[4] = {HSB_SINK_N, HSB_SINK_S, HSB_SINK_W, HSB_SINK_E};
  const int nodesS[4] = {HSB_SP_N, HSB_SP_S, HSB_SP_W, HSB_SP_E};
  for (int s = 0; s < 4; s++) {
    const bool y = s < 2;
    gamb_p[nodesO[s]] = 1.0 / (pk.r_hs_per + pk.r_amb_per);
    link(nodesO[s], nodesC[s], (y ? pk.r_hs2_y : pk.r_hs2_x) + pk.r_hs);
    gamb_p[nodesC[s]] = 1.0 / (y ? pk.r_hs_c_per_y + pk.r_amb_c_per_y : pk.r_hs_c_per_x + pk.r_amb_c_per_x);
    link(nodesC[s], nodesS[s], y ? pk.r_sp_per_y : pk.r_sp_per_x);
    edge(nodesC[s], m->hsidx, s);
    edge(nodesS[s], m->spidx, s);
  }
  if (m->nx > HSB_EXTRA) {   // temperature_grid.c:2228-2379
    const int pO[4] = {HSB_PCB_N, HSB_PCB_S, HSB_PCB_W, HSB_PCB_E};
    const int pC[4] = {HSB_PCB_C_N, HSB_PCB_C_S, HSB_PCB_C_W, HSB_PCB_C_E};
    const int sO[4] = {HSB_SOLDER_N, HSB_SOLDER_S, HSB_SOLDER_W, HSB_SOLDER_E};
    const int bO[4] = {HSB_SUB_N, HSB_SUB_S, HSB_SUB_W, HSB_SUB_E};
    for (int s = 0; s < 4; s++) {
      const bool y = s < 2;
      gamb_p[pO[s]] = 1.0 / pk.r_amb_sec_per;
      link(pO[s], pC[s], (y ? pk.r_pcb2_y : pk.r_pcb2_x) + pk.r_pcb);
      gamb_p[pC[s]] = 1.0 / (y ? pk.r_amb_sec_c_per_y : pk.r_amb_sec_c_per_x);
      link(pC[s], sO[s], y ? pk.r_pcb_c_per_y : pk.r_pcb_c_per_x);
      link(sO[s], bO[s], y ? pk.r_solder_per_y : pk.r_solder_per_x);
      edge(pC[s], el[2], s);
      edge(sO[s], el[3], s);
      edge(bO[s], el[4], s);
    }
  }
  ps.nx = m->nx;
  for (int k = 0; k < NXP; k++) {
    ps.gamb[k] = (float)gamb_p[k];
    ps.ge0[k] = (float)ge_p[k];
    for (int o = 0; o < NXP; o++) ps.link[k][o] = (float)link64[k * NXP + o];
  }
  w->ps = ps;
  HSB_CUDA(cudaMemcpyAsync(w->d_ps, &ps, sizeof(ps), cudaMemcpyHostToDevice, m->stream));
  // the package block of every level (FP64 Gauss-Jordan, partial pivoting),
  // as the smoother's package solve uses it: D = cells * ge0 * 2^l + gamb + links
  for (int l = 0; l < w->nlev; l++) {
    const MgLevel &L = w->lv[l];
    double M[NXP][2 * NXP];
    for (int a = 0; a < NXP; a++) {
      const int cnt = ps.elayer[a] < 0 ? 0 : (ps.eside[a] < 2 ? L.nc : L.nr);
      const double ge = (double)ps.ge0[a] * (double)(1 << l);
      double D = cnt * ge + ps.gamb[a];
      for (int o = 0; o < NXP; o++) {
        D += ps.link[a][o];
        M[a][o] = -(double)ps.link[a][o];
        M[a][NXP + o] = a == o ? 1.0 : 0.0;
      }
      M[a][a] = D;
    }
    for (int c = 0; c < NXP; c++) {
      int piv = c;
      for (int r = c + 1; r < NXP; r++)
        if (fabs(M[r][c]) > fabs(M[piv][c])) piv = r;
      if (piv != c)
        for (int q = 0; q < 2 * NXP; q++) {
          const double t = M[c][q];
          M[c][q] = M[piv][q];
          M[piv][q] = t;
        }
      const double inv = 1.0 / M[c][c];
      for (int q = 0; q < 2 * NXP; q++) M[c][q] *= inv;
      for (int r = 0; r < NXP; r++)
        if (r != c && M[r][c] != 0.0) {
          const double fct = M[r][c];
          for (int q = 0; q < 2 * NXP; q++) M[r][q] -= fct * M[c][q];
        }
    }
    float inv32[NXP * NXP];
    for (int a = 0; a < NXP; a++)
      for (int o = 0; o < NXP; o++) inv32[a * NXP + o] = (float)M[a][NXP + o];
    HSB_CUDA(h2d_on(L.pinv, inv32, sizeof(inv32), m->stream));
  }
  double pack64[HSB_MAX_LAYERS + 3 * NXP + NXP * NXP];
  memcpy(pack64, gamb, sizeof(double) * HSB_MAX_LAYERS);
  memcpy(pack64 + HSB_MAX_LAYERS, ge_p, sizeof(double) * NXP);
  memcpy(pack64 + HSB_MAX_LAYERS + NXP, gamb_p, sizeof(double) * NXP);
  memcpy(pack64 + HSB_MAX_LAYERS + 3 * NXP, link64, sizeof(double) * NXP * NXP);
  HSB_CUDA(cudaMemcpyAsync(w->gAmb64, pack64, sizeof(pack64), cudaMemcpyHostToDevice, m->stream));
  HSB_CUDA(cudaMemcpyAsync(w->gEdgeNS64, gens, sizeof(double) * HSB_MAX_LAYERS, cudaMemcpyHostToDevice, m->stream));
  HSB_CUDA(cudaMemcpyAsync(w->gEdgeEW64, geew, sizeof(double) * HSB_MAX_LAYERS, cudaMemcpyHostToDevice, m->stream));
  // FP32 levels
  for (int l = 0; l < w->nlev; l++) {
    MgLevel &L = w->lv[l];
    float ga[HSB_MAX_LAYERS], gn[HSB_MAX_LAYERS], ge[HSB_MAX_LAYERS];
    const double mul4 = (double)(1ll << (2 * l)), mul2 = (double)(1ll << l);
    for (int n = 0; n < nl; n++) {
      ga[n] = (float)(gamb[n] * mul4);   // ambient per cell grows with the cell area
      gn[n] = (float)(gens[n] * mul2);   // an edge cell spans 2^l fine edge cells
      ge[n] = (float)(geew[n] * mul2);
    }
    HSB_CUDA(cudaMemcpyAsync(L.gAmbL, ga, sizeof(float) * nl, cudaMemcpyHostToDevice, m->stream));
    HSB_CUDA(cudaMemcpyAsync(L.gEdgeNS, gn, sizeof(float) * nl, cudaMemcpyHostToDevice, m->stream));
    HSB_CUDA(cudaMemcpyAsync(L.gEdgeEW, ge, sizeof(float) * nl, cudaMemcpyHostToDevice, m->stream));
    if (l == 0) {
      d2f<<<nb(L.ncell), MGT, 0, m->stream>>>(w->gE64, L.gE, L.ncell);
      d2f<<<nb(L.ncell), MGT, 0, m->stream>>>(w->gS64, L.gS, L.ncell);
      d2f<<<nb(L.ncell), MGT, 0, m->stream>>>(w->gB64, L.gB, L.ncell);
    } else {
      const MgLevel &F = w->lv[l - 1];
      mg_coarsen<<<nb(L.ncell), MGT, 0, m->stream>>>(F.gE, F.gS, F.gB, L.gE, L.gS, L.gB, nl, L.nr, L.nc);
    }
    mg_diag<<<nb(L.ncell), MGT, 0, m->stream>>>(dev_level(m, L, l), L.diag);
  }
  HSB_CUDA(cudaGetLastError());
  // the coarsest level exactly: the smoother cannot resolve the near-null
  // mode of the system (the overall temperature level, tied to ambient only
  // through the weak convection), so its operator is assembled on the host,
  // as mg_apply_cells applies it, and inverted once
  {
    const int lc = w->nlev - 1;
    const MgLevel &C = w->lv[lc];
    const long long n = C.ncell + NXP;
    if (w->cinv) {
      cudaFree(w->cinv);
      w->cinv = nullptr;
    }
    w->cn = 0;
    if (n <= MG_COARSE_MAX) {
      std::vector<float> gE(C.ncell), gS(C.ncell), gB(C.ncell), dg(C.ncell);
      HSB_CUDA(cudaMemcpyAsync(gE.data(), C.gE, sizeof(float) * C.ncell, cudaMemcpyDeviceToHost, m->stream));
      HSB_CUDA(cudaMemcpyAsync(gS.data(), C.gS, sizeof(float) * C.ncell, cudaMemcpyDeviceToHost, m->stream));
      HSB_CUDA(cudaMemcpyAsync(gB.data(), C.gB, sizeof(float) * C.ncell, cudaMemcpyDeviceToHost, m->stream));
      HSB_CUDA(cudaMemcpyAsync(dg.data(), C.diag, sizeof(float) * C.ncell, cudaMemcpyDeviceToHost, m->stream));
      HSB_CUDA(cudaStreamSynchronize(m->stream));
      const double scale = (double)(1ll << lc);
      std::vector<double> A((size_t)n * 2 * n, 0.0);   // [A | I], Gauss-Jordan in place
      auto at = [&](long long r, long long c) -> double & { return A[(size_t)r * 2 * n + c]; };
      const long long N = C.ncell, pl = C.plane;
      int el[5];
      edge_layers(m, el);
      auto node_of = [&](int layer, int side) -> int { return edge_node(layer, side, el); };
      for (long long c = 0; c < N; c++) {
        const int ln = (int)(c / pl);
        const long long q = c - ln * pl;
        const int i = (int)(q / C.nc), j = (int)(q - (long long)i * C.nc);
        at(c, c) = dg[c];
        if (j < C.nc - 1) at(c, c + 1) -= gE[c];
        if (j > 0) at(c, c - 1) -= gE[c - 1];
        if (i < C.nr - 1) at(c, c + C.nc) -= gS[c];
        if (i > 0) at(c, c - C.nc) -= gS[c - C.nc];
        if (ln < nl - 1) at(c, c + pl) -= gB[c];
        if (ln > 0) at(c, c - pl) -= gB[c - pl];
        if (edge_layer(ln, el)) {
          const float gn = (float)(gens[ln] * scale), gw = (float)(geew[ln] * scale);
          if (i == 0) at(c, N + node_of(ln, 0)) -= gn;
          if (i == C.nr - 1) at(c, N + node_of(ln, 1)) -= gn;
          if (j == 0) at(c, N + node_of(ln, 2)) -= gw;
          if (j == C.nc - 1) at(c, N + node_of(ln, 3)) -= gw;
        }
      }
      for (int k = 0; k < NXP; k++) {
        const int cnt = ps.elayer[k] < 0 ? 0 : (ps.eside[k] < 2 ? C.nc : C.nr);
        const float ge = ps.ge0[k] * (float)scale;
        float D = cnt * ge + ps.gamb[k];
        for (int o = 0; o < NXP; o++) D += ps.link[k][o];
        at(N + k, N + k) += D;
        for (int o = 0; o < NXP; o++) at(N + k, N + o) -= ps.link[k][o];
        if (ps.elayer[k] >= 0) {
          const int layer = ps.elayer[k], side = ps.eside[k];
          const int len = side < 2 ? C.nc : C.nr;
          const long long base = (long long)layer * pl +
                                 (side == 0 ? 0 : side == 1 ? (long long)(C.nr - 1) * C.nc : side == 2 ? 0 : C.nc - 1);
          const long long stp = side < 2 ? 1 : C.nc;
          for (int qq = 0; qq < len; qq++) at(N + k, base + qq * stp) -= ge;
        }
      }
      for (long long r = 0; r < n; r++) at(r, n + r) = 1.0;
      bool ok = true;
      for (long long c = 0; c < n && ok; c++) {
        long long piv = c;
        for (long long r = c + 1; r < n; r++)
          if (fabs(at(r, c)) > fabs(at(piv, c))) piv = r;
        if (at(piv, c) == 0.0) {
          ok = false;
          break;
        }
        if (piv != c)
          for (long long q2 = 0; q2 < 2 * n; q2++) std::swap(at(c, q2), at(piv, q2));
        const double inv = 1.0 / at(c, c);
        for (long long q2 = 0; q2 < 2 * n; q2++) at(c, q2) *= inv;
        for (long long r = 0; r < n; r++)
          if (r != c && at(r, c) != 0.0) {
            const double fct = at(r, c);
            for (long long q2 = c; q2 < 2 * n; q2++) at(r, q2) -= fct * at(c, q2);
          }
      }
      if (ok) {
        std::vector<double> inv((size_t)n * n);
        for (long long r = 0; r < n; r++)
          for (long long c = 0; c < n; c++) inv[(size_t)r * n + c] = at(r, n + c);
        HSB_CUDA(cudaMalloc(&w->cinv, sizeof(double) * n * n));
        HSB_CUDA(h2d_on(w->cinv, inv.data(), sizeof(double) * n * n, m->stream));
        w->cn = (int)n;
      }
    }
  }
  // the coarse levels that fuse into one single-CTA kernel: from the first
  // level of at most MG_FUSE_PLANE columns whose levels down to the coarsest
  // fit MG_FUSE_SMEM of shared memory (vectors and coefficients); needs the
  // exact coarsest inverse and at most 16 layers
  w->fuse = -1;
  w->fuse_smem = 0;
  if (w->cn > 0 && m->nl <= 16) {
    for (int l = 0; l < w->nlev; l++) {
      if (w->lv[l].plane > MG_FUSE_PLANE || w->nlev - l > MG_FUSE_MAXLEV) continue;
      size_t bytes = 0;
      for (int k = l; k < w->nlev; k++) bytes += sizeof(float) * (size_t)fused_block_floats(w->lv[k].ncell, m->nl);
      if (bytes > MG_FUSE_SMEM) continue;
      const void *fn = m->nl <= 8 ? (const void *)mg_cycle_fused<8> : (const void *)mg_cycle_fused<16>;
      int rc;
      if ((rc = raise_smem_limit(fn, bytes))) return rc;
      w->fuse = l;
      w->fuse_smem = bytes;
      break;
    }
  }
  return HSB_OK;
}

template <int NL>
static void zline_n(hsb_dev_model *m, const MgLevel &L, const MgLevelDev &d, float *x, const float *f, int color,
                    int first) {
  mg_zline_t<NL><<<nb(L.plane), MGT, 0, m->stream>>>(d, x, f, color, first);
}

// one colour of z-lines: the kernel compiled for the model's layer count
// (up to 16; first: x counts as zero, see mg_zline_t), else the generic one
static void zline(hsb_dev_model *m, const MgLevel &L, const MgLevelDev &d, float *x, const float *f, int color,
                  int first = 0) {
  if (first && m->nl > 16) mg_zero<<<nb(L.n), MGT, 0, m->stream>>>(x, L.n);
  switch (m->nl) {
    case 1: zline_n<1>(m, L, d, x, f, color, first); break;
    case 2: zline_n<2>(m, L, d, x, f, color, first); break;
    case 3: zline_n<3>(m, L, d, x, f, color, first); break;
    case 4: zline_n<4>(m, L, d, x, f, color, first); break;
    case 5: zline_n<5>(m, L, d, x, f, color, first); break;
    case 6: zline_n<6>(m, L, d, x, f, color, first); break;
    case 7: zline_n<7>(m, L, d, x, f, color, first); break;
    case 8: zline_n<8>(m, L, d, x, f, color, first); break;
    case 9: zline_n<9>(m, L, d, x, f, color, first); break;
    case 10: zline_n<10>(m, L, d, x, f, color, first); break;
    case 11: zline_n<11>(m, L, d, x, f, color, first); break;
    case 12: zline_n<12>(m, L, d, x, f, color, first); break;
    case 13: zline_n<13>(m, L, d, x, f, color, first); break;
    case 14: zline_n<14>(m, L, d, x, f, color, first); break;
    case 15: zline_n<15>(m, L, d, x, f, color, first); break;
    case 16: zline_n<16>(m, L, d, x, f, color, first); break;
    default: mg_zline<<<nb(L.plane), MGT, 0, m->stream>>>(d, x, f, color);
  }
}

// first: x counts as zero on entry (the pre-smoothing of a V-cycle level)
static void smooth(hsb_dev_model *m, MgWork *w, int l, float *x, const float *f, int pre, int sweeps,
                   int first = 0) {
  const MgLevel &L = w->lv[l];
  const MgLevelDev d = dev_level(m, L, l);
  for (int s = 0; s < sweeps; s++) {
    if (pre) {
      zline(m, L, d, x, f, 0, first && s == 0);
      zline(m, L, d, x, f, 1);
      mg_pack_solve<<<1, 384, 0, m->stream>>>(d, w->d_ps, x, f);
    } else {
      mg_pack_solve<<<1, 384, 0, m->stream>>>(d, w->d_ps, x, f);
      zline(m, L, d, x, f, 1);
      zline(m, L, d, x, f, 0);
    }
  }
}

// z = V-cycle(r) on level l (x <- approximate solution of A x = f, from x = 0)
static void vcycle(hsb_dev_model *m, MgWork *w, int l, float *x, const float *f) {
  const MgLevel &L = w->lv[l];
  if (l == w->fuse) {   // this level and all coarser ones in one kernel
    FusedArgs A;
    memset(&A, 0, sizeof(A));
    A.nf = w->nlev - l;
    long long off = 0;
    for (int k = 0; k < A.nf; k++) {
      A.L[k] = dev_level(m, w->lv[l + k], l + k);
      A.off[k] = (int)off;
      off += fused_block_floats(w->lv[l + k].ncell, m->nl);
    }
    A.ps = w->d_ps;
    A.cinv = w->cinv;
    A.cn = w->cn;
    A.f_in = f;
    A.x_out = x;
    if (m->nl <= 8) mg_cycle_fused<8><<<1, MG_FUSE_THREADS, w->fuse_smem, m->stream>>>(A);
    else mg_cycle_fused<16><<<1, MG_FUSE_THREADS, w->fuse_smem, m->stream>>>(A);
    return;
  }
  if (l == w->nlev - 1) {
    if (w->cn > 0) {
      mg_coarse_direct<<<1, 1024, 0, m->stream>>>(w->cinv, w->cn, x, f);   // writes every entry
    } else {
      mg_zero<<<nb(L.n), MGT, 0, m->stream>>>(x, L.n);
      mg_coarse_solve<<<1, 1024, 0, m->stream>>>(dev_level(m, L, l), w->d_ps, x, f, 8);
    }
    return;
  }
  const MgLevelDev d = dev_level(m, L, l);
  smooth(m, w, l, x, f, 1, MG_SWEEPS, 1);   // from x = 0: the first half sweep zeroes the rest
  mg_apply_cells<<<nb(L.ncell) + 1, MGT, 0, m->stream>>>(d, x, L.r, f, 1, w->d_ps);
  MgLevel &C = w->lv[l + 1];
  mg_restrict_f<<<nb(C.n), MGT, 0, m->stream>>>(L.r, C.f, m->nl, C.nr, C.nc, m->nx);
  vcycle(m, w, l + 1, C.x, C.f);
  mg_prolong_add<<<nb(L.n), MGT, 0, m->stream>>>(C.x, x, m->nl, C.nr, C.nc, m->nx);
  smooth(m, w, l, x, f, 0, MG_SWEEPS);
}

static int dot(hsb_dev_model *m, MgWork *w, const float *a, const float *b, long long n, double *out,
               double *shift = nullptr) {
  const int np = 296;
  dot_one<<<np, MGT, 0, m->stream>>>(a, b, n, w->red + 16, w->dot_ticket, out, shift);
  return HSB_OK;
}

int mg_steady(hsb_dev_model *m, const hsb_solver_opts *o, hsb_stats *st) {

  if (m->uchan_mask) return set_error(HSB_E_ARG, "advection makes the system non-symmetric: use BiCGStab");
  MgWork *w = (MgWork *)m->mg;
  int rc;
  if (!w) {
    if ((rc = mg_setup(m, &w))) return rc;
    m->mg = w;
    m->mg_free = free_mg;
  }
  if (w->coef_version != m->coef_version) {
    if ((rc = mg_build(m, w))) return rc;
    w->coef_version = m->coef_version;
  }
  const StencilArgs S = make_args(m, m->L0, m->nr, m->nc);
  const long long n0 = m->vlen;
  const double tol = (o && o->steady_tol > 0) ? o->steady_tol : 1e-7;
  const int max_ref = (o && o->max_iters > 0) ? o->max_iters : 60;
  double *T = m->ys;
  double *gambL = w->gAmb64, *ge_p = w->gAmb64 + HSB_MAX_LAYERS, *gamb_p = ge_p + NXP;
  double *link64 = w->gAmb64 + HSB_MAX_LAYERS + 3 * NXP;
  build_rhs64<<<nb(n0), MGT, 0, m->stream>>>(S, m->pgrid, gambL, gamb_p, w->b64);
  heuristic_start<<<nb(m->plane), MGT, 0, m->stream>>>(S, m->pgrid, T);
  HSB_CUDA(cudaGetLastError());
  const MgLevel &L0 = w->lv[0];
  const MgLevelDev d0 = dev_level(m, L0, 0);
  double *sc = w->red;   // [0] rz, [1] pq, [2] rz_new, [3] max|e| bits, [4] max|r| bits
  unsigned long long *maxbits = (unsigned long long *)(w->red + 4);
  const int inner = MG_INNER;
  // one refinement pass: r = b - G T (FP64), `inner` PCG iterations on
  // G e = r (FP32), T += e, |e|_2^2 to the host; the same kernel sequence
  // every time, so it is captured once as a CUDA graph and replayed
  auto head = [&]() {
    cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), m->stream);
    fine_residual64<<<nb(m->ncell), MGT, 0, m->stream>>>(S, w->gE64, w->gS64, w->gB64, gambL, w->gEdgeNS64,
                                                         w->gEdgeEW64, T, w->b64, w->r64, w->rr, maxbits);
    pack_residual64<<<1, 384, 0, m->stream>>>(S, w->d_ps, ge_p, link64, gamb_p, T, w->b64, w->r64, w->rr, maxbits);
    mg_zero<<<nb(n0), MGT, 0, m->stream>>>(w->e, n0);
  };
  auto iteration = [&](int it) {
    vcycle(m, w, 0, w->z, w->rr);
    dot(m, w, w->rr, w->z, n0, sc + 2, sc);   // rz (sc[2]); its previous value to sc[0]
    pcg_update_p<<<nb(n0), MGT, 0, m->stream>>>(w->p, w->z, sc, n0, it == 0);
    mg_apply_cells<<<nb(L0.ncell) + 1, MGT, 0, m->stream>>>(d0, w->p, w->q, nullptr, 0, w->d_ps);
    dot(m, w, w->p, w->q, n0, sc + 1);
    pcg_update_xr<<<nb(n0), MGT, 0, m->stream>>>(w->e, w->rr, w->p, w->q, sc, n0);
  };
  auto tail = [&]() {
    // the max norm of this correction (K) decides convergence
    cudaMemsetAsync(sc + 3, 0, sizeof(double), m->stream);
    add_correction<<<nb(n0), MGT, 0, m->stream>>>(T, w->e, n0, (unsigned long long *)(sc + 3));
    cudaMemcpyAsync(w->h_red, sc, sizeof(double) * 5, cudaMemcpyDeviceToHost, m->stream);
  };
  auto capture = [&](auto &&fn, cudaGraphExec_t *out, const char *what) -> int {
    if (*out) {
      cudaGraphExecDestroy(*out);
      *out = nullptr;
    }
    cudaGraph_t g;
    HSB_CUDA(cudaStreamBeginCapture(m->stream, cudaStreamCaptureModeThreadLocal));
    fn();
    const cudaError_t ce = cudaStreamEndCapture(m->stream, &g);
    if (ce != cudaSuccess) return cuda_check(ce, what);
    const cudaError_t ie = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
      *out = nullptr;
      return cuda_check(ie, what);
    }
    return HSB_OK;
  };
  // a background request (one a scheduler may hold, m->yield_fn) on a large
  // model runs each pass iteration by iteration and offers to yield between
  // them, so that it holds the device for one iteration at most after a
  // priority request arrives; otherwise one graph per pass
  const bool pieces = m->yield_fn && m->ncell >= MG_YIELD_SPLIT_CELLS && inner > 1;
  const int inner_next = MG_INNER_NEXT < inner ? MG_INNER_NEXT : inner;
  if (!pieces && (!w->pass_exec || w->pass_T != T || w->pass_version != m->coef_version)) {
    if ((rc = capture([&]() {
                        head();
                        for (int it = 0; it < inner; it++) iteration(it);
                        tail();
                      },
                      &w->pass_exec, "capturing the multigrid refinement pass")) ||
        (rc = capture([&]() {
                        head();
                        for (int it = 0; it < inner_next; it++) iteration(it);
                        tail();
                      },
                      &w->pass_exec_next, "capturing the later multigrid refinement passes")))
      return rc;
    w->pass_T = T;
    w->pass_version = m->coef_version;
  }
  if (pieces && (!w->piece_exec[0] || w->piece_T != T || w->piece_version != m->coef_version)) {
    if ((rc = capture([&]() {
                        head();
                        iteration(0);
                      },
                      &w->piece_exec[0], "capturing the multigrid pass head")) ||
        (rc = capture([&]() { iteration(1); }, &w->piece_exec[1], "capturing a multigrid pass iteration")) ||
        (rc = capture([&]() { tail(); }, &w->piece_exec[2], "capturing the multigrid pass tail")))
      return rc;
    w->piece_T = T;
    w->piece_version = m->coef_version;
  }
  // Stopping: the last correction is below tol, or the passes contract so
  // fast that the next correction -- the error left in T, estimated as
  // rho * |e_k| with rho = |e_k| / |e_k-1| -- is below tol / 10 (rho < 0.1).
  // Refinement passes contract at a steady rate set by the FP32 inner solve,
  // so the estimate saves the pass that would only confirm convergence.
  int refine = 0;
  double rmax = 0.0, emax = 1e300, eprev = 0.0;
  bool converged = false;
  for (refine = 0; refine < max_ref; refine++) {
    // the first pass takes the solution from the heuristic start; the later
    // ones correct an error the FP32 inner solve left, a few digits each
    const int n_it = refine == 0 ? inner : inner_next;
    if (pieces) {
      HSB_CUDA(cudaGraphLaunch(w->piece_exec[0], m->stream));
      for (int it = 1; it < n_it; it++) {
        HSB_CUDA(cudaStreamSynchronize(m->stream));
        m->yield_fn(m->yield_ctx);
        HSB_CUDA(cudaGraphLaunch(w->piece_exec[1], m->stream));
      }
      HSB_CUDA(cudaGraphLaunch(w->piece_exec[2], m->stream));
    } else {
      HSB_CUDA(cudaGraphLaunch(refine == 0 ? w->pass_exec : w->pass_exec_next, m->stream));
    }
    HSB_CUDA(cudaStreamSynchronize(m->stream));
    {
      unsigned long long bits;
      memcpy(&bits, w->h_red + 3, sizeof(bits));
      memcpy(&emax, &bits, sizeof(emax));
    }
    st->refinements += 1;
    st->cycles += n_it;
    if (emax < tol) {
      converged = true;
      break;
    }
    if (refine > 0 && eprev > 0.0) {
      const double rho = emax / eprev;
      if (rho < 0.1 && 10.0 * rho * emax < tol) {
        converged = true;
        break;
      }
    }
    eprev = emax;
    if (m->yield_fn) m->yield_fn(m->yield_ctx);
  }
  // final FP64 residual for the record
  HSB_CUDA(cudaMemsetAsync(maxbits, 0, sizeof(unsigned long long), m->stream));
  fine_residual64<<<nb(m->ncell), MGT, 0, m->stream>>>(S, w->gE64, w->gS64, w->gB64, gambL, w->gEdgeNS64,
                                                       w->gEdgeEW64, T, w->b64, w->r64, w->rr, maxbits);
  pack_residual64<<<1, 384, 0, m->stream>>>(S, w->d_ps, ge_p, link64, gamb_p, T, w->b64, w->r64, w->rr, maxbits);
  HSB_CUDA(cudaMemcpyAsync(w->h_red, sc, sizeof(double) * 5, cudaMemcpyDeviceToHost, m->stream));
  HSB_CUDA(cudaStreamSynchronize(m->stream));
  {
    unsigned long long bits;
    memcpy(&bits, w->h_red + 4, sizeof(bits));
    memcpy(&rmax, &bits, sizeof(rmax));
  }
  st->residual = rmax;
  if (!converged) return set_error(HSB_E_NOCONV, "multigrid steady solve did not converge");
  return HSB_OK;
}

}  // namespace hsb
