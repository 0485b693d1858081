// gs_exact.cu -- steady state in the reference's exact operation order
// (compiled with -fmad=false).
//
// The reference solves the steady state with "nested iteration"
// (recursive_multigrid, temperature_grid.c:2733-2797): restrict the power to
// ever coarser grids, start from a heuristic at the coarsest, and at every
// level run in-place lexicographic Gauss-Seidel sweeps over (n, i, j)
// followed by a sequential update of the package nodes, until the largest
// change of a sweep is below 1e-6 K.  Its result stops ~1e-3 K short of the
// converged fixed point, so matching it to 1e-6 K means replaying the same
// updates in the same order.
//
// Lexicographic GS is replayed exactly by a hyperplane wavefront: cell
// (n,i,j) reads its N, W and upper neighbours after their update in the
// same sweep and its S, E and lower neighbours before it; all three "before"
// neighbours lie on hyperplane n+i+j-1 and the "after" ones on n+i+j+1, so
// sweeping hyperplanes in order with all cells of one hyperplane in parallel
// performs exactly the reference's updates.  One CTA runs many sweeps
// back-to-back with a __syncthreads() per hyperplane; the level's vector
// lives in shared memory when it fits (227 KB/SM), else in L2-resident global
// memory.  Sweeps are bounded per launch so no launch runs unbounded.
#include <cmath>

#include "stencil_exact.cuh"

namespace hsb {

#define GS_THREADS 1024
#define GS_DELTA 1.0e-6

// One cell's in-place GS update (temperature_grid.c:2459-2604).
template <bool FIELD>
__device__ __forceinline__ double gs_cell(const StencilArgs &A, double *v, const double *__restrict__ p,
                                          int n, int i, int j, long long c) {
  const LayerCoef &Ln = A.L[n];
  double csum = 0.0, wsum = 0.0, R;
  // csum = NC + SC + EC + WC + AC + BC; wsum = NT + ST + ET + WT + AT + BT
  if (i > 0) { R = FIELD ? A.rN[c] : Ln.rNS; csum += 1.0 / R; wsum += v[c - A.nc] / R; }
  if (i < A.nr - 1) { R = FIELD ? A.rS[c] : Ln.rNS; csum += 1.0 / R; wsum += v[c + A.nc] / R; }
  if (j < A.nc - 1) { R = FIELD ? A.rE[c] : Ln.rEW; csum += 1.0 / R; wsum += v[c + 1] / R; }
  if (j > 0) { R = FIELD ? A.rW[c] : Ln.rEW; csum += 1.0 / R; wsum += v[c - 1] / R; }
  if (n > 0) { R = FIELD ? A.rA[c] : A.L[n - 1].rz; csum += 1.0 / R; wsum += v[c - A.plane] / R; }
  if (n < A.nl - 1) { R = FIELD ? A.rB[c] : Ln.rz; csum += 1.0 / R; wsum += v[c + A.plane] / R; }
  if (Ln.kind != LK_PLAIN) {
    const double *x = v + A.ncell;
    int eN, eS, eE, eW;
    switch (Ln.kind) {
      case LK_SPREADER: eN = HSB_SP_N; eS = HSB_SP_S; eE = HSB_SP_E; eW = HSB_SP_W; break;
      case LK_SINK:
        csum += 1.0 / Ln.ramb;
        wsum += A.ambient / Ln.ramb;
        eN = HSB_SINK_C_N; eS = HSB_SINK_C_S; eE = HSB_SINK_C_E; eW = HSB_SINK_C_W; break;
      case LK_PCB:
        csum += 1.0 / Ln.ramb;
        wsum += A.ambient / Ln.ramb;
        eN = HSB_PCB_C_N; eS = HSB_PCB_C_S; eE = HSB_PCB_C_E; eW = HSB_PCB_C_W; break;
      case LK_SUB: eN = HSB_SUB_N; eS = HSB_SUB_S; eE = HSB_SUB_E; eW = HSB_SUB_W; break;
      default: eN = HSB_SOLDER_N; eS = HSB_SOLDER_S; eE = HSB_SOLDER_E; eW = HSB_SOLDER_W; break;
    }
    if (i == 0) { csum += 1.0 / Ln.edgeNS; wsum += x[eN] / Ln.edgeNS; }
    if (i == A.nr - 1) { csum += 1.0 / Ln.edgeNS; wsum += x[eS] / Ln.edgeNS; }
    if (j == A.nc - 1) { csum += 1.0 / Ln.edgeEW; wsum += x[eE] / Ln.edgeEW; }
    if (j == 0) { csum += 1.0 / Ln.edgeEW; wsum += x[eW] / Ln.edgeEW; }
  }
  const double prev = v[c];
  const double nv = (p[c] + wsum) / csum;
  v[c] = nv;
  return fabs(prev - nv);
}

// Sequential package-node update (single_iteration_steady_pack,
// temperature_grid.c:2090-2393).  es[] are plain edge sums sum_k T_k in the
// order of edge_desc(); returns the largest change.
__device__ double gs_pack(const StencilArgs &A, double *v, const double *es, int nr, int nc,
                          int spidx, int hsidx, int subidx, int solderidx, int pcbidx) {
  const package_RC_t *pk = A.pk;
  const double amb = A.ambient;
  double *x = v + A.ncell;
  const LayerCoef &Ls = A.L[spidx], &Lh = A.L[hsidx];
  double delta[HSB_EXTRA + HSB_EXTRA_SEC];
  double csum, wsum, mx = 0;
  /* sink outer north/south */
  csum = 1.0 / (pk->r_hs_per + pk->r_amb_per) + 1.0 / (pk->r_hs2_y + pk->r_hs);
  wsum = amb / (pk->r_hs_per + pk->r_amb_per) + x[HSB_SINK_C_N] / (pk->r_hs2_y + pk->r_hs);
  delta[HSB_SINK_N] = fabs(x[HSB_SINK_N] - wsum / csum);
  x[HSB_SINK_N] = wsum / csum;
  wsum = amb / (pk->r_hs_per + pk->r_amb_per) + x[HSB_SINK_C_S] / (pk->r_hs2_y + pk->r_hs);
  delta[HSB_SINK_S] = fabs(x[HSB_SINK_S] - wsum / csum);
  x[HSB_SINK_S] = wsum / csum;
  /* sink outer west/east */
  csum = 1.0 / (pk->r_hs_per + pk->r_amb_per) + 1.0 / (pk->r_hs2_x + pk->r_hs);
  wsum = amb / (pk->r_hs_per + pk->r_amb_per) + x[HSB_SINK_C_W] / (pk->r_hs2_x + pk->r_hs);
  delta[HSB_SINK_W] = fabs(x[HSB_SINK_W] - wsum / csum);
  x[HSB_SINK_W] = wsum / csum;
  wsum = amb / (pk->r_hs_per + pk->r_amb_per) + x[HSB_SINK_C_E] / (pk->r_hs2_x + pk->r_hs);
  delta[HSB_SINK_E] = fabs(x[HSB_SINK_E] - wsum / csum);
  x[HSB_SINK_E] = wsum / csum;
  /* sink inner north/south */
  csum = nc / Lh.edgeNS;
  csum += 1.0 / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) + 1.0 / pk->r_sp_per_y +
          1.0 / (pk->r_hs2_y + pk->r_hs);
  wsum = es[0];
  wsum /= Lh.edgeNS;
  wsum += amb / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) + x[HSB_SP_N] / pk->r_sp_per_y +
          x[HSB_SINK_N] / (pk->r_hs2_y + pk->r_hs);
  delta[HSB_SINK_C_N] = fabs(x[HSB_SINK_C_N] - wsum / csum);
  x[HSB_SINK_C_N] = wsum / csum;
  wsum = es[1];
  wsum /= Lh.edgeNS;
  wsum += amb / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) + x[HSB_SP_S] / pk->r_sp_per_y +
          x[HSB_SINK_S] / (pk->r_hs2_y + pk->r_hs);
  delta[HSB_SINK_C_S] = fabs(x[HSB_SINK_C_S] - wsum / csum);
  x[HSB_SINK_C_S] = wsum / csum;
  /* sink inner west/east */
  csum = nr / Lh.edgeEW;
  csum += 1.0 / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) + 1.0 / pk->r_sp_per_x +
          1.0 / (pk->r_hs2_x + pk->r_hs);
  wsum = es[2];
  wsum /= Lh.edgeEW;
  wsum += amb / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) + x[HSB_SP_W] / pk->r_sp_per_x +
          x[HSB_SINK_W] / (pk->r_hs2_x + pk->r_hs);
  delta[HSB_SINK_C_W] = fabs(x[HSB_SINK_C_W] - wsum / csum);
  x[HSB_SINK_C_W] = wsum / csum;
  wsum = es[3];
  wsum /= Lh.edgeEW;
  wsum += amb / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) + x[HSB_SP_E] / pk->r_sp_per_x +
          x[HSB_SINK_E] / (pk->r_hs2_x + pk->r_hs);
  delta[HSB_SINK_C_E] = fabs(x[HSB_SINK_C_E] - wsum / csum);
  x[HSB_SINK_C_E] = wsum / csum;
  /* spreader north/south */
  csum = nc / Ls.edgeNS;
  csum += 1.0 / pk->r_sp_per_y;
  wsum = es[4];
  wsum /= Ls.edgeNS;
  wsum += x[HSB_SINK_C_N] / pk->r_sp_per_y;
  delta[HSB_SP_N] = fabs(x[HSB_SP_N] - wsum / csum);
  x[HSB_SP_N] = wsum / csum;
  wsum = es[5];
  wsum /= Ls.edgeNS;
  wsum += x[HSB_SINK_C_S] / pk->r_sp_per_y;
  delta[HSB_SP_S] = fabs(x[HSB_SP_S] - wsum / csum);
  x[HSB_SP_S] = wsum / csum;
  /* spreader west/east */
  csum = nr / Ls.edgeEW;
  csum += 1.0 / pk->r_sp_per_x;
  wsum = es[6];
  wsum /= Ls.edgeEW;
  wsum += x[HSB_SINK_C_W] / pk->r_sp_per_x;
  delta[HSB_SP_W] = fabs(x[HSB_SP_W] - wsum / csum);
  x[HSB_SP_W] = wsum / csum;
  wsum = es[7];
  wsum /= Ls.edgeEW;
  wsum += x[HSB_SINK_C_E] / pk->r_sp_per_x;
  delta[HSB_SP_E] = fabs(x[HSB_SP_E] - wsum / csum);
  x[HSB_SP_E] = wsum / csum;

  if (A.secondary) {
    const LayerCoef &Lp = A.L[pcbidx], &Lq = A.L[solderidx], &Lb = A.L[subidx];
    /* PCB outer north/south */
    csum = 1.0 / (pk->r_amb_sec_per) + 1.0 / (pk->r_pcb2_y + pk->r_pcb);
    wsum = amb / (pk->r_amb_sec_per) + x[HSB_PCB_C_N] / (pk->r_pcb2_y + pk->r_pcb);
    delta[HSB_PCB_N] = fabs(x[HSB_PCB_N] - wsum / csum);
    x[HSB_PCB_N] = wsum / csum;
    wsum = amb / (pk->r_amb_sec_per) + x[HSB_PCB_C_S] / (pk->r_pcb2_y + pk->r_pcb);
    delta[HSB_PCB_S] = fabs(x[HSB_PCB_S] - wsum / csum);
    x[HSB_PCB_S] = wsum / csum;
    /* PCB outer west/east */
    csum = 1.0 / (pk->r_amb_sec_per) + 1.0 / (pk->r_pcb2_x + pk->r_pcb);
    wsum = amb / (pk->r_amb_sec_per) + x[HSB_PCB_C_W] / (pk->r_pcb2_x + pk->r_pcb);
    delta[HSB_PCB_W] = fabs(x[HSB_PCB_W] - wsum / csum);
    x[HSB_PCB_W] = wsum / csum;
    wsum = amb / (pk->r_amb_sec_per) + x[HSB_PCB_C_E] / (pk->r_pcb2_x + pk->r_pcb);
    delta[HSB_PCB_E] = fabs(x[HSB_PCB_E] - wsum / csum);
    x[HSB_PCB_E] = wsum / csum;
    /* PCB inner north/south */
    csum = nc / Lp.edgeNS;
    csum += 1.0 / (pk->r_amb_sec_c_per_y) + 1.0 / pk->r_pcb_c_per_y + 1.0 / (pk->r_pcb2_y + pk->r_pcb);
    wsum = es[8];
    wsum /= Lp.edgeNS;
    wsum += amb / (pk->r_amb_sec_c_per_y) + x[HSB_SOLDER_N] / pk->r_pcb_c_per_y +
            x[HSB_PCB_N] / (pk->r_pcb2_y + pk->r_pcb);
    delta[HSB_PCB_C_N] = fabs(x[HSB_PCB_C_N] - wsum / csum);
    x[HSB_PCB_C_N] = wsum / csum;
    wsum = es[9];
    wsum /= Lp.edgeNS;
    wsum += amb / (pk->r_amb_sec_c_per_y) + x[HSB_SOLDER_S] / pk->r_pcb_c_per_y +
            x[HSB_PCB_S] / (pk->r_pcb2_y + pk->r_pcb);
    delta[HSB_PCB_C_S] = fabs(x[HSB_PCB_C_S] - wsum / csum);
    x[HSB_PCB_C_S] = wsum / csum;
    /* PCB inner west/east */
    csum = nr / Lp.edgeEW;
    csum += 1.0 / (pk->r_amb_sec_c_per_x) + 1.0 / pk->r_pcb_c_per_x + 1.0 / (pk->r_pcb2_x + pk->r_pcb);
    wsum = es[10];
    wsum /= Lp.edgeEW;
    wsum += amb / (pk->r_amb_sec_c_per_x) + x[HSB_SOLDER_W] / pk->r_pcb_c_per_x +
            x[HSB_PCB_W] / (pk->r_pcb2_x + pk->r_pcb);
    delta[HSB_PCB_C_W] = fabs(x[HSB_PCB_C_W] - wsum / csum);
    x[HSB_PCB_C_W] = wsum / csum;
    wsum = es[11];
    wsum /= Lp.edgeEW;
    wsum += amb / (pk->r_amb_sec_c_per_x) + x[HSB_SOLDER_E] / pk->r_pcb_c_per_x +
            x[HSB_PCB_E] / (pk->r_pcb2_x + pk->r_pcb);
    delta[HSB_PCB_C_E] = fabs(x[HSB_PCB_C_E] - wsum / csum);
    x[HSB_PCB_C_E] = wsum / csum;
    /* solder north/south */
    csum = nc / Lq.edgeNS;
    csum += 1.0 / pk->r_solder_per_y + 1.0 / pk->r_pcb_c_per_y;
    wsum = es[12];
    wsum /= Lq.edgeNS;
    wsum += x[HSB_PCB_C_N] / pk->r_pcb_c_per_y + x[HSB_SUB_N] / pk->r_solder_per_y;
    delta[HSB_SOLDER_N] = fabs(x[HSB_SOLDER_N] - wsum / csum);
    x[HSB_SOLDER_N] = wsum / csum;
    wsum = es[13];
    wsum /= Lq.edgeNS;
    wsum += x[HSB_PCB_C_S] / pk->r_pcb_c_per_y + x[HSB_SUB_S] / pk->r_solder_per_y;
    delta[HSB_SOLDER_S] = fabs(x[HSB_SOLDER_S] - wsum / csum);
    x[HSB_SOLDER_S] = wsum / csum;
    /* solder west/east */
    csum = nr / Lq.edgeEW;
    csum += 1.0 / pk->r_solder_per_x + 1.0 / pk->r_pcb_c_per_x;
    wsum = es[14];
    wsum /= Lq.edgeEW;
    wsum += x[HSB_PCB_C_W] / pk->r_pcb_c_per_x + x[HSB_SUB_W] / pk->r_solder_per_x;
    delta[HSB_SOLDER_W] = fabs(x[HSB_SOLDER_W] - wsum / csum);
    x[HSB_SOLDER_W] = wsum / csum;
    wsum = es[15];
    wsum /= Lq.edgeEW;
    wsum += x[HSB_PCB_C_E] / pk->r_pcb_c_per_x + x[HSB_SUB_E] / pk->r_solder_per_x;
    delta[HSB_SOLDER_E] = fabs(x[HSB_SOLDER_E] - wsum / csum);
    x[HSB_SOLDER_E] = wsum / csum;
    /* substrate north/south */
    csum = nc / Lb.edgeNS;
    csum += 1.0 / pk->r_solder_per_y;
    wsum = es[16];
    wsum /= Lb.edgeNS;
    wsum += x[HSB_SOLDER_N] / pk->r_solder_per_y;
    delta[HSB_SUB_N] = fabs(x[HSB_SUB_N] - wsum / csum);
    x[HSB_SUB_N] = wsum / csum;
    wsum = es[17];
    wsum /= Lb.edgeNS;
    wsum += x[HSB_SOLDER_S] / pk->r_solder_per_y;
    delta[HSB_SUB_S] = fabs(x[HSB_SUB_S] - wsum / csum);
    x[HSB_SUB_S] = wsum / csum;
    /* substrate west/east */
    csum = nr / Lb.edgeEW;
    csum += 1.0 / pk->r_solder_per_x;
    wsum = es[18];
    wsum /= Lb.edgeEW;
    wsum += x[HSB_SOLDER_W] / pk->r_solder_per_x;
    delta[HSB_SUB_W] = fabs(x[HSB_SUB_W] - wsum / csum);
    x[HSB_SUB_W] = wsum / csum;
    wsum = es[19];
    wsum /= Lb.edgeEW;
    wsum += x[HSB_SOLDER_E] / pk->r_solder_per_x;
    delta[HSB_SUB_E] = fabs(x[HSB_SUB_E] - wsum / csum);
    x[HSB_SUB_E] = wsum / csum;
  }
  for (int k = 0; k < A.nx; k++)
    if (delta[k] > mx) mx = delta[k];
  return mx;
}

// Up to max_sweeps sweeps (grid then package) at one level; stops after the
// first sweep whose max change is below 1e-6 (eq(delta, 0), util.c:17-20).
// status[0] = converged, status[1] = sweeps done, dout[0] = last delta.
template <bool FIELD, bool SMEM>
__global__ void __launch_bounds__(GS_THREADS)
gs_sweeps(StencilArgs A, double *__restrict__ vg, const double *__restrict__ p, int max_sweeps,
          int *status, double *dout, int spidx, int hsidx, int subidx, int solderidx, int pcbidx) {
  extern __shared__ double sv[];
  __shared__ double red[GS_THREADS / 32];
  __shared__ double es[20];
  __shared__ int done;
  const long long vlen = A.ncell + A.nx;
  double *v = SMEM ? sv : vg;
  if (SMEM) {
    for (long long k = threadIdx.x; k < vlen; k += blockDim.x) sv[k] = vg[k];
    __syncthreads();
  }
  const int nl = A.nl, nr = A.nr, nc = A.nc;
  const int K = nl + nr + nc - 2;  // hyperplanes 0..K-1
  int sweeps = 0;
  double delta = 0.0;
  if (threadIdx.x == 0) done = 0;
  __syncthreads();
  while (sweeps < max_sweeps && !done) {
    double lmax = 0.0;
    for (int k = 0; k < K; k++) {
      // cells (n, i, j = k-n-i) of hyperplane k, flattened over (n, i)
      int f = threadIdx.x;
      for (int n = 0; n < nl && n <= k; n++) {
        const int ilo = max(0, k - n - (nc - 1)), ihi = min(nr - 1, k - n);
        const int cnt = ihi - ilo + 1;
        if (cnt <= 0) continue;
        while (f < cnt) {
          const int i = ilo + f, j = k - n - i;
          const long long c = ((long long)n * nr + i) * nc + j;
          const double d = gs_cell<FIELD>(A, v, p, n, i, j, c);
          if (d > lmax) lmax = d;
          f += blockDim.x;
        }
        f -= cnt;
      }
      __syncthreads();
    }
    // edge sums of the updated grid, then the package nodes in order
    const int ne = A.secondary ? 20 : 8;
    if (threadIdx.x < ne) {
      int layer, which, node;
      edge_desc(threadIdx.x, spidx, hsidx, subidx, solderidx, pcbidx, &layer, &which, &node);
      double s = 0.0;
      const long long base = (long long)layer * A.plane;
      if (which < 2) {
        const long long r = base + (which == 0 ? 0 : (long long)(nr - 1) * nc);
        for (int j = 0; j < nc; j++) s += v[r + j];
      } else {
        const long long cc = base + (which == 2 ? 0 : nc - 1);
        for (int i = 0; i < nr; i++) s += v[cc + (long long)i * nc];
      }
      es[threadIdx.x] = s;
    }
    for (int o = 16; o > 0; o >>= 1) lmax = fmax(lmax, __shfl_down_sync(0xffffffffu, lmax, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = lmax;
    __syncthreads();
    if (threadIdx.x == 0) {
      double gmax = red[0];
      for (int w = 1; w < (int)(blockDim.x >> 5); w++) gmax = fmax(gmax, red[w]);
      // "return MAX(max, single_iteration_steady_pack(...))" (:2607): the
      // reference's MAX macro evaluates the package update twice when the
      // grid's change is not the larger one; the grid and so the edge sums
      // are unchanged between the two evaluations
      const double pmax = gs_pack(A, v, es, nr, nc, spidx, hsidx, subidx, solderidx, pcbidx);
      delta = gmax > pmax ? gmax
                          : gs_pack(A, v, es, nr, nc, spidx, hsidx, subidx, solderidx, pcbidx);
      red[0] = delta;
      if (fabs(delta - 0) < GS_DELTA) done = 1;
    }
    sweeps++;
    __syncthreads();
  }
  if (SMEM) {
    for (long long k = threadIdx.x; k < vlen; k += blockDim.x) vg[k] = sv[k];
  }
  if (threadIdx.x == 0) {
    status[0] = done;
    status[1] = sweeps;
    dout[0] = red[0];
  }
}

// restriction: coarse p = sum of the 4 fine cells (temperature_grid.c:2616-2638)
__global__ void mg_restrict(const double *__restrict__ src, double *__restrict__ dst, int nl,
                            int cnr, int cnc, int nx) {
  const long long cpl = (long long)cnr * cnc, ncell = cpl * nl;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int fnc = 2 * cnc;
  const long long fpl = 4 * cpl;
  if (t < ncell) {
    const int n = (int)(t / cpl);
    const long long r = t - n * cpl;
    const int i = (int)(r / cnc), j = (int)(r - (long long)i * cnc);
    const double *s = src + n * fpl;
    dst[t] = (s[(2 * i) * fnc + 2 * j] + s[(2 * i + 1) * fnc + 2 * j] +
              s[(2 * i) * fnc + 2 * j + 1] + s[(2 * i + 1) * fnc + 2 * j + 1]);
  } else if (t < ncell + nx) {
    dst[t] = src[fpl * nl + (t - ncell)];
  }
}

// prolongation (temperature_grid.c:2646-2715): bilinear 9/16-3/16-1/16 in the
// interior, nearest coarse value on the fine boundary rows and columns
__global__ void mg_prolong(const double *__restrict__ s, double *__restrict__ d, int nl, int nr,
                           int nc, int nx) {
  // one thread per fine cell; nr, nc are the coarse sizes
  const int fnr = 2 * nr, fnc = 2 * nc;
  const long long fpl = (long long)fnr * fnc, cpl = (long long)nr * nc;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < fpl * nl) {
    const int n = (int)(t / fpl);
    const long long r = t - n * fpl;
    const int fi = (int)(r / fnc), fj = (int)(r - (long long)fi * fnc);
    const double *S = s + n * cpl;
    double out;
    if (fi == 0 || fi == fnr - 1 || fj == 0 || fj == fnc - 1) {
      // boundary: rows take s[i][j] of the covering coarse cell
      out = S[(fi / 2) * nc + fj / 2];
    } else {
      // interior fine cell (fi, fj) lies in the square of coarse (i, j)-(i+1, j+1)
      const int i = (fi - 1) / 2, j = (fj - 1) / 2;
      const double a = S[i * nc + j], b = S[(i + 1) * nc + j];
      const double cc = S[(i + 1) * nc + j + 1], dd = S[i * nc + j + 1];
      const int oi = (fi - 1) & 1, oj = (fj - 1) & 1;
      if (!oi && !oj)
        out = 9.0 / 16.0 * a + 3.0 / 16.0 * b + 1.0 / 16.0 * cc + 3.0 / 16.0 * dd;
      else if (oi && !oj)
        out = 3.0 / 16.0 * a + 9.0 / 16.0 * b + 3.0 / 16.0 * cc + 1.0 / 16.0 * dd;
      else if (oi && oj)
        out = 1.0 / 16.0 * a + 3.0 / 16.0 * b + 9.0 / 16.0 * cc + 3.0 / 16.0 * dd;
      else
        out = 3.0 / 16.0 * a + 1.0 / 16.0 * b + 3.0 / 16.0 * cc + 9.0 / 16.0 * dd;
    }
    d[t] = out;
  } else if (t < fpl * nl + nx) {
    d[t] = s[cpl * nl + (t - fpl * nl)];
  }
}

// set_heuristic_temp (temperature_grid.c:2029-2087): lateral resistances
// ignored, each column conducts its cumulative power straight down
__global__ void heuristic_init(StencilArgs A, const double *__restrict__ p, double *__restrict__ v) {
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < A.plane) {
    double sum = 0.0;
    for (int n = 0; n < A.nl; n++) sum = sum + 1.0 * p[n * A.plane + t];
    const int nl = A.nl;
    v[(nl - 1) * A.plane + t] = A.ambient + sum * A.L[nl - 1].rz;
    sum = sum + -1.0 * p[(nl - 1) * A.plane + t];
    for (int n = nl - 2; n >= 0; n--) {
      v[n * A.plane + t] = v[(n + 1) * A.plane + t] + A.L[n].rz * sum;
      sum = sum + -1.0 * p[n * A.plane + t];
    }
  }
  if (t < A.nx) v[A.ncell + t] = A.ambient;
}

static int gs_level(hsb_dev_model *m, const StencilArgs &A, double *v, const double *p,
                    const hsb_solver_opts *o, hsb_stats *st) {
  const long long vlen = A.ncell + A.nx;
  const size_t smem = sizeof(double) * (size_t)vlen;
  const bool use_smem = smem <= 200 * 1024;
  const int chunk = 4096;                 // sweeps per launch
  const long long cap = (o && o->max_iters > 0) ? o->max_iters : 20000000LL;
  long long total = 0;
  for (;;) {
    const int ms = (int)((cap - total) < chunk ? (cap - total) : chunk);
    if (A.field) {
      if (use_smem) {
        raise_smem_limit((const void *)gs_sweeps<true, true>, smem);
        gs_sweeps<true, true><<<1, GS_THREADS, smem, m->stream>>>(A, v, p, ms, m->gs_status, m->gs_delta,
            m->spidx, m->hsidx, m->subidx, m->solderidx, m->pcbidx);
      } else {
        gs_sweeps<true, false><<<1, GS_THREADS, 0, m->stream>>>(A, v, p, ms, m->gs_status, m->gs_delta,
            m->spidx, m->hsidx, m->subidx, m->solderidx, m->pcbidx);
      }
    } else {
      if (use_smem) {
        raise_smem_limit((const void *)gs_sweeps<false, true>, smem);
        gs_sweeps<false, true><<<1, GS_THREADS, smem, m->stream>>>(A, v, p, ms, m->gs_status, m->gs_delta,
            m->spidx, m->hsidx, m->subidx, m->solderidx, m->pcbidx);
      } else {
        gs_sweeps<false, false><<<1, GS_THREADS, 0, m->stream>>>(A, v, p, ms, m->gs_status, m->gs_delta,
            m->spidx, m->hsidx, m->subidx, m->solderidx, m->pcbidx);
      }
    }
    HSB_CUDA(cudaGetLastError());
    HSB_CUDA(cudaMemcpyAsync(m->h_gs, m->gs_status, 2 * sizeof(int), cudaMemcpyDeviceToHost, m->stream));
    HSB_CUDA(cudaMemcpyAsync(m->h_gsd, m->gs_delta, sizeof(double), cudaMemcpyDeviceToHost, m->stream));
    HSB_CUDA(cudaStreamSynchronize(m->stream));
    total += m->h_gs[1];
    st->residual = m->h_gsd[0];
    if (m->h_gs[0]) break;
    if (total >= cap) {
      st->sweeps += total;
      return set_error(HSB_E_NOCONV, "steady Gauss-Seidel did not reach a sweep change below 1e-6 K");
    }
  }
  st->sweeps += total;
  return HSB_OK;
}

int gs_exact_steady(hsb_dev_model *m, const hsb_solver_opts *o, hsb_stats *st) {
  const int T = 256;
  int rc;
  if (m->field) {
    // detailed 3-D: no multigrid (temperature_grid.c:2826-2841)
    const StencilArgs A = make_args(m, m->L0, m->nr, m->nc);
    heuristic_init<<<(unsigned)((A.plane + T - 1) / T), T, 0, m->stream>>>(A, m->pgrid, m->ys);
    HSB_CUDA(cudaGetLastError());
    return gs_level(m, A, m->ys, m->pgrid, o, st);
  }
  const int L = m->n_levels;
  // restrict the power down to the coarsest level
  for (int l = 1; l < L; l++) {
    const LevelBuf &c = m->levels[l];
    const long long n = (long long)c.nr * c.nc * m->nl + m->nx;
    mg_restrict<<<(unsigned)((n + T - 1) / T), T, 0, m->stream>>>(m->levels[l - 1].p, c.p, m->nl,
                                                                 c.nr, c.nc, m->nx);
  }
  HSB_CUDA(cudaGetLastError());
  for (int l = L - 1; l >= 0; l--) {
    const LevelBuf &lv = m->levels[l];
    const StencilArgs A = make_args(m, lv.L, lv.nr, lv.nc);
    if (l == L - 1) {
      heuristic_init<<<(unsigned)((A.plane + T - 1) / T), T, 0, m->stream>>>(A, lv.p, lv.v);
    } else {
      const LevelBuf &c = m->levels[l + 1];
      const long long n = A.ncell + m->nx;
      mg_prolong<<<(unsigned)((n + T - 1) / T), T, 0, m->stream>>>(c.v, lv.v, m->nl, c.nr, c.nc, m->nx);
    }
    HSB_CUDA(cudaGetLastError());
    if ((rc = gs_level(m, A, lv.v, lv.p, o, st))) return rc;
  }
  return HSB_OK;
}

}  // namespace hsb
