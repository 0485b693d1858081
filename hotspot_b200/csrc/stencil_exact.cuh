// stencil_exact.cuh -- FP64 slope of the grid RC network in the reference's
// exact operation order.  Every expression below keeps the association and
// the operand order of the reference C code it restates, and the translation
// units that include this header are compiled with -fmad=false, so each
// result is the same double the reference computes (x86-64 gcc emits no FMA
// without -march flags).
#pragma once
#include "dev_model.cuh"

namespace hsb {

// dT/dt of grid cell c = (n,i,j) (temperature_grid.c:3162-3598):
//   [P + sum_nbr (T_nbr - T)/R + package edges + ambient + advection] / C
// tv(c) returns the temperature of cell c (or of extra node ncell + k).
template <bool FIELD, bool ADV, class TV>
__device__ __forceinline__ double slope_cell_exact(const StencilArgs &A, const TV &tv,
                                                    const double *__restrict__ p,
                                                    int n, int i, int j, long long c) {
  const LayerCoef &Ln = A.L[n];
  const double T = tv(c);
  double psum = 0.0;
  // NP + SP + EP + WP + AP + BP (:3176-3178); absent terms are +0.0 there,
  // and adding +0.0 first or skipping it gives the same double.
  if (i > 0) psum += (tv(c - A.nc) - T) / (FIELD ? A.rN[c] : Ln.rNS);
  if (i < A.nr - 1) psum += (tv(c + A.nc) - T) / (FIELD ? A.rS[c] : Ln.rNS);
  if (j < A.nc - 1) psum += (tv(c + 1) - T) / (FIELD ? A.rE[c] : Ln.rEW);
  if (j > 0) psum += (tv(c - 1) - T) / (FIELD ? A.rW[c] : Ln.rEW);
  if (n > 0) psum += (tv(c - A.plane) - T) / (FIELD ? A.rA[c] : A.L[n - 1].rz);
  if (n < A.nl - 1) psum += (tv(c + A.plane) - T) / (FIELD ? A.rB[c] : Ln.rz);

  if (Ln.kind != LK_PLAIN) {
    const long long X = A.ncell;
    int eN, eS, eE, eW;
    switch (Ln.kind) {
      case LK_SPREADER: eN = HSB_SP_N; eS = HSB_SP_S; eE = HSB_SP_E; eW = HSB_SP_W; break;
      case LK_SINK:
        psum += (A.ambient - T) / Ln.rz;      // :3198
        eN = HSB_SINK_C_N; eS = HSB_SINK_C_S; eE = HSB_SINK_C_E; eW = HSB_SINK_C_W; break;
      case LK_PCB:
        psum += (A.ambient - T) / Ln.ramb;  // :3213-3214
        eN = HSB_PCB_C_N; eS = HSB_PCB_C_S; eE = HSB_PCB_C_E; eW = HSB_PCB_C_W; break;
      case LK_SUB: eN = HSB_SUB_N; eS = HSB_SUB_S; eE = HSB_SUB_E; eW = HSB_SUB_W; break;
      default: eN = HSB_SOLDER_N; eS = HSB_SOLDER_S; eE = HSB_SOLDER_E; eW = HSB_SOLDER_W; break;
    }
    if (i == 0) psum += (tv(X + eN) - T) / Ln.edgeNS;
    if (i == A.nr - 1) psum += (tv(X + eS) - T) / Ln.edgeNS;
    if (j == A.nc - 1) psum += (tv(X + eE) - T) / Ln.edgeEW;
    if (j == 0) psum += (tv(X + eW) - T) / Ln.edgeEW;
  }

  if (ADV && ((A.uchan_mask >> n) & 1ull)) {
    // fluid neighbours N, S, W, E (:3256-3309): coeff * ((T_nbr + T) / 2.0);
    // coefficients are zero for non-fluid pairs and adding 0*x leaves psum.
    if (i > 0) psum += A.aN[c] * ((tv(c - A.nc) + T) / 2.0);
    if (i < A.nr - 1) psum += A.aS[c] * ((tv(c + A.nc) + T) / 2.0);
    if (j > 0) psum += A.aW[c] * ((tv(c - 1) + T) / 2.0);
    if (j < A.nc - 1) psum += A.aE[c] * ((tv(c + 1) + T) / 2.0);
    psum += A.qin[c];            // inlet: (Cv * -sum Q) * T_in   (:3452)
    psum += A.aO[c] * T;         // outlet: (Cv * -sum Q) * T      (:3586)
  }
  return (p[c] + psum) / (FIELD ? A.cap[c] : Ln.cap);
}

// sequential edge sums sum_k (T_edge_k - x) in the reference's loop order
template <class TV>
__device__ __forceinline__ double edge_sum_exact(const StencilArgs &A, const TV &tv,
                                                  int layer, int which, double x) {
  // which: 0 = row 0, 1 = row nr-1, 2 = col 0, 3 = col nc-1
  double s = 0.0;
  const long long base = (long long)layer * A.plane;
  if (which < 2) {
    const long long r = base + (which == 0 ? 0 : (long long)(A.nr - 1) * A.nc);
    for (int j = 0; j < A.nc; j++) s += (tv(r + j) - x);
  } else {
    const long long cc = base + (which == 2 ? 0 : A.nc - 1);
    for (int i = 0; i < A.nr; i++) s += (tv(cc + (long long)i * A.nc) - x);
  }
  return s;
}

// Package-node slopes (slope_fn_pack, temperature_grid.c:2857-3093).
// x: the n_extra node temperatures; es: edge sums in the order
// SINK_C_N,S,W,E, SP_N,S,W,E, [PCB_C_N,S,W,E, SOLDER_N,S,W,E, SUB_N,S,W,E];
// eNS/eEW of the sink/spreader/... layers are the edge resistances.
__device__ __forceinline__ void pack_slope_exact(const StencilArgs &A, const double *x,
                                                 const double *es, double *dv,
                                                 int spidx, int hsidx, int subidx,
                                                 int solderidx, int pcbidx) {
  const package_RC_t *pk = A.pk;
  const double amb = A.ambient;
  const LayerCoef &Ls = A.L[spidx], &Lh = A.L[hsidx];
  double psum;
  /* sink outer north/south */
  psum = (amb - x[HSB_SINK_N]) / (pk->r_hs_per + pk->r_amb_per) +
         (x[HSB_SINK_C_N] - x[HSB_SINK_N]) / (pk->r_hs2_y + pk->r_hs);
  dv[HSB_SINK_N] = psum / (pk->c_hs_per + pk->c_amb_per);
  psum = (amb - x[HSB_SINK_S]) / (pk->r_hs_per + pk->r_amb_per) +
         (x[HSB_SINK_C_S] - x[HSB_SINK_S]) / (pk->r_hs2_y + pk->r_hs);
  dv[HSB_SINK_S] = psum / (pk->c_hs_per + pk->c_amb_per);
  /* sink outer west/east */
  psum = (amb - x[HSB_SINK_W]) / (pk->r_hs_per + pk->r_amb_per) +
         (x[HSB_SINK_C_W] - x[HSB_SINK_W]) / (pk->r_hs2_x + pk->r_hs);
  dv[HSB_SINK_W] = psum / (pk->c_hs_per + pk->c_amb_per);
  psum = (amb - x[HSB_SINK_E]) / (pk->r_hs_per + pk->r_amb_per) +
         (x[HSB_SINK_C_E] - x[HSB_SINK_E]) / (pk->r_hs2_x + pk->r_hs);
  dv[HSB_SINK_E] = psum / (pk->c_hs_per + pk->c_amb_per);
  /* sink inner north/south */
  psum = es[0] / Lh.edgeNS;
  psum += (amb - x[HSB_SINK_C_N]) / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) +
          (x[HSB_SP_N] - x[HSB_SINK_C_N]) / pk->r_sp_per_y +
          (x[HSB_SINK_N] - x[HSB_SINK_C_N]) / (pk->r_hs2_y + pk->r_hs);
  dv[HSB_SINK_C_N] = psum / (pk->c_hs_c_per_y + pk->c_amb_c_per_y);
  psum = es[1] / Lh.edgeNS;
  psum += (amb - x[HSB_SINK_C_S]) / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) +
          (x[HSB_SP_S] - x[HSB_SINK_C_S]) / pk->r_sp_per_y +
          (x[HSB_SINK_S] - x[HSB_SINK_C_S]) / (pk->r_hs2_y + pk->r_hs);
  dv[HSB_SINK_C_S] = psum / (pk->c_hs_c_per_y + pk->c_amb_c_per_y);
  /* sink inner west/east */
  psum = es[2] / Lh.edgeEW;
  psum += (amb - x[HSB_SINK_C_W]) / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) +
          (x[HSB_SP_W] - x[HSB_SINK_C_W]) / pk->r_sp_per_x +
          (x[HSB_SINK_W] - x[HSB_SINK_C_W]) / (pk->r_hs2_x + pk->r_hs);
  dv[HSB_SINK_C_W] = psum / (pk->c_hs_c_per_x + pk->c_amb_c_per_x);
  psum = es[3] / Lh.edgeEW;
  psum += (amb - x[HSB_SINK_C_E]) / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) +
          (x[HSB_SP_E] - x[HSB_SINK_C_E]) / pk->r_sp_per_x +
          (x[HSB_SINK_E] - x[HSB_SINK_C_E]) / (pk->r_hs2_x + pk->r_hs);
  dv[HSB_SINK_C_E] = psum / (pk->c_hs_c_per_x + pk->c_amb_c_per_x);
  /* spreader north/south */
  psum = es[4] / Ls.edgeNS;
  psum += (x[HSB_SINK_C_N] - x[HSB_SP_N]) / pk->r_sp_per_y;
  dv[HSB_SP_N] = psum / pk->c_sp_per_y;
  psum = es[5] / Ls.edgeNS;
  psum += (x[HSB_SINK_C_S] - x[HSB_SP_S]) / pk->r_sp_per_y;
  dv[HSB_SP_S] = psum / pk->c_sp_per_y;
  /* spreader west/east */
  psum = es[6] / Ls.edgeEW;
  psum += (x[HSB_SINK_C_W] - x[HSB_SP_W]) / pk->r_sp_per_x;
  dv[HSB_SP_W] = psum / pk->c_sp_per_x;
  psum = es[7] / Ls.edgeEW;
  psum += (x[HSB_SINK_C_E] - x[HSB_SP_E]) / pk->r_sp_per_x;
  dv[HSB_SP_E] = psum / pk->c_sp_per_x;

  if (A.secondary) {
    const LayerCoef &Lp = A.L[pcbidx], &Lq = A.L[solderidx], &Lb = A.L[subidx];
    /* PCB outer north/south */
    psum = (amb - x[HSB_PCB_N]) / (pk->r_amb_sec_per) +
           (x[HSB_PCB_C_N] - x[HSB_PCB_N]) / (pk->r_pcb2_y + pk->r_pcb);
    dv[HSB_PCB_N] = psum / (pk->c_pcb_per + pk->c_amb_sec_per);
    psum = (amb - x[HSB_PCB_S]) / (pk->r_amb_sec_per) +
           (x[HSB_PCB_C_S] - x[HSB_PCB_S]) / (pk->r_pcb2_y + pk->r_pcb);
    dv[HSB_PCB_S] = psum / (pk->c_pcb_per + pk->c_amb_sec_per);
    /* PCB outer west/east */
    psum = (amb - x[HSB_PCB_W]) / (pk->r_amb_sec_per) +
           (x[HSB_PCB_C_W] - x[HSB_PCB_W]) / (pk->r_pcb2_x + pk->r_pcb);
    dv[HSB_PCB_W] = psum / (pk->c_pcb_per + pk->c_amb_sec_per);
    psum = (amb - x[HSB_PCB_E]) / (pk->r_amb_sec_per) +
           (x[HSB_PCB_C_E] - x[HSB_PCB_E]) / (pk->r_pcb2_x + pk->r_pcb);
    dv[HSB_PCB_E] = psum / (pk->c_pcb_per + pk->c_amb_sec_per);
    /* PCB inner north/south */
    psum = es[8] / Lp.edgeNS;
    psum += (amb - x[HSB_PCB_C_N]) / (pk->r_amb_sec_c_per_y) +
            (x[HSB_SOLDER_N] - x[HSB_PCB_C_N]) / pk->r_pcb_c_per_y +
            (x[HSB_PCB_N] - x[HSB_PCB_C_N]) / (pk->r_pcb2_y + pk->r_pcb);
    dv[HSB_PCB_C_N] = psum / (pk->c_pcb_c_per_y + pk->c_amb_sec_c_per_y);
    psum = es[9] / Lp.edgeNS;
    psum += (amb - x[HSB_PCB_C_S]) / (pk->r_amb_sec_c_per_y) +
            (x[HSB_SOLDER_S] - x[HSB_PCB_C_S]) / pk->r_pcb_c_per_y +
            (x[HSB_PCB_S] - x[HSB_PCB_C_S]) / (pk->r_pcb2_y + pk->r_pcb);
    dv[HSB_PCB_C_S] = psum / (pk->c_pcb_c_per_y + pk->c_amb_sec_c_per_y);
    /* PCB inner west/east */
    psum = es[10] / Lp.edgeEW;
    psum += (amb - x[HSB_PCB_C_W]) / (pk->r_amb_sec_c_per_x) +
            (x[HSB_SOLDER_W] - x[HSB_PCB_C_W]) / pk->r_pcb_c_per_x +
            (x[HSB_PCB_W] - x[HSB_PCB_C_W]) / (pk->r_pcb2_x + pk->r_pcb);
    dv[HSB_PCB_C_W] = psum / (pk->c_pcb_c_per_x + pk->c_amb_sec_c_per_x);
    psum = es[11] / Lp.edgeEW;
    psum += (amb - x[HSB_PCB_C_E]) / (pk->r_amb_sec_c_per_x) +
            (x[HSB_SOLDER_E] - x[HSB_PCB_C_E]) / pk->r_pcb_c_per_x +
            (x[HSB_PCB_E] - x[HSB_PCB_C_E]) / (pk->r_pcb2_x + pk->r_pcb);
    dv[HSB_PCB_C_E] = psum / (pk->c_pcb_c_per_x + pk->c_amb_sec_c_per_x);
    /* solder north/south */
    psum = es[12] / Lq.edgeNS;
    psum += (x[HSB_PCB_C_N] - x[HSB_SOLDER_N]) / pk->r_pcb_c_per_y;
    dv[HSB_SOLDER_N] = psum / pk->c_solder_per_y;
    psum = es[13] / Lq.edgeNS;
    psum += (x[HSB_PCB_C_S] - x[HSB_SOLDER_S]) / pk->r_pcb_c_per_y;
    dv[HSB_SOLDER_S] = psum / pk->c_solder_per_y;
    /* solder west/east */
    psum = es[14] / Lq.edgeEW;
    psum += (x[HSB_PCB_C_W] - x[HSB_SOLDER_W]) / pk->r_pcb_c_per_x;
    dv[HSB_SOLDER_W] = psum / pk->c_solder_per_x;
    psum = es[15] / Lq.edgeEW;
    psum += (x[HSB_PCB_C_E] - x[HSB_SOLDER_E]) / pk->r_pcb_c_per_x;
    dv[HSB_SOLDER_E] = psum / pk->c_solder_per_x;
    /* substrate north/south */
    psum = es[16] / Lb.edgeNS;
    psum += (x[HSB_SOLDER_N] - x[HSB_SUB_N]) / pk->r_solder_per_y;
    dv[HSB_SUB_N] = psum / pk->c_sub_per_y;
    psum = es[17] / Lb.edgeNS;
    psum += (x[HSB_SOLDER_S] - x[HSB_SUB_S]) / pk->r_solder_per_y;
    dv[HSB_SUB_S] = psum / pk->c_sub_per_y;
    /* substrate west/east */
    psum = es[18] / Lb.edgeEW;
    psum += (x[HSB_SOLDER_W] - x[HSB_SUB_W]) / pk->r_solder_per_x;
    dv[HSB_SUB_W] = psum / pk->c_sub_per_x;
    psum = es[19] / Lb.edgeEW;
    psum += (x[HSB_SOLDER_E] - x[HSB_SUB_E]) / pk->r_solder_per_x;
    dv[HSB_SUB_E] = psum / pk->c_sub_per_x;
  }
}

// (layer, edge) of each package edge sum, in pack_slope_exact's es[] order
__device__ __forceinline__ void edge_desc(int e, int spidx, int hsidx, int subidx, int solderidx,
                                          int pcbidx, int *layer, int *which, int *node) {
  // node groups: SINK_C_* (4), SP_* (0), PCB_C_* (20), SOLDER_* (16), SUB_* (12);
  // inside a group the reference numbers W, E, N, S and the sums run N, S, W, E
  const int g = e >> 2;
  const int base = g == 0 ? HSB_SINK_C_W : g == 1 ? HSB_SP_W : g == 2 ? HSB_PCB_C_W
                 : g == 3 ? HSB_SOLDER_W : HSB_SUB_W;
  *which = e & 3;
  *node = base + ((*which + 2) & 3);
  *layer = g == 0 ? hsidx : g == 1 ? spidx : g == 2 ? pcbidx : g == 3 ? solderidx : subidx;
}

}  // namespace hsb
