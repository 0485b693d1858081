/*
 * grid_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in plain C99, of the numerical core of HotSpot's grid
 * model, used as the test oracle of libhotspot_b200 in tests/, smoke() and the
 * CPU-baseline leg of bench.py.  It follows the reference's loops literally:
 * lexicographic (n, i, j) sweeps, the same association of every sum, no FMA
 * (-ffp-contract=off), so that on identical inputs it reproduces the
 * reference's doubles.  Cited per function:
 *
 *   find_res / slope terms   temperature_grid.c:26-136, :3095-3601
 *   slope_fn_pack            temperature_grid.c:2857-3093
 *   rk4_core / rk4           RCutil.c:440-640
 *   compute_temp_grid loop   temperature_grid.c:3676-3692
 *   Gauss-Seidel sweep       temperature_grid.c:2426-2608, :2090-2393
 *   nested multigrid         temperature_grid.c:2616-2797
 *   heuristic start          temperature_grid.c:2029-2087
 *
 * Model set-up (layers, occupancy maps, R/C values, flow rates) is done by
 * oracle/restatement.py and passed in as flat arrays.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "grid_oracle.h"

typedef struct {
  double r_sp1_x, r_sp1_y, r_hs1_x, r_hs1_y, r_hs2_x, r_hs2_y, r_hs;
  double r_sp_per_x, r_sp_per_y, r_hs_c_per_x, r_hs_c_per_y, r_hs_per;
  double c_sp_per_x, c_sp_per_y, c_hs_c_per_x, c_hs_c_per_y, c_hs_per;
  double r_amb_c_per_x, c_amb_c_per_x, r_amb_c_per_y, c_amb_c_per_y;
  double r_amb_per, c_amb_per;
  double r_sub1_x, r_sub1_y, r_solder1_x, r_solder1_y;
  double r_pcb1_x, r_pcb1_y, r_pcb2_x, r_pcb2_y, r_pcb;
  double r_sub_per_x, r_sub_per_y, r_solder_per_x, r_solder_per_y;
  double r_pcb_c_per_x, r_pcb_c_per_y, r_pcb_per;
  double c_sub_per_x, c_sub_per_y, c_solder_per_x, c_solder_per_y;
  double c_pcb_c_per_x, c_pcb_c_per_y, c_pcb_per;
  double r_amb_sec_c_per_x, c_amb_sec_c_per_x, r_amb_sec_c_per_y, c_amb_sec_c_per_y;
  double r_amb_sec_per, c_amb_sec_per;
} pk_t;

enum { SP_W, SP_E, SP_N, SP_S, SINK_C_W, SINK_C_E, SINK_C_N, SINK_C_S, SINK_W, SINK_E, SINK_N, SINK_S,
       SUB_W, SUB_E, SUB_N, SUB_S, SOLDER_W, SOLDER_E, SOLDER_N, SOLDER_S,
       PCB_C_W, PCB_C_E, PCB_C_N, PCB_C_S, PCB_W, PCB_E, PCB_N, PCB_S };

/* one level of the (multigrid) hierarchy: grid size and the layer values as
 * the reference has them at that level (rz /= 4 and c *= 4 per level) */
typedef struct {
  int nr, nc;
  double rz[64], c[64];
} level_t;

#define V3(v, n, i, j) (v)[((size_t)(n) * L->nr + (i)) * L->nc + (j)]

/* find_res(model, neighbour..., cell...) for the uniform model */
static double res_lat_ns(const orc_model *m, int n) { return (m->rx[n] / 2.0) + (m->rx[n] / 2.0); }
static double res_lat_ew(const orc_model *m, int n) { return (m->ry[n] / 2.0) + (m->ry[n] / 2.0); }

static int is_sec(const orc_model *m) { return m->nx > 12; }

/* ---------------------------------------------------------------------- */
/* slope                                                                   */
/* ---------------------------------------------------------------------- */
static void slope_pack(const orc_model *m, const level_t *L, const double *v, double *dv)
{
  const pk_t *pk = (const pk_t *)m->pack;
  const int nl = m->nl, nr = L->nr, nc = L->nc, hs = m->hsidx, sp = m->spidx;
  const double amb = m->ambient;
  const double *x = v + (size_t)nl * nr * nc;
  double *d = dv + (size_t)nl * nr * nc;
  double psum;
  int i, j;
  psum = (amb - x[SINK_N]) / (pk->r_hs_per + pk->r_amb_per) + (x[SINK_C_N] - x[SINK_N]) / (pk->r_hs2_y + pk->r_hs);
  d[SINK_N] = psum / (pk->c_hs_per + pk->c_amb_per);
  psum = (amb - x[SINK_S]) / (pk->r_hs_per + pk->r_amb_per) + (x[SINK_C_S] - x[SINK_S]) / (pk->r_hs2_y + pk->r_hs);
  d[SINK_S] = psum / (pk->c_hs_per + pk->c_amb_per);
  psum = (amb - x[SINK_W]) / (pk->r_hs_per + pk->r_amb_per) + (x[SINK_C_W] - x[SINK_W]) / (pk->r_hs2_x + pk->r_hs);
  d[SINK_W] = psum / (pk->c_hs_per + pk->c_amb_per);
  psum = (amb - x[SINK_E]) / (pk->r_hs_per + pk->r_amb_per) + (x[SINK_C_E] - x[SINK_E]) / (pk->r_hs2_x + pk->r_hs);
  d[SINK_E] = psum / (pk->c_hs_per + pk->c_amb_per);

  psum = 0.0;
  for (j = 0; j < nc; j++) psum += (V3(v, hs, 0, j) - x[SINK_C_N]);
  psum /= (m->ry[hs] / 2.0 + nc * pk->r_hs1_y);
  psum += (amb - x[SINK_C_N]) / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) + (x[SP_N] - x[SINK_C_N]) / pk->r_sp_per_y +
          (x[SINK_N] - x[SINK_C_N]) / (pk->r_hs2_y + pk->r_hs);
  d[SINK_C_N] = psum / (pk->c_hs_c_per_y + pk->c_amb_c_per_y);
  psum = 0.0;
  for (j = 0; j < nc; j++) psum += (V3(v, hs, nr - 1, j) - x[SINK_C_S]);
  psum /= (m->ry[hs] / 2.0 + nc * pk->r_hs1_y);
  psum += (amb - x[SINK_C_S]) / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) + (x[SP_S] - x[SINK_C_S]) / pk->r_sp_per_y +
          (x[SINK_S] - x[SINK_C_S]) / (pk->r_hs2_y + pk->r_hs);
  d[SINK_C_S] = psum / (pk->c_hs_c_per_y + pk->c_amb_c_per_y);
  psum = 0.0;
  for (i = 0; i < nr; i++) psum += (V3(v, hs, i, 0) - x[SINK_C_W]);
  psum /= (m->rx[hs] / 2.0 + nr * pk->r_hs1_x);
  psum += (amb - x[SINK_C_W]) / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) + (x[SP_W] - x[SINK_C_W]) / pk->r_sp_per_x +
          (x[SINK_W] - x[SINK_C_W]) / (pk->r_hs2_x + pk->r_hs);
  d[SINK_C_W] = psum / (pk->c_hs_c_per_x + pk->c_amb_c_per_x);
  psum = 0.0;
  for (i = 0; i < nr; i++) psum += (V3(v, hs, i, nc - 1) - x[SINK_C_E]);
  psum /= (m->rx[hs] / 2.0 + nr * pk->r_hs1_x);
  psum += (amb - x[SINK_C_E]) / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) + (x[SP_E] - x[SINK_C_E]) / pk->r_sp_per_x +
          (x[SINK_E] - x[SINK_C_E]) / (pk->r_hs2_x + pk->r_hs);
  d[SINK_C_E] = psum / (pk->c_hs_c_per_x + pk->c_amb_c_per_x);

  psum = 0.0;
  for (j = 0; j < nc; j++) psum += (V3(v, sp, 0, j) - x[SP_N]);
  psum /= (m->ry[sp] / 2.0 + nc * pk->r_sp1_y);
  psum += (x[SINK_C_N] - x[SP_N]) / pk->r_sp_per_y;
  d[SP_N] = psum / pk->c_sp_per_y;
  psum = 0.0;
  for (j = 0; j < nc; j++) psum += (V3(v, sp, nr - 1, j) - x[SP_S]);
  psum /= (m->ry[sp] / 2.0 + nc * pk->r_sp1_y);
  psum += (x[SINK_C_S] - x[SP_S]) / pk->r_sp_per_y;
  d[SP_S] = psum / pk->c_sp_per_y;
  psum = 0.0;
  for (i = 0; i < nr; i++) psum += (V3(v, sp, i, 0) - x[SP_W]);
  psum /= (m->rx[sp] / 2.0 + nr * pk->r_sp1_x);
  psum += (x[SINK_C_W] - x[SP_W]) / pk->r_sp_per_x;
  d[SP_W] = psum / pk->c_sp_per_x;
  psum = 0.0;
  for (i = 0; i < nr; i++) psum += (V3(v, sp, i, nc - 1) - x[SP_E]);
  psum /= (m->rx[sp] / 2.0 + nr * pk->r_sp1_x);
  psum += (x[SINK_C_E] - x[SP_E]) / pk->r_sp_per_x;
  d[SP_E] = psum / pk->c_sp_per_x;

  if (is_sec(m)) {
    const int pcb = m->pcbidx, sol = m->solderidx, sub = m->subidx;
    psum = (amb - x[PCB_N]) / (pk->r_amb_sec_per) + (x[PCB_C_N] - x[PCB_N]) / (pk->r_pcb2_y + pk->r_pcb);
    d[PCB_N] = psum / (pk->c_pcb_per + pk->c_amb_sec_per);
    psum = (amb - x[PCB_S]) / (pk->r_amb_sec_per) + (x[PCB_C_S] - x[PCB_S]) / (pk->r_pcb2_y + pk->r_pcb);
    d[PCB_S] = psum / (pk->c_pcb_per + pk->c_amb_sec_per);
    psum = (amb - x[PCB_W]) / (pk->r_amb_sec_per) + (x[PCB_C_W] - x[PCB_W]) / (pk->r_pcb2_x + pk->r_pcb);
    d[PCB_W] = psum / (pk->c_pcb_per + pk->c_amb_sec_per);
    psum = (amb - x[PCB_E]) / (pk->r_amb_sec_per) + (x[PCB_C_E] - x[PCB_E]) / (pk->r_pcb2_x + pk->r_pcb);
    d[PCB_E] = psum / (pk->c_pcb_per + pk->c_amb_sec_per);
    psum = 0.0;
    for (j = 0; j < nc; j++) psum += (V3(v, pcb, 0, j) - x[PCB_C_N]);
    psum /= (m->ry[pcb] / 2.0 + nc * pk->r_pcb1_y);
    psum += (amb - x[PCB_C_N]) / (pk->r_amb_sec_c_per_y) + (x[SOLDER_N] - x[PCB_C_N]) / pk->r_pcb_c_per_y +
            (x[PCB_N] - x[PCB_C_N]) / (pk->r_pcb2_y + pk->r_pcb);
    d[PCB_C_N] = psum / (pk->c_pcb_c_per_y + pk->c_amb_sec_c_per_y);
    psum = 0.0;
    for (j = 0; j < nc; j++) psum += (V3(v, pcb, nr - 1, j) - x[PCB_C_S]);
    psum /= (m->ry[pcb] / 2.0 + nc * pk->r_pcb1_y);
    psum += (amb - x[PCB_C_S]) / (pk->r_amb_sec_c_per_y) + (x[SOLDER_S] - x[PCB_C_S]) / pk->r_pcb_c_per_y +
            (x[PCB_S] - x[PCB_C_S]) / (pk->r_pcb2_y + pk->r_pcb);
    d[PCB_C_S] = psum / (pk->c_pcb_c_per_y + pk->c_amb_sec_c_per_y);
    psum = 0.0;
    for (i = 0; i < nr; i++) psum += (V3(v, pcb, i, 0) - x[PCB_C_W]);
    psum /= (m->rx[pcb] / 2.0 + nr * pk->r_pcb1_x);
    psum += (amb - x[PCB_C_W]) / (pk->r_amb_sec_c_per_x) + (x[SOLDER_W] - x[PCB_C_W]) / pk->r_pcb_c_per_x +
            (x[PCB_W] - x[PCB_C_W]) / (pk->r_pcb2_x + pk->r_pcb);
    d[PCB_C_W] = psum / (pk->c_pcb_c_per_x + pk->c_amb_sec_c_per_x);
    psum = 0.0;
    for (i = 0; i < nr; i++) psum += (V3(v, pcb, i, nc - 1) - x[PCB_C_E]);
    psum /= (m->rx[pcb] / 2.0 + nr * pk->r_pcb1_x);
    psum += (amb - x[PCB_C_E]) / (pk->r_amb_sec_c_per_x) + (x[SOLDER_E] - x[PCB_C_E]) / pk->r_pcb_c_per_x +
            (x[PCB_E] - x[PCB_C_E]) / (pk->r_pcb2_x + pk->r_pcb);
    d[PCB_C_E] = psum / (pk->c_pcb_c_per_x + pk->c_amb_sec_c_per_x);
    psum = 0.0;
    for (j = 0; j < nc; j++) psum += (V3(v, sol, 0, j) - x[SOLDER_N]);
    psum /= (m->ry[sol] / 2.0 + nc * pk->r_solder1_y);
    psum += (x[PCB_C_N] - x[SOLDER_N]) / pk->r_pcb_c_per_y;
    d[SOLDER_N] = psum / pk->c_solder_per_y;
    psum = 0.0;
    for (j = 0; j < nc; j++) psum += (V3(v, sol, nr - 1, j) - x[SOLDER_S]);
    psum /= (m->ry[sol] / 2.0 + nc * pk->r_solder1_y);
    psum += (x[PCB_C_S] - x[SOLDER_S]) / pk->r_pcb_c_per_y;
    d[SOLDER_S] = psum / pk->c_solder_per_y;
    psum = 0.0;
    for (i = 0; i < nr; i++) psum += (V3(v, sol, i, 0) - x[SOLDER_W]);
    psum /= (m->rx[sol] / 2.0 + nr * pk->r_solder1_x);
    psum += (x[PCB_C_W] - x[SOLDER_W]) / pk->r_pcb_c_per_x;
    d[SOLDER_W] = psum / pk->c_solder_per_x;
    psum = 0.0;
    for (i = 0; i < nr; i++) psum += (V3(v, sol, i, nc - 1) - x[SOLDER_E]);
    psum /= (m->rx[sol] / 2.0 + nr * pk->r_solder1_x);
    psum += (x[PCB_C_E] - x[SOLDER_E]) / pk->r_pcb_c_per_x;
    d[SOLDER_E] = psum / pk->c_solder_per_x;
    psum = 0.0;
    for (j = 0; j < nc; j++) psum += (V3(v, sub, 0, j) - x[SUB_N]);
    psum /= (m->ry[sub] / 2.0 + nc * pk->r_sub1_y);
    psum += (x[SOLDER_N] - x[SUB_N]) / pk->r_solder_per_y;
    d[SUB_N] = psum / pk->c_sub_per_y;
    psum = 0.0;
    for (j = 0; j < nc; j++) psum += (V3(v, sub, nr - 1, j) - x[SUB_S]);
    psum /= (m->ry[sub] / 2.0 + nc * pk->r_sub1_y);
    psum += (x[SOLDER_S] - x[SUB_S]) / pk->r_solder_per_y;
    d[SUB_S] = psum / pk->c_sub_per_y;
    psum = 0.0;
    for (i = 0; i < nr; i++) psum += (V3(v, sub, i, 0) - x[SUB_W]);
    psum /= (m->rx[sub] / 2.0 + nr * pk->r_sub1_x);
    psum += (x[SOLDER_W] - x[SUB_W]) / pk->r_solder_per_x;
    d[SUB_W] = psum / pk->c_sub_per_x;
    psum = 0.0;
    for (i = 0; i < nr; i++) psum += (V3(v, sub, i, nc - 1) - x[SUB_E]);
    psum /= (m->rx[sub] / 2.0 + nr * pk->r_sub1_x);
    psum += (x[SOLDER_E] - x[SUB_E]) / pk->r_solder_per_x;
    d[SUB_E] = psum / pk->c_sub_per_x;
  }
}

static void slope_level(const orc_model *m, const level_t *L, const double *v, const double *p, double *dv)
{
  const pk_t *pk = (const pk_t *)m->pack;
  const int nl = m->nl, nr = L->nr, nc = L->nc;
  const double *x = v + (size_t)nl * nr * nc;
  const double cw = m->width / nc, ch = m->height / nr;
  int n, i, j;
  for (n = 0; n < nl; n++)
    for (i = 0; i < nr; i++)
      for (j = 0; j < nc; j++) {
        const size_t c = ((size_t)n * nr + i) * nc + j;
        const double T = v[c];
        double NP = 0.0, SP = 0.0, EP = 0.0, WP = 0.0, AP = 0.0, BP = 0.0, psum;
        if (m->field) {
          if (i > 0) NP = (v[c - nc] - T) / m->rN[c];
          if (i < nr - 1) SP = (v[c + nc] - T) / m->rS[c];
          if (j < nc - 1) EP = (v[c + 1] - T) / m->rE[c];
          if (j > 0) WP = (v[c - 1] - T) / m->rW[c];
          if (n > 0) AP = (v[c - (size_t)nr * nc] - T) / m->rA[c];
          if (n < nl - 1) BP = (v[c + (size_t)nr * nc] - T) / m->rB[c];
        } else {
          if (i > 0) NP = (v[c - nc] - T) / res_lat_ns(m, n);
          if (i < nr - 1) SP = (v[c + nc] - T) / res_lat_ns(m, n);
          if (j < nc - 1) EP = (v[c + 1] - T) / res_lat_ew(m, n);
          if (j > 0) WP = (v[c - 1] - T) / res_lat_ew(m, n);
          if (n > 0) AP = (v[c - (size_t)nr * nc] - T) / L->rz[n - 1];
          if (n < nl - 1) BP = (v[c + (size_t)nr * nc] - T) / L->rz[n];
        }
        psum = NP + SP + EP + WP + AP + BP;
        if (n == m->spidx) {
          if (i == 0) psum += (x[SP_N] - T) / (m->ry[n] / 2.0 + nc * pk->r_sp1_y);
          if (i == nr - 1) psum += (x[SP_S] - T) / (m->ry[n] / 2.0 + nc * pk->r_sp1_y);
          if (j == nc - 1) psum += (x[SP_E] - T) / (m->rx[n] / 2.0 + nr * pk->r_sp1_x);
          if (j == 0) psum += (x[SP_W] - T) / (m->rx[n] / 2.0 + nr * pk->r_sp1_x);
        } else if (n == m->hsidx) {
          psum += (m->ambient - T) / L->rz[n];
          if (i == 0) psum += (x[SINK_C_N] - T) / (m->ry[n] / 2.0 + nc * pk->r_hs1_y);
          if (i == nr - 1) psum += (x[SINK_C_S] - T) / (m->ry[n] / 2.0 + nc * pk->r_hs1_y);
          if (j == nc - 1) psum += (x[SINK_C_E] - T) / (m->rx[n] / 2.0 + nr * pk->r_hs1_x);
          if (j == 0) psum += (x[SINK_C_W] - T) / (m->rx[n] / 2.0 + nr * pk->r_hs1_x);
        } else if (n == m->pcbidx && is_sec(m)) {
          psum += (m->ambient - T) / (m->pcb_amb_num / (cw * ch));
          if (i == 0) psum += (x[PCB_C_N] - T) / (m->ry[n] / 2.0 + nc * pk->r_pcb1_y);
          if (i == nr - 1) psum += (x[PCB_C_S] - T) / (m->ry[n] / 2.0 + nc * pk->r_pcb1_y);
          if (j == nc - 1) psum += (x[PCB_C_E] - T) / (m->rx[n] / 2.0 + nr * pk->r_pcb1_x);
          if (j == 0) psum += (x[PCB_C_W] - T) / (m->rx[n] / 2.0 + nr * pk->r_pcb1_x);
        } else if (n == m->subidx && is_sec(m)) {
          if (i == 0) psum += (x[SUB_N] - T) / (m->ry[n] / 2.0 + nc * pk->r_sub1_y);
          if (i == nr - 1) psum += (x[SUB_S] - T) / (m->ry[n] / 2.0 + nc * pk->r_sub1_y);
          if (j == nc - 1) psum += (x[SUB_E] - T) / (m->rx[n] / 2.0 + nr * pk->r_sub1_x);
          if (j == 0) psum += (x[SUB_W] - T) / (m->rx[n] / 2.0 + nr * pk->r_sub1_x);
        } else if (n == m->solderidx && is_sec(m)) {
          if (i == 0) psum += (x[SOLDER_N] - T) / (m->ry[n] / 2.0 + nc * pk->r_solder1_y);
          if (i == nr - 1) psum += (x[SOLDER_S] - T) / (m->ry[n] / 2.0 + nc * pk->r_solder1_y);
          if (j == nc - 1) psum += (x[SOLDER_E] - T) / (m->rx[n] / 2.0 + nr * pk->r_solder1_x);
          if (j == 0) psum += (x[SOLDER_W] - T) / (m->rx[n] / 2.0 + nr * pk->r_solder1_x);
        }
        if (m->adv) {
          if (i > 0) psum += m->aN[c] * ((v[c - nc] + T) / 2.0);
          if (i < nr - 1) psum += m->aS[c] * ((v[c + nc] + T) / 2.0);
          if (j > 0) psum += m->aW[c] * ((v[c - 1] + T) / 2.0);
          if (j < nc - 1) psum += m->aE[c] * ((v[c + 1] + T) / 2.0);
          psum += m->qin[c];
          psum += m->aO[c] * T;
        }
        dv[c] = (p[c] + psum) / (m->field ? m->cap[c] : L->c[n]);
      }
  slope_pack(m, L, v, dv);
}

static void finest(const orc_model *m, level_t *L)
{
  int n;
  L->nr = m->nr;
  L->nc = m->nc;
  for (n = 0; n < m->nl; n++) {
    L->rz[n] = m->rz[n];
    L->c[n] = m->c ? m->c[n] : 0.0;
  }
}

void orc_slope(const orc_model *m, const double *y, const double *p, double *dy)
{
  level_t L;
  finest(m, &L);
  slope_level(m, &L, y, p, dy);
}

/* ---------------------------------------------------------------------- */
/* RK4 with step doubling                                                  */
/* ---------------------------------------------------------------------- */
static void rk4_core(const orc_model *m, const double *y, const double *k1, const double *p, size_t n, double h,
                     double *yout, double *k2, double *k3, double *k4, double *t)
{
  size_t i;
  for (i = 0; i < n; i++) t[i] = y[i] + h / 2.0 * k1[i];
  orc_slope(m, t, p, k2);
  for (i = 0; i < n; i++) t[i] = y[i] + h / 2.0 * k2[i];
  orc_slope(m, t, p, k3);
  for (i = 0; i < n; i++) t[i] = y[i] + h * k3[i];
  orc_slope(m, t, p, k4);
  for (i = 0; i < n; i++) yout[i] = y[i] + h * (k1[i] + 2 * k2[i] + 2 * k3[i] + k4[i]) / 6.0;
}

/* RK4 attempts (accepted and rejected) since the library was loaded */
long long orc_attempts = 0;

double orc_rk4(const orc_model *m, double *y, const double *p, double *h)
{
  const size_t n = (size_t)m->nl * m->nr * m->nc + m->nx;
  double *w = malloc(sizeof(double) * n * 8);
  double *k1 = w, *t1 = w + n, *t2 = w + 2 * n, *ytemp = w + 3 * n;
  double *k2 = w + 4 * n, *k3 = w + 5 * n, *k4 = w + 6 * n, *t = w + 7 * n;
  double max, new_h = *h;
  size_t i;
  orc_slope(m, y, p, k1);
  do {
    *h = new_h;
    orc_attempts++;
    rk4_core(m, y, k1, p, n, *h, ytemp, k2, k3, k4, t);
    rk4_core(m, y, k1, p, n, (*h) / 2.0, t1, k2, k3, k4, t);
    orc_slope(m, t1, p, k1);
    rk4_core(m, t1, k1, p, n, (*h) / 2.0, t2, k2, k3, k4, t);
    for (i = 0; i < n; i++) t1[i] = fabs(ytemp[i] - t2[i]);
    max = t1[0];
    for (i = 1; i < n; i++)
      if (max < t1[i]) max = t1[i];
    if (max <= 0.01) {
      new_h = 0.95 * (*h) * pow(fabs(0.01 / max), 0.2);
      if (new_h > 5.0 * (*h)) new_h = 5.0 * (*h);
    } else {
      new_h = 0.95 * (*h) * pow(fabs(0.01 / max), 0.25);
      if (new_h < (*h) / 10.0) new_h = (*h) / 10.0;
    }
  } while (new_h < (*h));
  memcpy(y, ytemp, sizeof(double) * n);
  free(w);
  return new_h;
}

long long orc_compute_temp(const orc_model *m, double *y, const double *p, double time_elapsed)
{
  double t, h = 0, new_h;
  long long steps = 0;
  for (t = 0, new_h = 1e-7; t < time_elapsed && new_h >= 1e-7 * 1.0e-6; t += h) {
    h = new_h;
    new_h = orc_rk4(m, y, p, &h);
    new_h = (new_h < time_elapsed - t - h) ? new_h : time_elapsed - t - h;
    steps++;
  }
  return steps;
}

/* ---------------------------------------------------------------------- */
/* steady state: Gauss-Seidel, nested multigrid                             */
/* ---------------------------------------------------------------------- */
static double gs_pack(const orc_model *m, const level_t *L, double *v)
{
  const pk_t *pk = (const pk_t *)m->pack;
  const int nl = m->nl, nr = L->nr, nc = L->nc, hs = m->hsidx, sp = m->spidx;
  const double amb = m->ambient;
  double *x = v + (size_t)nl * nr * nc;
  double delta[28], csum, wsum, max = 0;
  int i, j;
  csum = 1.0 / (pk->r_hs_per + pk->r_amb_per) + 1.0 / (pk->r_hs2_y + pk->r_hs);
  wsum = amb / (pk->r_hs_per + pk->r_amb_per) + x[SINK_C_N] / (pk->r_hs2_y + pk->r_hs);
  delta[SINK_N] = fabs(x[SINK_N] - wsum / csum); x[SINK_N] = wsum / csum;
  wsum = amb / (pk->r_hs_per + pk->r_amb_per) + x[SINK_C_S] / (pk->r_hs2_y + pk->r_hs);
  delta[SINK_S] = fabs(x[SINK_S] - wsum / csum); x[SINK_S] = wsum / csum;
  csum = 1.0 / (pk->r_hs_per + pk->r_amb_per) + 1.0 / (pk->r_hs2_x + pk->r_hs);
  wsum = amb / (pk->r_hs_per + pk->r_amb_per) + x[SINK_C_W] / (pk->r_hs2_x + pk->r_hs);
  delta[SINK_W] = fabs(x[SINK_W] - wsum / csum); x[SINK_W] = wsum / csum;
  wsum = amb / (pk->r_hs_per + pk->r_amb_per) + x[SINK_C_E] / (pk->r_hs2_x + pk->r_hs);
  delta[SINK_E] = fabs(x[SINK_E] - wsum / csum); x[SINK_E] = wsum / csum;

  csum = nc / (m->ry[hs] / 2.0 + nc * pk->r_hs1_y);
  csum += 1.0 / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) + 1.0 / pk->r_sp_per_y + 1.0 / (pk->r_hs2_y + pk->r_hs);
  wsum = 0.0;
  for (j = 0; j < nc; j++) wsum += V3(v, hs, 0, j);
  wsum /= (m->ry[hs] / 2.0 + nc * pk->r_hs1_y);
  wsum += amb / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) + x[SP_N] / pk->r_sp_per_y + x[SINK_N] / (pk->r_hs2_y + pk->r_hs);
  delta[SINK_C_N] = fabs(x[SINK_C_N] - wsum / csum); x[SINK_C_N] = wsum / csum;
  wsum = 0.0;
  for (j = 0; j < nc; j++) wsum += V3(v, hs, nr - 1, j);
  wsum /= (m->ry[hs] / 2.0 + nc * pk->r_hs1_y);
  wsum += amb / (pk->r_hs_c_per_y + pk->r_amb_c_per_y) + x[SP_S] / pk->r_sp_per_y + x[SINK_S] / (pk->r_hs2_y + pk->r_hs);
  delta[SINK_C_S] = fabs(x[SINK_C_S] - wsum / csum); x[SINK_C_S] = wsum / csum;
  csum = nr / (m->rx[hs] / 2.0 + nr * pk->r_hs1_x);
  csum += 1.0 / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) + 1.0 / pk->r_sp_per_x + 1.0 / (pk->r_hs2_x + pk->r_hs);
  wsum = 0.0;
  for (i = 0; i < nr; i++) wsum += V3(v, hs, i, 0);
  wsum /= (m->rx[hs] / 2.0 + nr * pk->r_hs1_x);
  wsum += amb / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) + x[SP_W] / pk->r_sp_per_x + x[SINK_W] / (pk->r_hs2_x + pk->r_hs);
  delta[SINK_C_W] = fabs(x[SINK_C_W] - wsum / csum); x[SINK_C_W] = wsum / csum;
  wsum = 0.0;
  for (i = 0; i < nr; i++) wsum += V3(v, hs, i, nc - 1);
  wsum /= (m->rx[hs] / 2.0 + nr * pk->r_hs1_x);
  wsum += amb / (pk->r_hs_c_per_x + pk->r_amb_c_per_x) + x[SP_E] / pk->r_sp_per_x + x[SINK_E] / (pk->r_hs2_x + pk->r_hs);
  delta[SINK_C_E] = fabs(x[SINK_C_E] - wsum / csum); x[SINK_C_E] = wsum / csum;

  csum = nc / (m->ry[sp] / 2.0 + nc * pk->r_sp1_y);
  csum += 1.0 / pk->r_sp_per_y;
  wsum = 0.0;
  for (j = 0; j < nc; j++) wsum += V3(v, sp, 0, j);
  wsum /= (m->ry[sp] / 2.0 + nc * pk->r_sp1_y);
  wsum += x[SINK_C_N] / pk->r_sp_per_y;
  delta[SP_N] = fabs(x[SP_N] - wsum / csum); x[SP_N] = wsum / csum;
  wsum = 0.0;
  for (j = 0; j < nc; j++) wsum += V3(v, sp, nr - 1, j);
  wsum /= (m->ry[sp] / 2.0 + nc * pk->r_sp1_y);
  wsum += x[SINK_C_S] / pk->r_sp_per_y;
  delta[SP_S] = fabs(x[SP_S] - wsum / csum); x[SP_S] = wsum / csum;
  csum = nr / (m->rx[sp] / 2.0 + nr * pk->r_sp1_x);
  csum += 1.0 / pk->r_sp_per_x;
  wsum = 0.0;
  for (i = 0; i < nr; i++) wsum += V3(v, sp, i, 0);
  wsum /= (m->rx[sp] / 2.0 + nr * pk->r_sp1_x);
  wsum += x[SINK_C_W] / pk->r_sp_per_x;
  delta[SP_W] = fabs(x[SP_W] - wsum / csum); x[SP_W] = wsum / csum;
  wsum = 0.0;
  for (i = 0; i < nr; i++) wsum += V3(v, sp, i, nc - 1);
  wsum /= (m->rx[sp] / 2.0 + nr * pk->r_sp1_x);
  wsum += x[SINK_C_E] / pk->r_sp_per_x;
  delta[SP_E] = fabs(x[SP_E] - wsum / csum); x[SP_E] = wsum / csum;

  if (is_sec(m)) {
    const int pcb = m->pcbidx, sol = m->solderidx, sub = m->subidx;
    csum = 1.0 / (pk->r_amb_sec_per) + 1.0 / (pk->r_pcb2_y + pk->r_pcb);
    wsum = amb / (pk->r_amb_sec_per) + x[PCB_C_N] / (pk->r_pcb2_y + pk->r_pcb);
    delta[PCB_N] = fabs(x[PCB_N] - wsum / csum); x[PCB_N] = wsum / csum;
    wsum = amb / (pk->r_amb_sec_per) + x[PCB_C_S] / (pk->r_pcb2_y + pk->r_pcb);
    delta[PCB_S] = fabs(x[PCB_S] - wsum / csum); x[PCB_S] = wsum / csum;
    csum = 1.0 / (pk->r_amb_sec_per) + 1.0 / (pk->r_pcb2_x + pk->r_pcb);
    wsum = amb / (pk->r_amb_sec_per) + x[PCB_C_W] / (pk->r_pcb2_x + pk->r_pcb);
    delta[PCB_W] = fabs(x[PCB_W] - wsum / csum); x[PCB_W] = wsum / csum;
    wsum = amb / (pk->r_amb_sec_per) + x[PCB_C_E] / (pk->r_pcb2_x + pk->r_pcb);
    delta[PCB_E] = fabs(x[PCB_E] - wsum / csum); x[PCB_E] = wsum / csum;
    csum = nc / (m->ry[pcb] / 2.0 + nc * pk->r_pcb1_y);
    csum += 1.0 / (pk->r_amb_sec_c_per_y) + 1.0 / pk->r_pcb_c_per_y + 1.0 / (pk->r_pcb2_y + pk->r_pcb);
    wsum = 0.0;
    for (j = 0; j < nc; j++) wsum += V3(v, pcb, 0, j);
    wsum /= (m->ry[pcb] / 2.0 + nc * pk->r_pcb1_y);
    wsum += amb / (pk->r_amb_sec_c_per_y) + x[SOLDER_N] / pk->r_pcb_c_per_y + x[PCB_N] / (pk->r_pcb2_y + pk->r_pcb);
    delta[PCB_C_N] = fabs(x[PCB_C_N] - wsum / csum); x[PCB_C_N] = wsum / csum;
    wsum = 0.0;
    for (j = 0; j < nc; j++) wsum += V3(v, pcb, nr - 1, j);
    wsum /= (m->ry[pcb] / 2.0 + nc * pk->r_pcb1_y);
    wsum += amb / (pk->r_amb_sec_c_per_y) + x[SOLDER_S] / pk->r_pcb_c_per_y + x[PCB_S] / (pk->r_pcb2_y + pk->r_pcb);
    delta[PCB_C_S] = fabs(x[PCB_C_S] - wsum / csum); x[PCB_C_S] = wsum / csum;
    csum = nr / (m->rx[pcb] / 2.0 + nr * pk->r_pcb1_x);
    csum += 1.0 / (pk->r_amb_sec_c_per_x) + 1.0 / pk->r_pcb_c_per_x + 1.0 / (pk->r_pcb2_x + pk->r_pcb);
    wsum = 0.0;
    for (i = 0; i < nr; i++) wsum += V3(v, pcb, i, 0);
    wsum /= (m->rx[pcb] / 2.0 + nr * pk->r_pcb1_x);
    wsum += amb / (pk->r_amb_sec_c_per_x) + x[SOLDER_W] / pk->r_pcb_c_per_x + x[PCB_W] / (pk->r_pcb2_x + pk->r_pcb);
    delta[PCB_C_W] = fabs(x[PCB_C_W] - wsum / csum); x[PCB_C_W] = wsum / csum;
    wsum = 0.0;
    for (i = 0; i < nr; i++) wsum += V3(v, pcb, i, nc - 1);
    wsum /= (m->rx[pcb] / 2.0 + nr * pk->r_pcb1_x);
    wsum += amb / (pk->r_amb_sec_c_per_x) + x[SOLDER_E] / pk->r_pcb_c_per_x + x[PCB_E] / (pk->r_pcb2_x + pk->r_pcb);
    delta[PCB_C_E] = fabs(x[PCB_C_E] - wsum / csum); x[PCB_C_E] = wsum / csum;
    csum = nc / (m->ry[sol] / 2.0 + nc * pk->r_solder1_y);
    csum += 1.0 / pk->r_solder_per_y + 1.0 / pk->r_pcb_c_per_y;
    wsum = 0.0;
    for (j = 0; j < nc; j++) wsum += V3(v, sol, 0, j);
    wsum /= (m->ry[sol] / 2.0 + nc * pk->r_solder1_y);
    wsum += x[PCB_C_N] / pk->r_pcb_c_per_y + x[SUB_N] / pk->r_solder_per_y;
    delta[SOLDER_N] = fabs(x[SOLDER_N] - wsum / csum); x[SOLDER_N] = wsum / csum;
    wsum = 0.0;
    for (j = 0; j < nc; j++) wsum += V3(v, sol, nr - 1, j);
    wsum /= (m->ry[sol] / 2.0 + nc * pk->r_solder1_y);
    wsum += x[PCB_C_S] / pk->r_pcb_c_per_y + x[SUB_S] / pk->r_solder_per_y;
    delta[SOLDER_S] = fabs(x[SOLDER_S] - wsum / csum); x[SOLDER_S] = wsum / csum;
    csum = nr / (m->rx[sol] / 2.0 + nr * pk->r_solder1_x);
    csum += 1.0 / pk->r_solder_per_x + 1.0 / pk->r_pcb_c_per_x;
    wsum = 0.0;
    for (i = 0; i < nr; i++) wsum += V3(v, sol, i, 0);
    wsum /= (m->rx[sol] / 2.0 + nr * pk->r_solder1_x);
    wsum += x[PCB_C_W] / pk->r_pcb_c_per_x + x[SUB_W] / pk->r_solder_per_x;
    delta[SOLDER_W] = fabs(x[SOLDER_W] - wsum / csum); x[SOLDER_W] = wsum / csum;
    wsum = 0.0;
    for (i = 0; i < nr; i++) wsum += V3(v, sol, i, nc - 1);
    wsum /= (m->rx[sol] / 2.0 + nr * pk->r_solder1_x);
    wsum += x[PCB_C_E] / pk->r_pcb_c_per_x + x[SUB_E] / pk->r_solder_per_x;
    delta[SOLDER_E] = fabs(x[SOLDER_E] - wsum / csum); x[SOLDER_E] = wsum / csum;
    csum = nc / (m->ry[sub] / 2.0 + nc * pk->r_sub1_y);
    csum += 1.0 / pk->r_solder_per_y;
    wsum = 0.0;
    for (j = 0; j < nc; j++) wsum += V3(v, sub, 0, j);
    wsum /= (m->ry[sub] / 2.0 + nc * pk->r_sub1_y);
    wsum += x[SOLDER_N] / pk->r_solder_per_y;
    delta[SUB_N] = fabs(x[SUB_N] - wsum / csum); x[SUB_N] = wsum / csum;
    wsum = 0.0;
    for (j = 0; j < nc; j++) wsum += V3(v, sub, nr - 1, j);
    wsum /= (m->ry[sub] / 2.0 + nc * pk->r_sub1_y);
    wsum += x[SOLDER_S] / pk->r_solder_per_y;
    delta[SUB_S] = fabs(x[SUB_S] - wsum / csum); x[SUB_S] = wsum / csum;
    csum = nr / (m->rx[sub] / 2.0 + nr * pk->r_sub1_x);
    csum += 1.0 / pk->r_solder_per_x;
    wsum = 0.0;
    for (i = 0; i < nr; i++) wsum += V3(v, sub, i, 0);
    wsum /= (m->rx[sub] / 2.0 + nr * pk->r_sub1_x);
    wsum += x[SOLDER_W] / pk->r_solder_per_x;
    delta[SUB_W] = fabs(x[SUB_W] - wsum / csum); x[SUB_W] = wsum / csum;
    wsum = 0.0;
    for (i = 0; i < nr; i++) wsum += V3(v, sub, i, nc - 1);
    wsum /= (m->rx[sub] / 2.0 + nr * pk->r_sub1_x);
    wsum += x[SOLDER_E] / pk->r_solder_per_x;
    delta[SUB_E] = fabs(x[SUB_E] - wsum / csum); x[SUB_E] = wsum / csum;
  }
  for (i = 0; i < m->nx; i++)
    if (delta[i] > max) max = delta[i];
  return max;
}

static double gs_sweep_level(const orc_model *m, const level_t *L, double *v, const double *p)
{
  const pk_t *pk = (const pk_t *)m->pack;
  const int nl = m->nl, nr = L->nr, nc = L->nc;
  const size_t pl = (size_t)nr * nc;
  double *x = v + (size_t)nl * pl;
  const double cw = m->width / nc, ch = m->height / nr;
  double max = 0, pmax;
  int n, i, j;
  for (n = 0; n < nl; n++)
    for (i = 0; i < nr; i++)
      for (j = 0; j < nc; j++) {
        const size_t c = (size_t)n * pl + (size_t)i * nc + j;
        double RN, RS, RE, RW, RA, RB, csum, wsum, prev, d, R;
        if (m->field) {
          RN = m->rN[c]; RS = m->rS[c]; RE = m->rE[c]; RW = m->rW[c]; RA = m->rA[c]; RB = m->rB[c];
        } else {
          RN = RS = res_lat_ns(m, n);
          RE = RW = res_lat_ew(m, n);
          RA = n > 0 ? L->rz[n - 1] : 0;
          RB = L->rz[n];
        }
        csum = ((i > 0) ? 1.0 / RN : 0.0) + ((i < nr - 1) ? 1.0 / RS : 0.0) + ((j < nc - 1) ? 1.0 / RE : 0.0) +
               ((j > 0) ? 1.0 / RW : 0.0) + ((n > 0) ? 1.0 / RA : 0.0) + ((n < nl - 1) ? 1.0 / RB : 0.0);
        wsum = ((i > 0) ? v[c - nc] / RN : 0.0) + ((i < nr - 1) ? v[c + nc] / RS : 0.0) +
               ((j < nc - 1) ? v[c + 1] / RE : 0.0) + ((j > 0) ? v[c - 1] / RW : 0.0) +
               ((n > 0) ? v[c - pl] / RA : 0.0) + ((n < nl - 1) ? v[c + pl] / RB : 0.0);
        if (n == m->spidx) {
          R = m->ry[n] / 2.0 + nc * pk->r_sp1_y;
          if (i == 0) { csum += 1.0 / R; wsum += x[SP_N] / R; }
          if (i == nr - 1) { csum += 1.0 / R; wsum += x[SP_S] / R; }
          R = m->rx[n] / 2.0 + nr * pk->r_sp1_x;
          if (j == nc - 1) { csum += 1.0 / R; wsum += x[SP_E] / R; }
          if (j == 0) { csum += 1.0 / R; wsum += x[SP_W] / R; }
        } else if (n == m->hsidx) {
          csum += 1.0 / L->rz[n];
          wsum += m->ambient / L->rz[n];
          R = m->ry[n] / 2.0 + nc * pk->r_hs1_y;
          if (i == 0) { csum += 1.0 / R; wsum += x[SINK_C_N] / R; }
          if (i == nr - 1) { csum += 1.0 / R; wsum += x[SINK_C_S] / R; }
          R = m->rx[n] / 2.0 + nr * pk->r_hs1_x;
          if (j == nc - 1) { csum += 1.0 / R; wsum += x[SINK_C_E] / R; }
          if (j == 0) { csum += 1.0 / R; wsum += x[SINK_C_W] / R; }
        } else if (n == m->subidx && is_sec(m)) {
          R = m->ry[n] / 2.0 + nc * pk->r_sub1_y;
          if (i == 0) { csum += 1.0 / R; wsum += x[SUB_N] / R; }
          if (i == nr - 1) { csum += 1.0 / R; wsum += x[SUB_S] / R; }
          R = m->rx[n] / 2.0 + nr * pk->r_sub1_x;
          if (j == nc - 1) { csum += 1.0 / R; wsum += x[SUB_E] / R; }
          if (j == 0) { csum += 1.0 / R; wsum += x[SUB_W] / R; }
        } else if (n == m->solderidx && is_sec(m)) {
          R = m->ry[n] / 2.0 + nc * pk->r_solder1_y;
          if (i == 0) { csum += 1.0 / R; wsum += x[SOLDER_N] / R; }
          if (i == nr - 1) { csum += 1.0 / R; wsum += x[SOLDER_S] / R; }
          R = m->rx[n] / 2.0 + nr * pk->r_solder1_x;
          if (j == nc - 1) { csum += 1.0 / R; wsum += x[SOLDER_E] / R; }
          if (j == 0) { csum += 1.0 / R; wsum += x[SOLDER_W] / R; }
        } else if (n == m->pcbidx && is_sec(m)) {
          const double ra = m->pcb_amb_num / (cw * ch);
          csum += 1.0 / ra;
          wsum += m->ambient / ra;
          R = m->ry[n] / 2.0 + nc * pk->r_pcb1_y;
          if (i == 0) { csum += 1.0 / R; wsum += x[PCB_C_N] / R; }
          if (i == nr - 1) { csum += 1.0 / R; wsum += x[PCB_C_S] / R; }
          R = m->rx[n] / 2.0 + nr * pk->r_pcb1_x;
          if (j == nc - 1) { csum += 1.0 / R; wsum += x[PCB_C_E] / R; }
          if (j == 0) { csum += 1.0 / R; wsum += x[PCB_C_W] / R; }
        }
        prev = v[c];
        v[c] = (p[c] + wsum) / csum;
        d = fabs(prev - v[c]);
        if (d > max) max = d;
      }
  /* "return MAX(max, single_iteration_steady_pack(...))" (:2607) with the
   * reference's MAX macro evaluates the package update a second time
   * whenever the grid's change is not larger than the package's */
  pmax = gs_pack(m, L, v);
  if (max > pmax) return max;
  return gs_pack(m, L, v);
}

double orc_gs_sweep(const orc_model *m, double *v, const double *p)
{
  level_t L;
  finest(m, &L);
  return gs_sweep_level(m, &L, v, p);
}

static void heuristic(const orc_model *m, const level_t *L, const double *p, double *v)
{
  const int nl = m->nl;
  const size_t pl = (size_t)L->nr * L->nc;
  double *sum = calloc(pl, sizeof(double));
  size_t k;
  int n;
  for (k = 0; k < (size_t)m->nx; k++) v[(size_t)nl * pl + k] = m->ambient;
  for (n = 0; n < nl; n++)
    for (k = 0; k < pl; k++) sum[k] = sum[k] + 1.0 * p[n * pl + k];
  for (k = 0; k < pl; k++) v[(nl - 1) * pl + k] = m->ambient + sum[k] * L->rz[nl - 1];
  for (k = 0; k < pl; k++) sum[k] = sum[k] + -1.0 * p[(nl - 1) * pl + k];
  for (n = nl - 2; n >= 0; n--) {
    for (k = 0; k < pl; k++) v[n * pl + k] = v[(n + 1) * pl + k] + L->rz[n] * sum[k];
    for (k = 0; k < pl; k++) sum[k] = sum[k] + -1.0 * p[n * pl + k];
  }
  free(sum);
}

static long long gs_converge(const orc_model *m, const level_t *L, double *v, const double *p, long long cap)
{
  long long it = 0;
  double d;
  do {
    d = gs_sweep_level(m, L, v, p);
    it++;
    if (it >= cap) return -1;
  } while (!(fabs(d - 0) < 1.0e-6));
  return it;
}

static long long multigrid(const orc_model *m, level_t *L, double *v, const double *p, long long cap)
{
  const int nl = m->nl, nx = m->nx;
  long long total = 0, k;
  int n, i, j;
  if (L->nr <= 1 || L->nc <= 1) {
    heuristic(m, L, p, v);
  } else {
    level_t C = *L;
    const int cnr = L->nr / 2, cnc = L->nc / 2, fnc = L->nc;
    const size_t cpl = (size_t)cnr * cnc, fpl = (size_t)L->nr * L->nc;
    double *cp = calloc(cpl * nl + nx, sizeof(double)), *cv = calloc(cpl * nl + nx, sizeof(double));
    C.nr = cnr;
    C.nc = cnc;
    for (n = 0; n < nl; n++) {
      C.rz[n] = L->rz[n] / 4;
      C.c[n] = L->c[n] * 4;
    }
    for (n = 0; n < nl; n++)
      for (i = 0; i < cnr; i++)
        for (j = 0; j < cnc; j++)
          cp[n * cpl + i * cnc + j] = (p[n * fpl + (2 * i) * fnc + 2 * j] + p[n * fpl + (2 * i + 1) * fnc + 2 * j] +
                                       p[n * fpl + (2 * i) * fnc + 2 * j + 1] + p[n * fpl + (2 * i + 1) * fnc + 2 * j + 1]);
    for (k = 0; k < nx; k++) cp[cpl * nl + k] = p[fpl * nl + k];
    k = multigrid(m, &C, cv, cp, cap);
    if (k < 0) {
      free(cp);
      free(cv);
      return -1;
    }
    total += k;
    /* prolongation */
    for (n = 0; n < nl; n++) {
      const double *s = cv + n * cpl;
      double *d = v + n * fpl;
      for (i = 0; i < cnr - 1; i++)
        for (j = 0; j < cnc - 1; j++) {
          const double a = s[i * cnc + j], b = s[(i + 1) * cnc + j], cc = s[(i + 1) * cnc + j + 1], dd = s[i * cnc + j + 1];
          d[(2 * i + 1) * fnc + 2 * j + 1] = 9.0 / 16.0 * a + 3.0 / 16.0 * b + 1.0 / 16.0 * cc + 3.0 / 16.0 * dd;
          d[(2 * i + 2) * fnc + 2 * j + 1] = 3.0 / 16.0 * a + 9.0 / 16.0 * b + 3.0 / 16.0 * cc + 1.0 / 16.0 * dd;
          d[(2 * i + 2) * fnc + 2 * j + 2] = 1.0 / 16.0 * a + 3.0 / 16.0 * b + 9.0 / 16.0 * cc + 3.0 / 16.0 * dd;
          d[(2 * i + 1) * fnc + 2 * j + 2] = 3.0 / 16.0 * a + 1.0 / 16.0 * b + 3.0 / 16.0 * cc + 9.0 / 16.0 * dd;
        }
      for (i = 0; i < cnr; i++) {
        d[(2 * i) * fnc + 0] = d[(2 * i + 1) * fnc + 0] = s[i * cnc + 0];
        d[(2 * i) * fnc + 2 * cnc - 1] = d[(2 * i + 1) * fnc + 2 * cnc - 1] = s[i * cnc + cnc - 1];
      }
      for (j = 0; j < cnc; j++) {
        d[0 * fnc + 2 * j] = d[0 * fnc + 2 * j + 1] = s[0 * cnc + j];
        d[(2 * cnr - 1) * fnc + 2 * j] = d[(2 * cnr - 1) * fnc + 2 * j + 1] = s[(cnr - 1) * cnc + j];
      }
    }
    for (k = 0; k < nx; k++) v[fpl * nl + k] = cv[cpl * nl + k];
    free(cp);
    free(cv);
  }
  k = gs_converge(m, L, v, p, cap);
  if (k < 0) return -1;
  return total + k;
}

long long orc_steady(const orc_model *m, double *v, const double *p, long long max_sweeps)
{
  level_t L;
  finest(m, &L);
  if (m->field) {
    heuristic(m, &L, p, v);
    return gs_converge(m, &L, v, p, max_sweeps);
  }
  return multigrid(m, &L, v, p, max_sweeps);
}
