/* grid_oracle.h -- TEST INFRASTRUCTURE ONLY: CPU restatement of the HotSpot
 * grid-model numerics used as the test oracle of libhotspot_b200.  Never linked
 * into, or called by, the product. */
#ifndef GRID_ORACLE_H
#define GRID_ORACLE_H

typedef struct orc_model {
  int nl, nr, nc, nx;                 /* layers, rows, cols, package nodes (12/28) */
  int spidx, hsidx, subidx, solderidx, pcbidx;
  int field;                          /* per-cell resistances/capacitances */
  int adv;                            /* advection arrays present */
  double ambient, width, height, pcb_amb_num;
  const double *rx, *ry, *rz, *c;     /* per layer (finest grid) */
  const double *pack;                 /* package_RC_t, 52 doubles */
  /* per cell, as find_res(neighbour, cell); zero where absent */
  const double *rN, *rS, *rW, *rE, *rA, *rB, *cap;
  /* advection per cell: Cv*flow(nbr->cell) for fluid pairs, outlet self, inlet source */
  const double *aN, *aS, *aW, *aE, *aO, *qin;
} orc_model;

/* slope_fn_grid + slope_fn_pack (temperature_grid.c:3130-3601, 2857-3093) */
void orc_slope(const orc_model *m, const double *y, const double *p, double *dy);
/* rk4 (RCutil.c:544-640): advances y in place, returns the next step */
double orc_rk4(const orc_model *m, double *y, const double *p, double *h);
/* compute_temp_grid's loop (temperature_grid.c:3676-3692); returns RK4 steps */
long long orc_compute_temp(const orc_model *m, double *y, const double *p, double time_elapsed);
/* steady_state_temp_grid without SuperLU (temperature_grid.c:2799-2851):
 * nested-iteration multigrid with lexicographic Gauss-Seidel (uniform
 * model) or plain Gauss-Seidel from the heuristic (detailed 3-D); v is the
 * finest-level vector; returns total sweeps, or -1 on the sweep cap */
long long orc_steady(const orc_model *m, double *v, const double *p, long long max_sweeps);
/* one Gauss-Seidel sweep at the finest level (single_iteration_steady_grid) */
double orc_gs_sweep(const orc_model *m, double *v, const double *p);

#endif
