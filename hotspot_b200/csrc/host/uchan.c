/* uchan.c -- microchannel network set-up for libhotspot_b200.
 *
 * Same semantics as the reference's microchannel.c (cell-type CSV
 * :258-315, generated floorplan :317-353, hydraulic conductance :361-376,
 * pressure network :378-565, flow rate :567-571), with one design change:
 * the reference assembles the pressure network as a dense n_fluid x n_fluid
 * matrix and solves it by Gauss-Jordan (:420-429, util.c:621), which needs
 * ~137 GB at 512x512.  Here the network is kept sparse (5-point Laplacian
 * over fluid cells with Dirichlet inlets/outlets, or a pump node behind an
 * internal resistance) and solved by Jacobi-preconditioned conjugate
 * gradients in FP64 to a relative residual of 1e-15. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "host_internal.h"

#define FLUIDT(t) ((t) == HSB_FLUID || (t) == HSB_INLET || (t) == HSB_OUTLET)
#define IS_FLUID(u, i, j) FLUIDT((u)->cell_types[i][j])

double hsb_uchan_hydroC(const microchannel_config_t *u)
{
  const double h = u->cell_thickness, w = u->cell_width, L = u->cell_height;
  const double visc = u->coolant_visc;
  if (h == w) return (0.42229 * pow(h, 4)) / (12 * visc * L);
  if (h > w) return ((1 - 0.63 * (w / h)) * (pow(w, 3)) * (h)) / (12 * visc * L);
  return ((1 - 0.63 * (h / w)) * (pow(h, 3)) * (w)) / (12 * visc * L);
}

double hsb_uchan_flow(const microchannel_config_t *u, int i1, int j1, int i2, int j2)
{
  return (u->b[u->mapping[i1][j1]] - u->b[u->mapping[i2][j2]]) * hsb_uchan_hydroC(u);
}

/* Pressure of every fluid cell.  Unknowns are the fluid cells that are not
 * Dirichlet nodes; with an ideal pump (pump_internal_res == 0) inlets sit at
 * pumping_pressure and outlets at 0; otherwise inlets connect to a pump node
 * at pumping_pressure through 1/pump_internal_res. */
static int solve_pressure(microchannel_config_t *u)
{
  const int nr = u->num_rows, nc = u->num_columns, nf = u->n_fluid_cells;
  const double g = hsb_uchan_hydroC(u);
  const int ideal = u->pump_internal_res == 0;
  const double gp = ideal ? 0.0 : 1.0 / u->pump_internal_res;
  int *ci = malloc(sizeof(int) * nf), *cj = malloc(sizeof(int) * nf), *fixed = calloc(nf, sizeof(int));
  double *x = u->b, *r = calloc(nf, sizeof(double)), *z = calloc(nf, sizeof(double));
  double *pv = calloc(nf, sizeof(double)), *q = calloc(nf, sizeof(double)), *diag = calloc(nf, sizeof(double));
  double *rhs = calloc(nf, sizeof(double));
  int i, j, k, it, rc = HSB_OK;
  static const int di[4] = {-1, 1, 0, 0}, dj[4] = {0, 0, -1, 1};
  if (!ci || !cj || !fixed || !r || !z || !pv || !q || !diag || !rhs) {
    rc = hsb_seterr(HSB_E_NOMEM, "Unable to allocate the pressure circuit\n");
    goto out;
  }
  for (i = 0; i < nr; i++)
    for (j = 0; j < nc; j++)
      if (u->mapping[i][j] >= 0) {
        ci[u->mapping[i][j]] = i;
        cj[u->mapping[i][j]] = j;
      }
  for (k = 0; k < nf; k++) {
    const int t = u->cell_types[ci[k]][cj[k]];
    x[k] = 0.0;
    if (t == HSB_OUTLET) { fixed[k] = 1; x[k] = 0.0; }
    else if (t == HSB_INLET && ideal) { fixed[k] = 1; x[k] = u->pumping_pressure; }
  }
  /* operator: (A p)_k = sum_nbr g (p_k - p_nbr) [+ gp p_k for inlets];
   * rhs carries the Dirichlet neighbours and the pump */
  for (k = 0; k < nf; k++) {
    if (fixed[k]) continue;
    double d = 0.0, b = 0.0;
    for (int e = 0; e < 4; e++) {
      const int ii = ci[k] + di[e], jj = cj[k] + dj[e];
      if (ii < 0 || ii >= nr || jj < 0 || jj >= nc || !IS_FLUID(u, ii, jj)) continue;
      const int m = u->mapping[ii][jj];
      d += g;
      if (fixed[m]) b += g * x[m];
    }
    if (!ideal && u->cell_types[ci[k]][cj[k]] == HSB_INLET) {
      d += gp;
      b += gp * u->pumping_pressure;
    }
    diag[k] = d;
    rhs[k] = b;
  }
#define APPLY(src, dst)                                                     \
  for (k = 0; k < nf; k++) {                                                \
    if (fixed[k]) { dst[k] = 0.0; continue; }                               \
    double s = diag[k] * src[k];                                            \
    for (int e = 0; e < 4; e++) {                                           \
      const int ii = ci[k] + di[e], jj = cj[k] + dj[e];                     \
      if (ii < 0 || ii >= nr || jj < 0 || jj >= nc || !IS_FLUID(u, ii, jj)) continue; \
      const int m = u->mapping[ii][jj];                                     \
      if (!fixed[m]) s -= g * src[m];                                       \
    }                                                                       \
    dst[k] = s;                                                             \
  }
  {
    /* x = 0 on the unknowns as the start; r = rhs */
    double rz = 0.0, bnorm = 0.0, rnorm;
    for (k = 0; k < nf; k++) {
      if (fixed[k]) continue;
      if (diag[k] == 0.0) {
        rc = hsb_seterr(HSB_E_ARG, "isolated fluid cell in the microchannel network\n");
        goto out;
      }
      r[k] = rhs[k];
      bnorm += rhs[k] * rhs[k];
    }
    bnorm = sqrt(bnorm);
    if (bnorm == 0.0) goto done;
    for (k = 0; k < nf; k++) {
      if (fixed[k]) continue;
      z[k] = r[k] / diag[k];
      pv[k] = z[k];
      rz += r[k] * z[k];
    }
    for (it = 0; it < 100000; it++) {
      double pq = 0.0, alpha, rz2 = 0.0, beta;
      APPLY(pv, q);
      for (k = 0; k < nf; k++) pq += pv[k] * q[k];
      alpha = rz / pq;
      rnorm = 0.0;
      for (k = 0; k < nf; k++) {
        if (fixed[k]) continue;
        x[k] += alpha * pv[k];
        r[k] -= alpha * q[k];
        rnorm += r[k] * r[k];
      }
      if (sqrt(rnorm) <= 1e-15 * bnorm) break;
      for (k = 0; k < nf; k++) {
        if (fixed[k]) continue;
        z[k] = r[k] / diag[k];
        rz2 += r[k] * z[k];
      }
      beta = rz2 / rz;
      rz = rz2;
      for (k = 0; k < nf; k++)
        if (!fixed[k]) pv[k] = z[k] + beta * pv[k];
    }
  }
#undef APPLY
done:
out:
  free(ci); free(cj); free(fixed); free(r); free(z); free(pv); free(q); free(diag); free(rhs);
  return rc;
}

/* Read the CSV of cell types, generate the layer's floorplan exactly as the
 * reference prints it (one "%e"-formatted unit per cell, so the geometry is
 * the same rounded doubles), write that .flp next to the CSV like the
 * reference does, and solve the pressure network. */
int hsb_uchan_build(microchannel_config_t *u, flp_t **flp_out)
{
  FILE *fp = fopen(u->network_file, "r");
  char line[4096], *cell, *ext;
  const int nr = u->num_rows, nc = u->num_columns;
  int i = 0, j = 0, n = 0, rc;
  size_t cap, len = 0;
  char *text;
  if (!fp) return hsb_seterr(HSB_E_ARG, "Unable to open %s\n", u->network_file);
  u->cell_types = calloc(nr, sizeof(int *));
  u->mapping = calloc(nr, sizeof(int *));
  for (i = 0; i < nr; i++) {
    u->cell_types[i] = calloc(nc, sizeof(int));
    u->mapping[i] = calloc(nc, sizeof(int));
  }
  i = 0;
  while (fgets(line, sizeof(line), fp)) {
    j = 0;
    for (cell = strtok(line, " ,\n"); cell; cell = strtok(NULL, " ,\n")) {
      if (j >= nc) {
        fclose(fp);
        return hsb_seterr(HSB_E_ARG, "Microchannel row %d has more cells than num_columns(%d)\n", i, nc);
      }
      if (i >= nr) {
        fclose(fp);
        return hsb_seterr(HSB_E_ARG, "Microchannel has more rows than num_rows(%d)\n", nr);
      }
      u->cell_types[i][j++] = atoi(cell);
    }
    i++;
  }
  fclose(fp);

  /* generated floorplan, "%e" fields as microchannel.c:335-349 */
  strcpy(u->floorplan_file, u->network_file);
  ext = strstr(u->floorplan_file, ".csv");
  if (ext) strcpy(ext, ".flp");
  cap = (size_t)nr * nc * 128 + 64;
  text = malloc(cap);
  if (!text) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  len += snprintf(text + len, cap - len, "# Name\tw\th\tx\ty\tc_v\tp\n");
  for (i = 0; i < nr; i++)
    for (j = 0; j < nc; j++) {
      const int fl = IS_FLUID(u, i, j);
      len += snprintf(text + len, cap - len, "Cell_%d_%d\t%e\t%e\t%e\t%e\t%e\t%e\n", i, j, u->cell_width,
                      u->cell_height, j * u->cell_width, (u->num_rows - i - 1) * u->cell_height,
                      fl ? u->coolant_capac : u->wall_capac, fl ? u->coolant_res : u->wall_res);
    }
  fp = fopen(u->floorplan_file, "w");
  if (fp) {
    fwrite(text, 1, len, fp);
    fclose(fp);
  }
  rc = hsb_read_flp_text(text, u->floorplan_file, flp_out);
  free(text);
  if (rc) return rc;

  /* number the fluid cells (microchannel.c:397-408) */
  for (i = 0; i < nr; i++)
    for (j = 0; j < nc; j++) u->mapping[i][j] = IS_FLUID(u, i, j) ? n++ : -1;
  u->n_fluid_cells = n;
  u->A = NULL;
  u->nnz = 0;
  u->b = calloc(n > 0 ? n : 1, sizeof(double));
  if (!u->b) return hsb_seterr(HSB_E_NOMEM, "Unable to allocate the pressure vector\n");
  return n ? solve_pressure(u) : HSB_OK;
}

void hsb_uchan_free(microchannel_config_t *u)
{
  int i;
  if (!u) return;
  if (u->cell_types) {
    for (i = 0; i < u->num_rows; i++) free(u->cell_types[i]);
    free(u->cell_types);
  }
  if (u->mapping) {
    for (i = 0; i < u->num_rows; i++) free(u->mapping[i]);
    free(u->mapping);
  }
  free(u->b);
  free(u);
}
