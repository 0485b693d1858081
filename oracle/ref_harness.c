/*
 * ref_harness.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A thin C harness linked against the reference HotSpot C sources (compiled
 * from where they lie by oracle/Makefile, target `ref`) so that the tests can
 * drive the reference's own grid model in-process through ctypes and read its
 * in-memory FP64 vectors (`last_trans`, `last_steady`), which the reference
 * only ever prints with "%.2f".  Nothing here is part of the product; the
 * product never links this file or the library it builds.
 *
 * Every entry point calls straight into the reference's public functions:
 *   thermal_config_add_from_strs   temperature.c:115
 *   alloc_RC_model / populate_*    temperature.c:616-650
 *   compute_temp / steady_state    temperature.c:656-780
 *   slope_fn_grid                  temperature_grid.c:3130
 *   single_iteration_steady_grid   temperature_grid.c:2426
 *   xlate_vector_b2g               temperature_grid.c:1888
 *   find_res                       temperature_grid.c:26
 *   flow_rate / hydroC             microchannel.c:567 / :361
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#include "temperature.h"
#include "temperature_grid.h"
#include "flp.h"
#include "util.h"
#include "materials.h"
#include "microchannel.h"

/* non-static reference functions without a header declaration */
double single_iteration_steady_grid(grid_model_t *model, grid_model_vector_t *power,
                                    grid_model_vector_t *temp);
void set_internal_power_grid(grid_model_t *model, double *power);
void slope_fn_grid(grid_model_t *model, double *v, grid_model_vector_t *p, double *dv);
double find_res(grid_model_t *model, int n1, int i1, int j1, int n2, int i2, int j2);
double hydroC(microchannel_config_t *config);

typedef struct {
  RC_model_t *m;
  flp_t *flp;
  materials_list_t ml;
  microchannel_config_t *uc;
  thermal_config_t cfg;
} ref_handle;

static int n_extra(grid_model_t *g)
{
  return g->config.model_secondary ? EXTRA + EXTRA_SEC : EXTRA;
}

void *ref_create(const char *flp_file, int n, const char **names, const char **values,
                 int detailed_3D, int use_uchan, const char *materials_file)
{
  int i, size;
  str_pair *table = calloc(MAX_ENTRIES, sizeof(str_pair));
  ref_handle *h = calloc(1, sizeof(ref_handle));
  for (i = 0; i < n && i < MAX_ENTRIES; i++) {
    strncpy(table[i].name, names[i], STR_SIZE - 1);
    strncpy(table[i].value, values[i], STR_SIZE - 1);
  }
  size = n;
  default_materials(&h->ml);
  if (materials_file && materials_file[0])
    materials_add_from_file(&h->ml, (char *)materials_file);
  h->cfg = default_thermal_config();
  thermal_config_add_from_strs(&h->cfg, &h->ml, table, size);
  if (use_uchan) {
    h->uc = malloc(sizeof(microchannel_config_t));
    *h->uc = default_microchannel_config();
    microchannel_config_add_from_strs(h->uc, &h->ml, table, size);
  }
  if (strcmp(h->cfg.grid_layer_file, NULLFILE))
    h->flp = NULL;
  else
    h->flp = read_flp((char *)flp_file, FALSE, FALSE);
  h->m = alloc_RC_model(&h->cfg, h->flp, h->uc, &h->ml, detailed_3D, use_uchan);
  free(table);
  return h;
}

void ref_populate(void *vh, int do_c)
{
  ref_handle *h = vh;
  populate_R_model(h->m, h->flp);
  if (do_c)
    populate_C_model(h->m, h->flp);
}

/* out: nl, nr, nc, total_n_blocks, n_extra, has_lcf */
void ref_info(void *vh, int *out)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  out[0] = g->n_layers;
  out[1] = g->rows;
  out[2] = g->cols;
  out[3] = g->total_n_blocks;
  out[4] = n_extra(g);
  out[5] = g->has_lcf;
}

/* number of blocks of layer l and whether it dissipates power */
void ref_layer_info(void *vh, int l, int *n_units, int *has_power)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  *n_units = g->layers[l].flp->n_units;
  *has_power = g->layers[l].has_power;
}

const char *ref_unit_name(void *vh, int l, int u)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  return g->layers[l].flp->units[u].name;
}

/* per layer: k, thickness, sp, rx, ry, rz, c, has_lateral, has_power, is_uchan */
void ref_layer_params(void *vh, double *out)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  int l;
  for (l = 0; l < g->n_layers; l++) {
    double *o = out + 10 * l;
    o[0] = g->layers[l].k;
    o[1] = g->layers[l].thickness;
    o[2] = g->layers[l].sp;
    o[3] = g->layers[l].rx;
    o[4] = g->layers[l].ry;
    o[5] = g->layers[l].rz;
    o[6] = g->layers[l].c;
    o[7] = g->layers[l].has_lateral;
    o[8] = g->layers[l].has_power;
    o[9] = g->layers[l].is_microchannel;
  }
}

void ref_package(void *vh, double *out)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  memcpy(out, &g->pack, sizeof(package_RC_t));
}

void ref_dims(void *vh, double *out)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  out[0] = g->width;
  out[1] = g->height;
}

void ref_compute_temp(void *vh, double *power, double *temp, double dt)
{
  compute_temp(((ref_handle *)vh)->m, power, temp, dt);
}

void ref_steady(void *vh, double *power, double *temp)
{
  steady_state_temp(((ref_handle *)vh)->m, power, temp);
}

/* which: 0 = last_trans, 1 = last_steady */
void ref_get_grid(void *vh, int which, double *out)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  grid_model_vector_t *v = which ? g->last_steady : g->last_trans;
  memcpy(out, v->cuboid[0][0],
         sizeof(double) * ((size_t)g->n_layers * g->rows * g->cols + n_extra(g)));
}

void ref_set_grid(void *vh, int which, const double *in)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  grid_model_vector_t *v = which ? g->last_steady : g->last_trans;
  memcpy(v->cuboid[0][0], in,
         sizeof(double) * ((size_t)g->n_layers * g->rows * g->cols + n_extra(g)));
}

/* block power -> grid power vector (N + extra), as the solvers see it */
void ref_power_grid(void *vh, double *power, double *out)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  grid_model_vector_t *p = new_grid_model_vector(g);
  set_internal_power_grid(g, power);
  xlate_vector_b2g(g, power, p, V_POWER);
  memcpy(out, p->cuboid[0][0],
         sizeof(double) * ((size_t)g->n_layers * g->rows * g->cols + n_extra(g)));
  free_grid_model_vector(p);
}

/* one slope evaluation dy = f(y) with a given grid power vector */
void ref_slope(void *vh, const double *y, const double *pgrid, double *dy)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  grid_model_vector_t *p = new_grid_model_vector(g);
  size_t n = (size_t)g->n_layers * g->rows * g->cols + n_extra(g);
  double *yy = malloc(sizeof(double) * n);
  memcpy(yy, y, sizeof(double) * n);
  memcpy(p->cuboid[0][0], pgrid, sizeof(double) * n);
  slope_fn_grid(g, yy, p, dy);
  free(yy);
  free_grid_model_vector(p);
}

/*
 * Keep sweeping the reference's own Gauss-Seidel update on last_steady,
 * starting from wherever steady_state_temp left it, until the per-sweep max
 * change drops below tol: the fully converged fixed point of the same
 * discrete system.  Returns the number of extra sweeps.
 */
int ref_gs_converge(void *vh, double *power, double tol, int max_sweeps)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  grid_model_vector_t *p = new_grid_model_vector(g);
  double d;
  int it = 0;
  set_internal_power_grid(g, power);
  xlate_vector_b2g(g, power, p, V_POWER);
  do {
    d = single_iteration_steady_grid(g, p, g->last_steady);
    it++;
  } while (d > tol && it < max_sweeps);
  free_grid_model_vector(p);
  return it;
}

double ref_find_res(void *vh, int n1, int i1, int j1, int n2, int i2, int j2)
{
  return find_res(((ref_handle *)vh)->m->grid, n1, i1, j1, n2, i2, j2);
}

double ref_find_cap(void *vh, int n, int i, int j)
{
  return find_cap_3D(n, i, j, ((ref_handle *)vh)->m->grid);
}

/* microchannel layer l: cell types (nr*nc ints), pressures by cell (nr*nc,
 * NAN for solid cells), returns hydroC */
double ref_uchan(void *vh, int l, int *types, double *pressure)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  microchannel_config_t *u = g->layers[l].microchannel_config;
  int i, j;
  if (!g->layers[l].is_microchannel)
    return -1.0;
  for (i = 0; i < u->num_rows; i++)
    for (j = 0; j < u->num_columns; j++) {
      types[i * u->num_columns + j] = u->cell_types[i][j];
      pressure[i * u->num_columns + j] =
        u->mapping[i][j] >= 0 ? u->b[u->mapping[i][j]] : NAN;
    }
  return hydroC(u);
}

double ref_flow_rate(void *vh, int l, int i1, int j1, int i2, int j2)
{
  grid_model_t *g = ((ref_handle *)vh)->m->grid;
  return flow_rate(g->layers[l].microchannel_config, i1, j1, i2, j2);
}

void ref_destroy(void *vh)
{
  ref_handle *h = vh;
  int lcf = h->m->grid->has_lcf;
  delete_RC_model(h->m);
  if (!lcf && h->flp)
    free_flp(h->flp, FALSE, FALSE);
  free_materials(&h->ml);
  free(h);
}
