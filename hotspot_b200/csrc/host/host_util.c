/* host_util.c -- error handling, tolerant arithmetic, floorplan reading,
 * materials lookup and package R/C for libhotspot_b200's host code.
 * Semantics follow the reference's util.c, flp.c, materials.c and
 * temperature.c (cited per function); the code is this library's own. */
#define _GNU_SOURCE
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "host_internal.h"

static __thread char g_msg[2048];

int hsb_seterr(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_msg, sizeof(g_msg), fmt, ap);
  va_end(ap);
  return code;
}

const char *hsb_errmsg(void) { return g_msg; }

void hsb_die(void)
{
  size_t n = strlen(g_msg);
  fprintf(stderr, "error: %s%s", g_msg, (n && g_msg[n - 1] == '\n') ? "" : "\n");
  exit(1);
}

void hsb_warn(const char *msg) { fprintf(stderr, "warning: %s", msg); }

/* util.c:17-20 */
int hsb_eq(double x, double y) { return fabs(x - y) < HSB_DELTA; }

/* util.c:57-77: values within DELTA of an integer snap to it */
int hsb_tolerant_ceil(double v)
{
  double nearest = floor(v + 0.5);
  if (hsb_eq(v, nearest)) return (int)nearest;
  return (int)ceil(v);
}

int hsb_tolerant_floor(double v)
{
  double nearest = floor(v + 0.5);
  if (hsb_eq(v, nearest)) return (int)nearest;
  return (int)floor(v);
}

/* RCutil.c:20-31 */
double hsb_getr(double k, double thickness, double area) { return thickness / (k * area); }
double hsb_getcap(double sp, double thickness, double area)
{
  return HSB_C_FACTOR * sp * thickness * area;
}

/* contiguous [nl][nr][nc] + tail, row pointers as dcuboid_tail (util.c:231-261) */
double ***hsb_dcuboid_tail(int nr, int nc, int nl, int xtra)
{
  int i, j;
  double ***m = calloc(nl, sizeof(double **));
  if (!m) return NULL;
  m[0] = calloc((size_t)nl * nr, sizeof(double *));
  m[0][0] = calloc((size_t)nl * nr * nc + xtra, sizeof(double));
  if (!m[0] || !m[0][0]) return NULL;
  for (i = 1; i < nl; i++) m[i] = m[0] + (size_t)nr * i;
  for (i = 0; i < nl; i++)
    for (j = 0; j < nr; j++) m[i][j] = m[0][0] + (size_t)nr * nc * i + (size_t)nc * j;
  return m;
}

void hsb_free_dcuboid(double ***m)
{
  if (!m) return;
  free(m[0][0]);
  free(m[0]);
  free(m);
}

/* ------------------------------------------------------------------------ */
/* floorplans                                                               */
/* ------------------------------------------------------------------------ */

/* Parse floorplan text: "name width height leftx bottomy [cv rho]" per unit,
 * '#' comments and blank lines skipped, 3-field connectivity lines ignored
 * (flp.c:1004-1124), then translated so the minimum corner is (0,0)
 * (flp.c:334-350). */
int hsb_read_flp_text(const char *text, const char *what, flp_t **out)
{
  char *buf = strdup(text), *save = NULL, *line, *ptr, name[HSB_STR_SIZE], name2[HSB_STR_SIZE];
  char lcopy[HSB_LINE_SIZE];
  double w, h, x, y, cp, res, extra;
  int count = 0, i = 0, k;
  flp_t *flp;
  if (!buf) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  /* pass 1: count units (lines with more than 4 numeric-looking fields) */
  for (line = strtok_r(buf, "\n", &save); line; line = strtok_r(NULL, "\n", &save)) {
    strncpy(lcopy, line, sizeof(lcopy) - 1);
    lcopy[sizeof(lcopy) - 1] = 0;
    ptr = strtok(lcopy, " \r\t\n");
    if (!ptr || ptr[0] == '#') continue;
    if (sscanf(line, "%s%lf%lf%lf%lf%lf%lf", name, &w, &h, &x, &y, &cp, &res) > 4) count++;
  }
  free(buf);
  if (!count) return hsb_seterr(HSB_E_ARG, "no units specified in the floorplan file %s\n", what);
  flp = calloc(1, sizeof(flp_t));
  if (!flp) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  flp->units = calloc(count, sizeof(unit_t));
  flp->n_units = count;
  buf = strdup(text);
  save = NULL;
  for (line = strtok_r(buf, "\n", &save); line; line = strtok_r(NULL, "\n", &save)) {
    strncpy(lcopy, line, sizeof(lcopy) - 1);
    lcopy[sizeof(lcopy) - 1] = 0;
    ptr = strtok(lcopy, " \r\t\n");
    if (!ptr || ptr[0] == '#') continue;
    cp = res = 0.0;
    k = sscanf(line, "%s%lf%lf%lf%lf%lf%lf%lf", name, &w, &h, &x, &y, &cp, &res, &extra);
    if (k > 7) {
      free(buf);
      hsb_free_flp(flp);
      return hsb_seterr(HSB_E_ARG, "invalid floorplan file format (%s)\n", what);
    }
    if (k == 7 || k == 5) {
      if (i >= count) break;
      unit_t *u = &flp->units[i++];
      strncpy(u->name, name, HSB_STR_SIZE - 1);
      u->width = w;
      u->height = h;
      u->leftx = x;
      u->bottomy = y;
      u->specificheat = k == 7 ? cp : 0.0;
      u->resistivity = k == 7 ? res : 0.0;
      u->hasRes = u->hasSh = (k == 7);
    } else if (sscanf(line, "%s%s%lf", name, name2, &extra) != 3) {
      free(buf);
      hsb_free_flp(flp);
      return hsb_seterr(HSB_E_ARG, "invalid floorplan file format (%s)\n", what);
    }
  }
  free(buf);
  if (i != count) {
    hsb_free_flp(flp);
    return hsb_seterr(HSB_E_ARG, "mismatch of number of units (%s)\n", what);
  }
  {
    double minx = flp->units[0].leftx, miny = flp->units[0].bottomy;
    for (i = 1; i < flp->n_units; i++) {
      if (minx > flp->units[i].leftx) minx = flp->units[i].leftx;
      if (miny > flp->units[i].bottomy) miny = flp->units[i].bottomy;
    }
    for (i = 0; i < flp->n_units; i++) {
      flp->units[i].leftx += (0 - minx);
      flp->units[i].bottomy += (0 - miny);
    }
  }
  *out = flp;
  return HSB_OK;
}

int hsb_read_flp_file(const char *file, flp_t **out)
{
  FILE *fp = fopen(file, "r");
  long n;
  char *text;
  int rc;
  if (!fp) return hsb_seterr(HSB_E_ARG, "error opening file %s\n", file);
  fseek(fp, 0, SEEK_END);
  n = ftell(fp);
  fseek(fp, 0, SEEK_SET);
  text = malloc(n + 1);
  if (!text) {
    fclose(fp);
    return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  }
  n = (long)fread(text, 1, n, fp);
  text[n] = 0;
  fclose(fp);
  rc = hsb_read_flp_text(text, file, out);
  free(text);
  return rc;
}

void hsb_free_flp(flp_t *flp)
{
  if (!flp) return;
  free(flp->units);
  free(flp);
}

/* flp.c:1501-1531 */
double hsb_flp_width(const flp_t *flp)
{
  int i;
  double mn = flp->units[0].leftx, mx = flp->units[0].leftx + flp->units[0].width;
  for (i = 1; i < flp->n_units; i++) {
    if (flp->units[i].leftx < mn) mn = flp->units[i].leftx;
    if (flp->units[i].leftx + flp->units[i].width > mx) mx = flp->units[i].leftx + flp->units[i].width;
  }
  return mx - mn;
}

double hsb_flp_height(const flp_t *flp)
{
  int i;
  double mn = flp->units[0].bottomy, mx = flp->units[0].bottomy + flp->units[0].height;
  for (i = 1; i < flp->n_units; i++) {
    if (flp->units[i].bottomy < mn) mn = flp->units[i].bottomy;
    if (flp->units[i].bottomy + flp->units[i].height > mx)
      mx = flp->units[i].bottomy + flp->units[i].height;
  }
  return mx - mn;
}

/* flp.c:1385-1400 (case-insensitive name match), -1 when absent */
int hsb_flp_index(const flp_t *flp, const char *name)
{
  int i;
  for (i = 0; i < flp->n_units; i++)
    if (!strcasecmp(name, flp->units[i].name)) return i;
  return -1;
}

/* ------------------------------------------------------------------------ */
/* materials: -1 when the name is unknown (materials.c:177-205)             */
/* ------------------------------------------------------------------------ */
double hsb_material_k(const materials_list_t *ml, const char *name)
{
  int i;
  if (ml)
    for (i = 0; i < ml->size; i++)
      if (!strncmp(ml->names[i], name, HSB_STR_SIZE)) return ml->material_properties[i].thermal_conductivity;
  return -1;
}

double hsb_material_cv(const materials_list_t *ml, const char *name)
{
  int i;
  if (ml)
    for (i = 0; i < ml->size; i++)
      if (!strncmp(ml->names[i], name, HSB_STR_SIZE))
        return ml->material_properties[i].volumetric_heat_capacity;
  return -1;
}

/* ------------------------------------------------------------------------ */
/* package R and C: the lumped spreader/sink periphery (temperature.c:458-569)
 * same formulas and the same operation order as the reference.            */
/* ------------------------------------------------------------------------ */
void hsb_package_R(package_RC_t *p, const thermal_config_t *c, double width, double height)
{
  const double s_spreader = c->s_spreader, t_spreader = c->t_spreader;
  const double s_sink = c->s_sink, t_sink = c->t_sink, r_convec = c->r_convec;
  const double s_sub = c->s_sub, t_sub = c->t_sub, s_solder = c->s_solder, t_solder = c->t_solder;
  const double s_pcb = c->s_pcb, t_pcb = c->t_pcb, r_convec_sec = c->r_convec_sec;
  const double k_sink = c->k_sink, k_spreader = c->k_spreader;

  p->r_sp1_x = hsb_getr(k_spreader, (s_spreader - width) / 4.0, (s_spreader + 3 * height) / 4.0 * t_spreader);
  p->r_sp1_y = hsb_getr(k_spreader, (s_spreader - height) / 4.0, (s_spreader + 3 * width) / 4.0 * t_spreader);
  p->r_hs1_x = hsb_getr(k_sink, (s_spreader - width) / 4.0, (s_spreader + 3 * height) / 4.0 * t_sink);
  p->r_hs1_y = hsb_getr(k_sink, (s_spreader - height) / 4.0, (s_spreader + 3 * width) / 4.0 * t_sink);
  p->r_hs2_x = hsb_getr(k_sink, (s_spreader - width) / 4.0, (3 * s_spreader + height) / 4.0 * t_sink);
  p->r_hs2_y = hsb_getr(k_sink, (s_spreader - height) / 4.0, (3 * s_spreader + width) / 4.0 * t_sink);
  p->r_hs = hsb_getr(k_sink, (s_sink - s_spreader) / 4.0, (s_sink + 3 * s_spreader) / 4.0 * t_sink);

  p->r_sp_per_x = hsb_getr(k_spreader, t_spreader, (s_spreader + height) * (s_spreader - width) / 4.0);
  p->r_sp_per_y = hsb_getr(k_spreader, t_spreader, (s_spreader + width) * (s_spreader - height) / 4.0);
  p->r_hs_c_per_x = hsb_getr(k_sink, t_sink, (s_spreader + height) * (s_spreader - width) / 4.0);
  p->r_hs_c_per_y = hsb_getr(k_sink, t_sink, (s_spreader + width) * (s_spreader - height) / 4.0);
  p->r_hs_per = hsb_getr(k_sink, t_sink, (s_sink * s_sink - s_spreader * s_spreader) / 4.0);

  p->r_amb_c_per_x = r_convec * (s_sink * s_sink) / ((s_spreader + height) * (s_spreader - width) / 4.0);
  p->r_amb_c_per_y = r_convec * (s_sink * s_sink) / ((s_spreader + width) * (s_spreader - height) / 4.0);
  p->r_amb_per = r_convec * (s_sink * s_sink) / ((s_sink * s_sink - s_spreader * s_spreader) / 4.0);

  p->r_sub1_x = hsb_getr(HSB_K_SUB, (s_sub - width) / 4.0, (s_sub + 3 * height) / 4.0 * t_sub);
  p->r_sub1_y = hsb_getr(HSB_K_SUB, (s_sub - height) / 4.0, (s_sub + 3 * width) / 4.0 * t_sub);
  p->r_solder1_x = hsb_getr(HSB_K_SOLDER, (s_solder - width) / 4.0, (s_solder + 3 * height) / 4.0 * t_solder);
  p->r_solder1_y = hsb_getr(HSB_K_SOLDER, (s_solder - height) / 4.0, (s_solder + 3 * width) / 4.0 * t_solder);
  p->r_pcb1_x = hsb_getr(HSB_K_PCB, (s_solder - width) / 4.0, (s_solder + 3 * height) / 4.0 * t_pcb);
  p->r_pcb1_y = hsb_getr(HSB_K_PCB, (s_solder - height) / 4.0, (s_solder + 3 * width) / 4.0 * t_pcb);
  p->r_pcb2_x = hsb_getr(HSB_K_PCB, (s_solder - width) / 4.0, (3 * s_solder + height) / 4.0 * t_pcb);
  p->r_pcb2_y = hsb_getr(HSB_K_PCB, (s_solder - height) / 4.0, (3 * s_solder + width) / 4.0 * t_pcb);
  p->r_pcb = hsb_getr(HSB_K_PCB, (s_pcb - s_solder) / 4.0, (s_pcb + 3 * s_solder) / 4.0 * t_pcb);

  p->r_sub_per_x = hsb_getr(HSB_K_SUB, t_sub, (s_sub + height) * (s_sub - width) / 4.0);
  p->r_sub_per_y = hsb_getr(HSB_K_SUB, t_sub, (s_sub + width) * (s_sub - height) / 4.0);
  p->r_solder_per_x = hsb_getr(HSB_K_SOLDER, t_solder, (s_solder + height) * (s_solder - width) / 4.0);
  p->r_solder_per_y = hsb_getr(HSB_K_SOLDER, t_solder, (s_solder + width) * (s_solder - height) / 4.0);
  p->r_pcb_c_per_x = hsb_getr(HSB_K_PCB, t_pcb, (s_solder + height) * (s_solder - width) / 4.0);
  p->r_pcb_c_per_y = hsb_getr(HSB_K_PCB, t_pcb, (s_solder + width) * (s_solder - height) / 4.0);
  p->r_pcb_per = hsb_getr(HSB_K_PCB, t_pcb, (s_pcb * s_pcb - s_solder * s_solder) / 4.0);

  p->r_amb_sec_c_per_x = r_convec_sec * (s_pcb * s_pcb) / ((s_solder + height) * (s_solder - width) / 4.0);
  p->r_amb_sec_c_per_y = r_convec_sec * (s_pcb * s_pcb) / ((s_solder + width) * (s_solder - height) / 4.0);
  p->r_amb_sec_per = r_convec_sec * (s_pcb * s_pcb) / ((s_pcb * s_pcb - s_solder * s_solder) / 4.0);
}

void hsb_package_C(package_RC_t *p, const thermal_config_t *c, double width, double height)
{
  const double s_spreader = c->s_spreader, t_spreader = c->t_spreader;
  const double s_sink = c->s_sink, t_sink = c->t_sink, c_convec = c->c_convec;
  const double s_sub = c->s_sub, t_sub = c->t_sub, s_solder = c->s_solder, t_solder = c->t_solder;
  const double s_pcb = c->s_pcb, t_pcb = c->t_pcb, c_convec_sec = c->c_convec_sec;
  const double p_sink = c->p_sink, p_spreader = c->p_spreader;

  p->c_sp_per_x = hsb_getcap(p_spreader, t_spreader, (s_spreader + height) * (s_spreader - width) / 4.0);
  p->c_sp_per_y = hsb_getcap(p_spreader, t_spreader, (s_spreader + width) * (s_spreader - height) / 4.0);
  p->c_hs_c_per_x = hsb_getcap(p_sink, t_sink, (s_spreader + height) * (s_spreader - width) / 4.0);
  p->c_hs_c_per_y = hsb_getcap(p_sink, t_sink, (s_spreader + width) * (s_spreader - height) / 4.0);
  p->c_hs_per = hsb_getcap(p_sink, t_sink, (s_sink * s_sink - s_spreader * s_spreader) / 4.0);

  p->c_amb_c_per_x = HSB_C_FACTOR * c_convec / (s_sink * s_sink) * ((s_spreader + height) * (s_spreader - width) / 4.0);
  p->c_amb_c_per_y = HSB_C_FACTOR * c_convec / (s_sink * s_sink) * ((s_spreader + width) * (s_spreader - height) / 4.0);
  p->c_amb_per = HSB_C_FACTOR * c_convec / (s_sink * s_sink) * ((s_sink * s_sink - s_spreader * s_spreader) / 4.0);

  p->c_sub_per_x = hsb_getcap(HSB_SPEC_HEAT_SUB, t_sub, (s_sub + height) * (s_sub - width) / 4.0);
  p->c_sub_per_y = hsb_getcap(HSB_SPEC_HEAT_SUB, t_sub, (s_sub + width) * (s_sub - height) / 4.0);
  p->c_solder_per_x = hsb_getcap(HSB_SPEC_HEAT_SOLDER, t_solder, (s_solder + height) * (s_solder - width) / 4.0);
  p->c_solder_per_y = hsb_getcap(HSB_SPEC_HEAT_SOLDER, t_solder, (s_solder + width) * (s_solder - height) / 4.0);
  p->c_pcb_c_per_x = hsb_getcap(HSB_SPEC_HEAT_PCB, t_pcb, (s_solder + height) * (s_solder - width) / 4.0);
  p->c_pcb_c_per_y = hsb_getcap(HSB_SPEC_HEAT_PCB, t_pcb, (s_solder + width) * (s_solder - height) / 4.0);
  p->c_pcb_per = hsb_getcap(HSB_SPEC_HEAT_PCB, t_pcb, (s_pcb * s_pcb - s_solder * s_solder) / 4.0);

  p->c_amb_sec_c_per_x = HSB_C_FACTOR * c_convec_sec / (s_pcb * s_pcb) * ((s_solder + height) * (s_solder - width) / 4.0);
  p->c_amb_sec_c_per_y = HSB_C_FACTOR * c_convec_sec / (s_pcb * s_pcb) * ((s_solder + width) * (s_solder - height) / 4.0);
  p->c_amb_sec_per = HSB_C_FACTOR * c_convec_sec / (s_pcb * s_pcb) * ((s_pcb * s_pcb - s_solder * s_solder) / 4.0);
}
