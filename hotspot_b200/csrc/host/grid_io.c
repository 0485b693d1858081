/* grid_io.c -- text I/O and block-vector queries of the grid-model API.
 * Formats and messages follow the reference functions cited per function;
 * the grid dumps read the state resident on the device. */
#define _GNU_SOURCE
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "host_internal.h"
#include "hotspot_b200.h"

static int n_extra(const grid_model_t *m)
{
  return m->config.model_secondary ? HSB_EXTRA + HSB_EXTRA_SEC : HSB_EXTRA;
}

static FILE *open_out(const char *file)
{
  if (!strcasecmp(file, "stdout")) return stdout;
  if (!strcasecmp(file, "stderr")) return stderr;
  return fopen(file, "w");
}

static void close_out(FILE *fp)
{
  if (fp != stdout && fp != stderr) fclose(fp);
}

static void die_open(const char *fmt, const char *file)
{
  hsb_seterr(HSB_E_ARG, fmt, file);
  hsb_die();
}

/* layer name prefixes of block-level dumps (temperature_grid.c:1351-1433) */
static int layer_prefix(const grid_model_t *m, int n, char *str)
{
  const int nl = m->n_layers;
  const int sp = nl - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SP, hs = nl - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SINK;
  if (!m->config.model_secondary) {
    if (!m->has_lcf) {
      if (n == HSB_LAYER_SI) strcpy(str, "");
      else if (n == HSB_LAYER_INT) strcpy(str, "iface_");
      else if (n == sp) strcpy(str, "hsp_");
      else if (n == hs) strcpy(str, "hsink_");
      else return -1;
    } else {
      if (n == sp) strcpy(str, "hsp_");
      else if (n == hs) strcpy(str, "hsink_");
      else sprintf(str, "layer_%d_", n);
    }
  } else {
    const int sil = HSB_SEC_PACK_LAYERS + HSB_SEC_CHIP_LAYERS + HSB_LAYER_SI;
    const int itf = HSB_SEC_PACK_LAYERS + HSB_SEC_CHIP_LAYERS + HSB_LAYER_INT;
    const int c4 = HSB_SEC_PACK_LAYERS + HSB_LAYER_C4, metal = HSB_SEC_PACK_LAYERS + HSB_LAYER_METAL;
    if (!m->has_lcf) {
      if (n == sil) strcpy(str, "");
      else if (n == itf) strcpy(str, "iface_");
      else if (n == sp) strcpy(str, "hsp_");
      else if (n == hs) strcpy(str, "hsink_");
      else if (n == metal) strcpy(str, "metal_");
      else if (n == c4) strcpy(str, "c4_");
      else if (n == HSB_LAYER_SUB) strcpy(str, "sub_");
      else if (n == HSB_LAYER_SOLDER) strcpy(str, "solder_");
      else if (n == HSB_LAYER_PCB) strcpy(str, "pcb_");
      else return -1;
    } else {
      if (n == sp) strcpy(str, "hsp_");
      else if (n == hs) strcpy(str, "hsink_");
      else if (n == HSB_LAYER_SUB) strcpy(str, "sub_");
      else if (n == HSB_LAYER_SOLDER) strcpy(str, "solder_");
      else if (n == HSB_LAYER_PCB) strcpy(str, "pcb_");
      else sprintf(str, "layer_%d_", n);
    }
  }
  return 0;
}

/* ------------------------------------------------------------------------
 * Grid dump rows, "%d\t%.2f\n" per cell, without printf per value.
 *
 * A value v in [0, 1e7) is rounded to hundredths from x = v * 100: the
 * product's rounding error is below 1e-7 there, so when x is at least 1e-6
 * away from a rounding tie (x - floor(x) = 0.5) the nearest integer to x is
 * the nearest integer to the exact 100 v, which is what printf's correctly
 * rounded "%.2f" prints.  Other values (near ties, negative, large, inf,
 * nan) go through snprintf.  The output is byte-identical to the reference's
 * fprintf loop.
 * ------------------------------------------------------------------------ */
#define GRID_ROW_MAX 400   /* bytes one row can take (an index and any double) */

static char *put_uint(char *p, unsigned long long u)
{
  char t[24];
  int k = 0;
  do {
    t[k++] = (char)('0' + u % 10);
    u /= 10;
  } while (u);
  while (k) *p++ = t[--k];
  return p;
}

static char *put_value(char *p, double v)
{
  if (!signbit(v) && v < 1e7) {   /* -0.0 prints as "-0.00": snprintf */
    const double x = v * 100.0, fl = floor(x), fr = x - fl;
    if (fabs(fr - 0.5) >= 1e-6) {
      const unsigned long long q = (unsigned long long)fl + (fr > 0.5 ? 1u : 0u);
      p = put_uint(p, q / 100);
      *p++ = '.';
      *p++ = (char)('0' + (q % 100) / 10);
      *p++ = (char)('0' + q % 10);
      return p;
    }
  }
  return p + snprintf(p, GRID_ROW_MAX - 16, "%.2f", v);
}

long long hsb_format_grid_rows(const double *v, long long n, char *out, long long cap)
{
  if (n < 0 || !out || (n && !v)) return HSB_E_ARG;
  if (cap < n * GRID_ROW_MAX) return HSB_E_ARG;
  char *p = out;
  for (long long k = 0; k < n; k++) {
    p = put_uint(p, (unsigned long long)k);
    *p++ = '\t';
    p = put_value(p, v[k]);
    *p++ = '\n';
  }
  return (long long)(p - out);
}

/* the "Layer %d:" blocks of a grid vector, rows formatted in chunks */
static int write_grid_layers(FILE *fp, const grid_model_t *model, const grid_model_vector_t *g)
{
  const long long plane = (long long)model->rows * model->cols, chunk = 8192;
  char *buf = malloc((size_t)(chunk * GRID_ROW_MAX));
  if (!buf) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  for (int l = 0; l < model->n_layers; l++) {
    fprintf(fp, "Layer %d:\n", l);
    const double *base = &g->cuboid[l][0][0];
    for (long long k0 = 0; k0 < plane; k0 += chunk) {
      const long long k = plane - k0 < chunk ? plane - k0 : chunk;
      char *p = buf;
      for (long long q = 0; q < k; q++) {   /* the row index runs over the whole plane */
        p = put_uint(p, (unsigned long long)(k0 + q));
        *p++ = '\t';
        p = put_value(p, base[k0 + q]);
        *p++ = '\n';
      }
      fwrite(buf, 1, (size_t)(p - buf), fp);
    }
  }
  free(buf);
  return HSB_OK;
}

/* ------------------------------------------------------------------------
 * Binary checkpoint of the grid state (no counterpart in the reference):
 * an 8-byte magic, the layer/row/column/extra-node counts (int32), the
 * vector length (int64), then the transient and the steady grid vectors
 * (FP64, native byte order).
 * ------------------------------------------------------------------------ */
static const char STATE_MAGIC[8] = {'H', 'S', 'B', 'G', 'R', 'I', 'D', '1'};

typedef struct {
  char magic[8];
  int32_t layers, rows, cols, extra;
  int64_t vlen;
} state_header_t;

static void state_header(const grid_model_t *m, state_header_t *h)
{
  memset(h, 0, sizeof(*h));
  memcpy(h->magic, STATE_MAGIC, sizeof(STATE_MAGIC));
  h->layers = m->n_layers;
  h->rows = m->rows;
  h->cols = m->cols;
  h->extra = n_extra(m);
  h->vlen = (int64_t)m->n_layers * m->rows * m->cols + h->extra;
}

int hsb_grid_save_state(grid_model_t *model, const char *path)
{
  if (!model || !path) return hsb_seterr(HSB_E_ARG, "null argument\n");
  state_header_t h;
  state_header(model, &h);
  double *v = malloc(sizeof(double) * (size_t)h.vlen * 2);
  if (!v) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  int rc = hsb_grid_get_state(model, 0, v);
  if (!rc) rc = hsb_grid_get_state(model, 1, v + h.vlen);
  if (rc) {
    free(v);
    return rc;
  }
  FILE *fp = fopen(path, "wb");
  if (!fp) {
    free(v);
    return hsb_seterr(HSB_E_ARG, "unable to open %s for writing\n", path);
  }
  const int ok = fwrite(&h, sizeof(h), 1, fp) == 1 && fwrite(v, sizeof(double), (size_t)h.vlen * 2, fp) ==
                 (size_t)h.vlen * 2;
  free(v);
  if (fclose(fp) != 0 || !ok) return hsb_seterr(HSB_E_ARG, "error writing %s\n", path);
  return HSB_OK;
}

int hsb_grid_load_state(grid_model_t *model, const char *path)
{
  if (!model || !path) return hsb_seterr(HSB_E_ARG, "null argument\n");
  state_header_t want, h;
  state_header(model, &want);
  FILE *fp = fopen(path, "rb");
  if (!fp) return hsb_seterr(HSB_E_ARG, "unable to open %s for reading\n", path);
  if (fread(&h, sizeof(h), 1, fp) != 1 || memcmp(h.magic, STATE_MAGIC, sizeof(STATE_MAGIC))) {
    fclose(fp);
    return hsb_seterr(HSB_E_ARG, "%s is not a grid-state checkpoint\n", path);
  }
  if (h.layers != want.layers || h.rows != want.rows || h.cols != want.cols || h.extra != want.extra ||
      h.vlen != want.vlen) {
    fclose(fp);
    return hsb_seterr(HSB_E_ARG, "checkpoint %s holds a %dx%dx%d grid with %d extra nodes; the model has "
                                 "%dx%dx%d with %d\n", path, h.layers, h.rows, h.cols, h.extra, want.layers,
                      want.rows, want.cols, want.extra);
  }
  double *v = malloc(sizeof(double) * (size_t)h.vlen * 2);
  if (!v) {
    fclose(fp);
    return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  }
  const size_t got = fread(v, sizeof(double), (size_t)h.vlen * 2, fp);
  fclose(fp);
  int rc = got == (size_t)h.vlen * 2 ? HSB_OK : hsb_seterr(HSB_E_ARG, "%s is truncated\n", path);
  if (!rc) rc = hsb_grid_set_state(model, 0, v);
  if (!rc) rc = hsb_grid_set_state(model, 1, v + h.vlen);
  free(v);
  return rc;
}

/* temperature_grid.c:1262-1295 */
void dump_steady_temp_grid(grid_model_t *model, char *file)
{
  FILE *fp;
  if (!model->r_ready) {
    hsb_seterr(HSB_E_ARG, "R model not ready\n");
    hsb_die();
  }
  if (hsb_grid_sync_host(model)) hsb_die();
  fp = open_out(file);
  if (!fp) die_open("error: %s could not be opened for writing\n", file);
  if (write_grid_layers(fp, model, model->last_steady)) hsb_die();
  close_out(fp);
}

/* temperature_grid.c:1297-1319 */
void dump_transient_temp_grid(grid_model_t *model, int trace_num, double sampling_intvl, char *filename)
{
  FILE *fp = fopen(filename, "a");
  if (!fp) die_open("Unable to open %s for appending\n", filename);
  if (hsb_grid_sync_host(model)) hsb_die();
  fprintf(fp, "t = %lf\n", trace_num * sampling_intvl);
  if (write_grid_layers(fp, model, model->last_trans)) hsb_die();
  fclose(fp);
}

/* temperature_grid.c:1322-1447 */
void dump_temp_grid(grid_model_t *model, double *temp, char *file)
{
  int i, n, base = 0;
  char str[HSB_STR_SIZE];
  FILE *fp = open_out(file);
  if (!fp) die_open("error: %s could not be opened for writing\n", file);
  for (n = 0; n < model->n_layers; n++) {
    if (layer_prefix(model, n, str)) {
      hsb_seterr(HSB_E_ARG, "unknown layer\n");
      hsb_die();
    }
    for (i = 0; i < model->layers[n].flp->n_units; i++)
      fprintf(fp, "%s%s\t%.2f\n", str, model->layers[n].flp->units[i].name, temp[base + i]);
    base += model->layers[n].flp->n_units;
  }
  for (i = 0; i < n_extra(model); i++) fprintf(fp, "inode_%d\t%.2f\n", i, temp[base + i]);
  close_out(fp);
}

/* temperature_grid.c:1462-1642 */
void read_temp_grid(grid_model_t *model, double *temp, char *file, int clip)
{
  int i, n, idx, base = 0;
  double max = 0, val;
  char *ptr, str1[HSB_LINE_SIZE], str2[HSB_LINE_SIZE], name[HSB_STR_SIZE], format[HSB_STR_SIZE], pre[HSB_STR_SIZE];
  FILE *fp = !strcasecmp(file, "stdin") ? stdin : fopen(file, "r");
  if (!fp) die_open("error: %s could not be opened for reading\n", file);
  for (n = 0; n < model->n_layers; n++) {
    if (layer_prefix(model, n, pre)) {
      hsb_seterr(HSB_E_ARG, "unknown layer\n");
      hsb_die();
    }
    snprintf(format, sizeof(format), "%s%%s%%lf", pre);
    for (i = 0; i < model->layers[n].flp->n_units; i++) {
      if (!fgets(str1, sizeof(str1), fp)) {
        hsb_seterr(HSB_E_ARG, "not enough lines in temperature file\n");
        hsb_die();
      }
      strcpy(str2, str1);
      ptr = strtok(str1, " \r\t\n");
      if (!ptr || ptr[0] == '#') {
        i--;
        continue;
      }
      if (sscanf(str2, format, name, &val) != 2) {
        hsb_seterr(HSB_E_ARG, "invalid temperature file format\n");
        hsb_die();
      }
      idx = hsb_flp_index(model->layers[n].flp, name);
      if (idx < 0) {
        hsb_seterr(HSB_E_ARG, "block %s not found\n", name);
        hsb_die();
      }
      temp[base + idx] = val;
      if (n == 0 && temp[idx] > max) max = temp[idx];
    }
    base += model->layers[n].flp->n_units;
  }
  for (i = 0; i < n_extra(model); i++) {
    if (!fgets(str1, sizeof(str1), fp)) {
      hsb_seterr(HSB_E_ARG, "not enough lines in temperature file\n");
      hsb_die();
    }
    strcpy(str2, str1);
    ptr = strtok(str1, " \r\t\n");
    if (!ptr || ptr[0] == '#') {
      i--;
      continue;
    }
    if (sscanf(str2, "%s%lf", name, &val) != 2) {
      hsb_seterr(HSB_E_ARG, "invalid temperature file format\n");
      hsb_die();
    }
    sprintf(str1, "inode_%d", i);
    if (strcasecmp(str1, name)) {
      hsb_seterr(HSB_E_ARG, "invalid temperature file format\n");
      hsb_die();
    }
    temp[base + i] = val;
  }
  if (fgets(str1, sizeof(str1), fp)) {
    hsb_seterr(HSB_E_ARG, "too many lines in temperature file\n");
    hsb_die();
  }
  if (fp != stdin) fclose(fp);
  if (clip && (max > model->config.thermal_threshold)) {
    const double factor = (model->config.thermal_threshold - model->config.ambient) / (max - model->config.ambient);
    for (i = 0; i < model->total_n_blocks + n_extra(model); i++)
      temp[i] = (temp[i] - model->config.ambient) * factor + model->config.ambient;
  }
}

/* temperature_grid.c:1645-1681 */
void dump_power_grid(grid_model_t *model, double *power, char *file)
{
  int i, n, base = 0;
  FILE *fp = open_out(file);
  if (!fp) die_open("error: %s could not be opened for writing\n", file);
  for (n = 0; n < model->n_layers; n++) {
    if (model->layers[n].has_power)
      for (i = 0; i < model->layers[n].flp->n_units; i++) {
        if (model->has_lcf)
          fprintf(fp, "layer_%d_%s\t%.6f\n", n, model->layers[n].flp->units[i].name, power[base + i]);
        else
          fprintf(fp, "%s\t%.6f\n", model->layers[n].flp->units[i].name, power[base + i]);
      }
    base += model->layers[n].flp->n_units;
  }
  close_out(fp);
}

/* temperature_grid.c:1684-1764 */
void read_power_grid(grid_model_t *model, double *power, char *file)
{
  int i, idx, n, base = 0;
  double val;
  char *ptr, str1[HSB_LINE_SIZE], str2[HSB_LINE_SIZE], name[HSB_STR_SIZE], format[HSB_STR_SIZE];
  FILE *fp = !strcasecmp(file, "stdin") ? stdin : fopen(file, "r");
  if (!fp) die_open("error: %s could not be opened for reading\n", file);
  if (model->has_lcf) {
    for (n = 0; n < model->n_layers; n++) {
      if (model->layers[n].has_power)
        for (i = 0; i < model->layers[n].flp->n_units; i++) {
          if (!fgets(str1, sizeof(str1), fp)) {
            hsb_seterr(HSB_E_ARG, "not enough lines in power file\n");
            hsb_die();
          }
          strcpy(str2, str1);
          ptr = strtok(str1, " \r\t\n");
          if (!ptr || ptr[0] == '#') {
            i--;
            continue;
          }
          sprintf(format, "layer_%d_%%s%%lf", n);
          if (sscanf(str2, format, name, &val) != 2) {
            hsb_seterr(HSB_E_ARG, "invalid power file format\n");
            hsb_die();
          }
          idx = hsb_flp_index(model->layers[n].flp, name);
          if (idx < 0) {
            hsb_seterr(HSB_E_ARG, "block %s not found\n", name);
            hsb_die();
          }
          power[base + idx] = val;
        }
      base += model->layers[n].flp->n_units;
    }
    if (fgets(str1, sizeof(str1), fp)) {
      hsb_seterr(HSB_E_ARG, "too many lines in power file\n");
      hsb_die();
    }
  } else {
    while (fgets(str1, sizeof(str1), fp)) {
      strcpy(str2, str1);
      ptr = strtok(str1, " \r\t\n");
      if (!ptr || ptr[0] == '#') continue;
      if (sscanf(str2, "%s%lf", name, &val) != 2) {
        hsb_seterr(HSB_E_ARG, "invalid power file format\n");
        hsb_die();
      }
      idx = hsb_flp_index(model->layers[HSB_LAYER_SI].flp, name);
      if (idx < 0) {
        hsb_seterr(HSB_E_ARG, "block %s not found\n", name);
        hsb_die();
      }
      power[idx] = val;
    }
  }
  if (fp != stdin) fclose(fp);
}

/* temperature_grid.c:1766-1790 */
double find_max_temp_grid(grid_model_t *model, double *temp)
{
  int i, sil;
  double max = 0.0;
  if (!model->config.model_secondary) sil = HSB_LAYER_SI;
  else sil = model->has_lcf ? HSB_SEC_PACK_LAYERS : HSB_SEC_PACK_LAYERS + HSB_SEC_CHIP_LAYERS;
  for (i = 0; i < model->layers[sil].flp->n_units; i++) {
    if (temp[i] < 0) {
      hsb_seterr(HSB_E_ARG, "negative temperature!\n");
      hsb_die();
    } else if (max < temp[i]) {
      max = temp[i];
    }
  }
  return max;
}

/* temperature_grid.c:1792-1814 */
double find_avg_temp_grid(grid_model_t *model, double *temp)
{
  int i, n, base = 0, count = 0;
  double sum = 0.0;
  for (n = 0; n < model->n_layers; n++) {
    if (model->layers[n].has_power) {
      for (i = 0; i < model->layers[n].flp->n_units; i++) {
        if (temp[base + i] < 0) {
          hsb_seterr(HSB_E_ARG, "negative temperature!\n");
          hsb_die();
        }
        sum += temp[base + i];
      }
      count += model->layers[n].flp->n_units;
    }
    base += model->layers[n].flp->n_units;
  }
  if (!count) {
    hsb_seterr(HSB_E_ARG, "no power dissipating units?!\n");
    hsb_die();
  }
  return sum / count;
}

/* temperature_grid.c:1816-1858 */
double calc_sink_temp_grid(grid_model_t *model, double *temp, thermal_config_t *config)
{
  int i, n, base = 0;
  const int hs = model->n_layers - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SINK;
  double sum = 0.0;
  const double spr_size = config->s_spreader * config->s_spreader;
  const double sink_size = config->s_sink * config->s_sink;
  for (n = 0; n < hs; n++) base += model->layers[n].flp->n_units;
  for (i = base; i < base + model->layers[n].flp->n_units; i++) {
    if (temp[i] < 0) {
      hsb_seterr(HSB_E_ARG, "negative temperature!\n");
      hsb_die();
    }
    sum += temp[i] * (model->layers[n].flp->units[i - base].width * model->layers[n].flp->units[i - base].height);
  }
  base = model->total_n_blocks;
  for (i = HSB_SINK_C_W; i <= HSB_SINK_C_E; i++) {
    if (temp[i + base] < 0) { hsb_seterr(HSB_E_ARG, "negative temperature!\n"); hsb_die(); }
    sum += temp[i + base] * 0.25 * (config->s_spreader + model->height) * (config->s_spreader - model->width);
  }
  for (i = HSB_SINK_C_N; i <= HSB_SINK_C_S; i++) {
    if (temp[i + base] < 0) { hsb_seterr(HSB_E_ARG, "negative temperature!\n"); hsb_die(); }
    sum += temp[i + base] * 0.25 * (config->s_spreader + model->width) * (config->s_spreader - model->height);
  }
  for (i = HSB_SINK_W; i <= HSB_SINK_S; i++) {
    if (temp[i + base] < 0) { hsb_seterr(HSB_E_ARG, "negative temperature!\n"); hsb_die(); }
    sum += temp[i + base] * 0.25 * (sink_size - spr_size);
  }
  return sum / sink_size;
}

/* temperature_grid.c:3792-3840 (summary form) */
void debug_print_grid(grid_model_t *model)
{
  int i;
  fprintf(stdout, "printing grid model information...\n");
  fprintf(stdout, "rows: %d\n", model->rows);
  fprintf(stdout, "cols: %d\n", model->cols);
  fprintf(stdout, "width: %f\n", model->width);
  fprintf(stdout, "height: %f\n", model->height);
  fprintf(stdout, "total_n_blocks: %d\n", model->total_n_blocks);
  fprintf(stdout, "map_mode: %d\n", model->map_mode);
  fprintf(stdout, "r_ready: %d\n", model->r_ready);
  fprintf(stdout, "c_ready: %d\n", model->c_ready);
  fprintf(stdout, "has_lcf: %d\n", model->has_lcf);
  for (i = 0; i < model->n_layers; i++) {
    const layer_t *L = &model->layers[i];
    fprintf(stdout, "layer %d: lateral %d power %d k %g thickness %g sp %g rx %g ry %g rz %g c %g uchan %d\n",
            L->no, L->has_lateral, L->has_power, L->k, L->thickness, L->sp, L->rx, L->ry, L->rz, L->c,
            L->is_microchannel);
  }
}

flp_t *hsb_read_flp(const char *file)
{
  flp_t *f = NULL;
  if (hsb_read_flp_file(file, &f)) return NULL;
  return f;
}

void hsb_free_flp_public(flp_t *flp) { hsb_free_flp(flp); }

/* struct sizes of the boundary types, so bindings can verify their layouts */
int hsb_abi_sizes(long long *out, int n)
{
  const long long s[] = {(long long)sizeof(thermal_config_t), (long long)sizeof(unit_t),
                         (long long)sizeof(flp_t), (long long)sizeof(materials_list_t),
                         (long long)sizeof(microchannel_config_t), (long long)sizeof(package_RC_t),
                         (long long)sizeof(layer_t), (long long)sizeof(grid_model_vector_t),
                         (long long)sizeof(grid_model_t), (long long)sizeof(hsb_stats)};
  const int k = (int)(sizeof(s) / sizeof(s[0]));
  for (int i = 0; i < n && i < k; i++) out[i] = s[i];
  return k;
}
