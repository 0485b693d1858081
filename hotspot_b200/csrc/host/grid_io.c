/* grid_io.c -- text I/O and block-vector queries of the grid-model API.
 * Formats and messages follow the reference functions cited per function;
 * the grid dumps read the state resident on the device. */
#define _GNU_SOURCE
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

/* temperature_grid.c:1262-1295 */
void dump_steady_temp_grid(grid_model_t *model, char *file)
{
  int i, j, n;
  FILE *fp;
  if (!model->r_ready) {
    hsb_seterr(HSB_E_ARG, "R model not ready\n");
    hsb_die();
  }
  if (hsb_grid_sync_host(model)) hsb_die();
  fp = open_out(file);
  if (!fp) die_open("error: %s could not be opened for writing\n", file);
  for (n = 0; n < model->n_layers; n++) {
    fprintf(fp, "Layer %d:\n", n);
    for (i = 0; i < model->rows; i++)
      for (j = 0; j < model->cols; j++)
        fprintf(fp, "%d\t%.2f\n", i * model->cols + j, model->last_steady->cuboid[n][i][j]);
  }
  close_out(fp);
}

/* temperature_grid.c:1297-1319 */
void dump_transient_temp_grid(grid_model_t *model, int trace_num, double sampling_intvl, char *filename)
{
  FILE *fp = fopen(filename, "a");
  if (!fp) die_open("Unable to open %s for appending\n", filename);
  if (hsb_grid_sync_host(model)) hsb_die();
  fprintf(fp, "t = %lf\n", trace_num * sampling_intvl);
  for (int l = 0; l < model->n_layers; l++) {
    fprintf(fp, "Layer %d:\n", l);
    for (int i = 0; i < model->rows; i++)
      for (int j = 0; j < model->cols; j++)
        fprintf(fp, "%d\t%.2f\n", i * model->cols + j, model->last_trans->cuboid[l][i][j]);
  }
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
