/* grid_model.c -- HotSpot's grid-model API (temperature_grid.h:194-254) as a
 * drop-in, backed by the device-resident model of hsb_device.h.
 *
 * The host side builds what the reference computes once per model (layers,
 * block<->grid occupancy lists, per-layer and per-cell R/C, package R/C,
 * microchannel flow) with the reference's arithmetic, then hands the arrays
 * to the device.  The hot loops (RK4 transient, steady solver, b2g/g2b) run
 * on the GPU; the model's grid state stays resident in HBM between calls.
 *
 * Error behaviour: the exported temperature_grid.h functions keep the
 * reference's fatal() semantics (message "error: ..." on stderr, exit(1),
 * util.c:32-36).  The hsb_grid_* extensions return status codes instead. */
#define _GNU_SOURCE
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "host_internal.h"
#include "hotspot_b200.h"

#define CHECK(expr)                 \
  do {                              \
    int rc_ = (expr);               \
    if (rc_) return rc_;            \
  } while (0)
#define OR_DIE(expr)                \
  do {                              \
    if ((expr) != HSB_OK) hsb_die(); \
  } while (0)

static int n_extra(const grid_model_t *m)
{
  return m->config.model_secondary ? HSB_EXTRA + HSB_EXTRA_SEC : HSB_EXTRA;
}

/* ------------------------------------------------------------------------ */
/* block lists (temperature_grid.c:193-320)                                  */
/* ------------------------------------------------------------------------ */
static blist_t *new_blist(int idx, double occupancy, double res, double sh, int first, int d3,
                          double cw, double ch, double thickness)
{
  blist_t *p = calloc(1, sizeof(blist_t));
  if (!p) return NULL;
  p->idx = idx;
  p->occupancy = occupancy;
  if (first && d3) {
    if (occupancy >= HSB_OCCUPANCY_THRESHOLD) {
      p->lock = 1;
      p->rx = hsb_getr(1 / res, cw, ch * thickness);
      p->ry = hsb_getr(1 / res, ch, cw * thickness);
      p->rz = hsb_getr(1 / res, thickness, cw * ch);
      p->capacitance = hsb_getcap(sh, thickness, cw * ch);
    } else {
      p->lock = 0;
      p->rx = 1 / ((1 / hsb_getr(1 / res, cw, ch * thickness)) * occupancy);
      p->ry = 1 / ((1 / hsb_getr(1 / res, ch, cw * thickness)) * occupancy);
      p->rz = 1 / ((1 / hsb_getr(1 / res, thickness, cw * ch)) * occupancy);
      p->capacitance = hsb_getcap(sh, thickness, cw * ch);
    }
  }
  return p;
}

static int blist_append(blist_t *head, int idx, double occupancy, double res, double sh, int first,
                        int d3, double cw, double ch, double thickness)
{
  blist_t *tail = NULL;
  if (d3 && head->lock != 1) {
    if (occupancy >= HSB_OCCUPANCY_THRESHOLD) {
      head->lock = 1;
      head->rx = hsb_getr(1 / res, cw, ch * thickness);
      head->ry = hsb_getr(1 / res, ch, cw * thickness);
      head->rz = hsb_getr(1 / res, thickness, cw * ch);
      head->capacitance = hsb_getcap(sh, thickness, cw * ch);
    } else {
      head->rx = 1 / ((1 / head->rx) + ((1 / hsb_getr(1 / res, cw, ch * thickness)) * occupancy));
      head->ry = 1 / ((1 / head->ry) + ((1 / hsb_getr(1 / res, ch, cw * thickness)) * occupancy));
      head->rz = 1 / ((1 / head->rz) + ((1 / hsb_getr(1 / res, thickness, cw * ch)) * occupancy));
      head->lock = 0;
    }
  }
  for (; head; head = head->next) tail = head;
  tail->next = new_blist(idx, occupancy, res, sh, first, d3, cw, ch, thickness);
  return tail->next ? HSB_OK : hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
}

static blist_t ***new_b2gmap(int rows, int cols)
{
  int i;
  blist_t ***b = calloc(rows, sizeof(blist_t **));
  if (!b) return NULL;
  b[0] = calloc((size_t)rows * cols, sizeof(blist_t *));
  if (!b[0]) return NULL;
  for (i = 1; i < rows; i++) b[i] = b[0] + (size_t)cols * i;
  return b;
}

static void reset_b2gmap(blist_t ***b, int rows, int cols)
{
  int i, j;
  for (i = 0; i < rows; i++)
    for (j = 0; j < cols; j++) {
      blist_t *p = b[i][j], *t;
      while (p) {
        t = p->next;
        free(p);
        p = t;
      }
      b[i][j] = NULL;
    }
}

static void delete_b2gmap(blist_t ***b, int rows, int cols)
{
  if (!b) return;
  reset_b2gmap(b, rows, cols);
  free(b[0]);
  free(b);
}

/* occupancy lists and block extents of one layer (set_bgmap,
 * temperature_grid.c:341-456) */
static int set_bgmap(grid_model_t *m, layer_t *layer)
{
  int i, j, u, i1, i2, j1, j2;
  const double cw = m->width / m->cols, ch = m->height / m->rows;
  const int d3 = m->config.detailed_3D_used;
  double sh, res;
  reset_b2gmap(layer->b2gmap, m->rows, m->cols);
  for (u = 0; u < layer->flp->n_units; u++) {
    const unit_t *U = &layer->flp->units[u];
    const double lu = U->leftx, ru = lu + U->width, bu = U->bottomy, tu = bu + U->height;
    i1 = m->rows - hsb_tolerant_ceil(tu / ch);
    i2 = m->rows - hsb_tolerant_floor(bu / ch);
    j1 = hsb_tolerant_floor(lu / cw);
    j2 = hsb_tolerant_ceil(ru / cw);
    if ((i1 < 0) || (j1 < 0)) return hsb_seterr(HSB_E_ARG, "negative grid cell start index!\n");
    if ((i2 > m->rows) || (j2 > m->cols))
      return hsb_seterr(HSB_E_ARG, "grid cell end index out of bounds!\n");
    if ((i1 >= i2) || (j1 >= j2))
      return hsb_seterr(HSB_E_ARG, "invalid floorplan spec or grid resolution\n");
    layer->g2bmap[u].i1 = i1;
    layer->g2bmap[u].i2 = i2;
    layer->g2bmap[u].j1 = j1;
    layer->g2bmap[u].j2 = j2;
    for (i = i1; i < i2; i++)
      for (j = j1; j < j2; j++) {
        res = (U->hasRes && d3) ? U->resistivity : 1 / layer->k;
        sh = (U->hasSh && d3) ? U->specificheat : layer->sp;
        if ((i > i1) && (i < i2 - 1) && (j > j1) && (j < j2 - 1)) {
          if (!layer->b2gmap[i][j]) {
            layer->b2gmap[i][j] = new_blist(u, 1.0, res, sh, 1, d3, cw, ch, layer->thickness);
            if (!layer->b2gmap[i][j]) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
            layer->b2gmap[i][j]->hasRes = 1;
            layer->b2gmap[i][j]->hasCap = U->hasSh;
          } else {
            CHECK(blist_append(layer->b2gmap[i][j], u, 1.0, res, sh, 1, d3, cw, ch, layer->thickness));
            hsb_warn("overlap of functional blocks?\n");
          }
        } else {
          const double lc = j * cw, rc = (j + 1) * cw;
          const double tc = m->height - i * ch, bc = m->height - (i + 1) * ch;
          double oh = (HSB_MIN(tu, tc) - HSB_MAX(bu, bc));
          double ow = (HSB_MIN(ru, rc) - HSB_MAX(lu, lc));
          double occ;
          if (hsb_eq(oh / ch, 0)) oh = 0;
          else if (hsb_eq(oh / ch, 1)) oh = ch;
          if (hsb_eq(ow / cw, 0)) ow = 0;
          else if (hsb_eq(ow / cw, 1)) ow = cw;
          occ = (oh * ow) / (ch * cw);
          if (oh < 0 || ow < 0) return hsb_seterr(HSB_E_ARG, "negative overlap!\n");
          if (!layer->b2gmap[i][j]) {
            layer->b2gmap[i][j] = new_blist(u, occ, res, sh, 1, d3, cw, ch, layer->thickness);
            if (!layer->b2gmap[i][j]) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
            layer->b2gmap[i][j]->hasRes = 1;
            layer->b2gmap[i][j]->hasCap = U->hasSh;
          } else {
            CHECK(blist_append(layer->b2gmap[i][j], u, occ, res, sh, 0, d3, cw, ch, layer->thickness));
          }
        }
      }
  }
  return HSB_OK;
}

/* ------------------------------------------------------------------------ */
/* per-model host extension and map ownership                                */
/* ------------------------------------------------------------------------ */
typedef struct hsb_owned {
  unsigned char own_b2g[HSB_MAX_LAYERS];
  unsigned char own_g2b[HSB_MAX_LAYERS];
  unsigned char own_flp[HSB_MAX_LAYERS];
} hsb_owned;

typedef struct ext_full {
  hsb_host_ext pub;
  hsb_owned own;
} ext_full;

static hsb_owned *owned(grid_model_t *m) { return &((ext_full *)m->ext)->own; }

static void default_opts(hsb_solver_opts *o)
{
  const char *f = getenv("HOTSPOT_B200_FORM");
  o->form = (f && !strcasecmp(f, "fast")) ? HSB_FORM_FAST : HSB_FORM_PARITY;
  o->steady_method = HSB_STEADY_AUTO;
  o->steady_tol = 0.0;
  o->max_iters = 0;
}

/* ------------------------------------------------------------------------ */
/* layers (temperature_grid.c:459-609 defaults/package, :612-833 LCF)        */
/* ------------------------------------------------------------------------ */
static void set_layer(layer_t *l, int no, int lateral, int power, double k, double t, double sp,
                      flp_t *flp)
{
  l->no = no;
  l->has_lateral = lateral;
  l->has_power = power;
  l->k = k;
  l->thickness = t;
  l->sp = sp;
  l->flp = flp;
}

static int default_layers(grid_model_t *m, flp_t *flp)
{
  int sil, itf, metal = 0, c4 = 0;
  const thermal_config_t *c = &m->config;
  if (!c->model_secondary) {
    sil = HSB_LAYER_SI;
    itf = HSB_LAYER_INT;
  } else {
    sil = HSB_SEC_PACK_LAYERS + HSB_SEC_CHIP_LAYERS + HSB_LAYER_SI;
    itf = HSB_SEC_PACK_LAYERS + HSB_SEC_CHIP_LAYERS + HSB_LAYER_INT;
    c4 = HSB_SEC_PACK_LAYERS + HSB_LAYER_C4;
    metal = HSB_SEC_PACK_LAYERS + HSB_LAYER_METAL;
  }
  set_layer(&m->layers[sil], sil, 1, 1, c->k_chip, c->t_chip, c->p_chip, flp);
  m->layers[sil].b2gmap = new_b2gmap(m->rows, m->cols);
  m->layers[sil].g2bmap = calloc(flp->n_units, sizeof(glist_t));
  if (!m->layers[sil].b2gmap || !m->layers[sil].g2bmap)
    return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  owned(m)->own_b2g[sil] = owned(m)->own_g2b[sil] = 1;
  set_layer(&m->layers[itf], itf, 1, 0, c->k_interface, c->t_interface, c->p_interface, flp);
  m->layers[itf].b2gmap = m->layers[sil].b2gmap;
  m->layers[itf].g2bmap = m->layers[sil].g2bmap;
  if (c->model_secondary) {
    set_layer(&m->layers[metal], metal, 1, 0, HSB_K_METAL, c->t_metal, HSB_SPEC_HEAT_METAL, flp);
    m->layers[metal].b2gmap = m->layers[sil].b2gmap;
    m->layers[metal].g2bmap = m->layers[sil].g2bmap;
    set_layer(&m->layers[c4], c4, 1, 0, HSB_K_C4, c->t_c4, HSB_SPEC_HEAT_C4, flp);
    m->layers[c4].b2gmap = m->layers[sil].b2gmap;
    m->layers[c4].g2bmap = m->layers[sil].g2bmap;
  }
  return HSB_OK;
}

static int append_package_layers(grid_model_t *m)
{
  const int nl = m->n_layers;
  const int sp = nl - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SP;
  const int hs = nl - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SINK;
  const thermal_config_t *c = &m->config;
  layer_t *L = m->layers;
  set_layer(&L[sp], sp, 1, 0, c->k_spreader, c->t_spreader, c->p_spreader, L[sp - 1].flp);
  L[sp].b2gmap = L[sp - 1].b2gmap;
  L[sp].g2bmap = L[sp - 1].g2bmap;
  set_layer(&L[hs], hs, 1, 0, c->k_sink, c->t_sink, c->p_sink, L[sp - 1].flp);
  L[hs].b2gmap = L[sp - 1].b2gmap;
  L[hs].g2bmap = L[sp - 1].g2bmap;
  if (c->detailed_3D_used) {
    L[sp].b2gmap = new_b2gmap(m->rows, m->cols);
    if (!L[sp].b2gmap) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
    owned(m)->own_b2g[sp] = 1;
    L[hs].b2gmap = L[sp].b2gmap;
  }
  if (c->model_secondary) {
    const int sil = m->has_lcf ? HSB_SEC_PACK_LAYERS
                               : HSB_SEC_PACK_LAYERS + HSB_SEC_CHIP_LAYERS + HSB_LAYER_SI;
    const int sub = HSB_LAYER_SUB, sol = HSB_LAYER_SOLDER, pcb = HSB_LAYER_PCB;
    set_layer(&L[sub], sub, 1, 0, HSB_K_SUB, c->t_sub, HSB_SPEC_HEAT_SUB, L[sil].flp);
    L[sub].b2gmap = L[sil].b2gmap;
    L[sub].g2bmap = L[sil].g2bmap;
    set_layer(&L[sol], sol, 1, 0, HSB_K_SOLDER, c->t_solder, HSB_SPEC_HEAT_SOLDER, L[sil].flp);
    L[sol].b2gmap = L[sil].b2gmap;
    L[sol].g2bmap = L[sil].g2bmap;
    set_layer(&L[pcb], pcb, 1, 0, HSB_K_PCB, c->t_pcb, HSB_SPEC_HEAT_PCB, L[sil].flp);
    L[pcb].b2gmap = L[sil].b2gmap;
    L[pcb].g2bmap = L[sil].g2bmap;
    if (c->detailed_3D_used) {
      L[sub].b2gmap = new_b2gmap(m->rows, m->cols);
      if (!L[sub].b2gmap) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
      owned(m)->own_b2g[sub] = 1;
      L[sol].b2gmap = L[sub].b2gmap;
      L[pcb].b2gmap = L[sub].b2gmap;
    }
  }
  return HSB_OK;
}

enum { F_SNO, F_LATERAL, F_POWER, F_SP, F_RHO, F_THICK, F_FLP };

/* next non-comment first token of the file, or NULL at EOF */
static char *lcf_token(FILE *fp, char *line, size_t n)
{
  char *p;
  while (fgets(line, (int)n, fp)) {
    p = strtok(line, " \r\t\n");
    if (!p || p[0] == '#') continue;
    return p;
  }
  return NULL;
}

/* count_num_layers (temperature_grid.c:755-833) */
static int count_lcf_layers(FILE *fp, int *out)
{
  char line[HSB_LINE_SIZE], sval[HSB_STR_SIZE], c, *p;
  int field = F_SNO, n = 0, iv;
  double dv;
  fseek(fp, 0, SEEK_SET);
  while ((p = lcf_token(fp, line, sizeof(line)))) {
    switch (field) {
      case F_SNO:
        if (sscanf(p, "%d", &iv) != 1) return hsb_seterr(HSB_E_ARG, "invalid layer number\n");
        field = F_LATERAL;
        break;
      case F_LATERAL:
        if (sscanf(p, "%c", &c) != 1) return hsb_seterr(HSB_E_ARG, "invalid layer heat flow indicator\n");
        field = F_POWER;
        break;
      case F_POWER:
        if (sscanf(p, "%c", &c) != 1)
          return hsb_seterr(HSB_E_ARG, "invalid layer power dissipation indicator\n");
        field = F_SP;
        break;
      case F_SP:
        if (sscanf(p, "%lf", &dv) != 1) {
          if (sscanf(p, "%s", sval) != 1)
            return hsb_seterr(HSB_E_ARG, "invalid: neither specific heat nor material name was specified\n");
          field = F_THICK;
        } else {
          field = F_RHO;
        }
        break;
      case F_RHO:
        if (sscanf(p, "%lf", &dv) != 1) return hsb_seterr(HSB_E_ARG, "invalid resistivity\n");
        field = F_THICK;
        break;
      case F_THICK:
        if (sscanf(p, "%lf", &dv) != 1) return hsb_seterr(HSB_E_ARG, "invalid thickness\n");
        field = F_FLP;
        break;
      default:
        if (sscanf(p, "%s", sval) != 1) return hsb_seterr(HSB_E_ARG, "invalid floorplan file");
        n++;
        field = F_SNO;
        break;
    }
  }
  *out = n;
  return HSB_OK;
}

/* parse_layer_file (temperature_grid.c:612-752) */
static int parse_lcf(grid_model_t *m, FILE *fp, const materials_list_t *ml)
{
  char line[HSB_LINE_SIZE], cval, *p;
  int count = 0, i = 0, field = F_SNO, ival, base, inner;
  double dval;
  if (!m->config.model_secondary) {
    base = 0;
    inner = m->n_layers - HSB_DEFAULT_PACK_LAYERS;
  } else {
    base = HSB_SEC_PACK_LAYERS;
    inner = m->n_layers - HSB_DEFAULT_PACK_LAYERS - HSB_SEC_PACK_LAYERS;
  }
  fseek(fp, 0, SEEK_SET);
  while ((p = lcf_token(fp, line, sizeof(line)))) {
    switch (field) {
      case F_SNO:
        if (sscanf(p, "%d", &ival) != 1) return hsb_seterr(HSB_E_ARG, "invalid layer number\n");
        if (ival >= inner || ival < 0)
          return hsb_seterr(HSB_E_ARG, "layer number must be >= 0 and < no. of layers specified\n");
        if (m->layers[base + ival].no != 0) return hsb_seterr(HSB_E_ARG, "layer numbers must be unique\n");
        i = base + ival;
        m->layers[i].no = base + ival;
        field = F_LATERAL;
        break;
      case F_LATERAL:
        if (sscanf(p, "%c", &cval) != 1) return hsb_seterr(HSB_E_ARG, "invalid layer heat flow indicator\n");
        if (cval == 'Y' || cval == 'y') m->layers[i].has_lateral = 1;
        else if (cval == 'N' || cval == 'n') m->layers[i].has_lateral = 0;
        else return hsb_seterr(HSB_E_ARG, "invalid layer heat flow indicator\n");
        field = F_POWER;
        break;
      case F_POWER:
        if (sscanf(p, "%c", &cval) != 1)
          return hsb_seterr(HSB_E_ARG, "invalid layer power dissipation indicator\n");
        if (cval == 'Y' || cval == 'y') m->layers[i].has_power = 1;
        else if (cval == 'N' || cval == 'n') m->layers[i].has_power = 0;
        else return hsb_seterr(HSB_E_ARG, "invalid layer power dissipation indicator\n");
        field = F_SP;
        break;
      case F_SP:
        if (sscanf(p, "%lf", &dval) != 1) {
          char mat[HSB_STR_SIZE];
          if (sscanf(p, "%s", mat) != 1)
            return hsb_seterr(HSB_E_ARG, "invalid: neither specific heat nor material name was specified\n");
          m->layers[i].sp = hsb_material_cv(ml, mat);
          m->layers[i].k = hsb_material_k(ml, mat);
          field = F_THICK;
        } else {
          m->layers[i].sp = dval;
          field = F_RHO;
        }
        break;
      case F_RHO:
        if (sscanf(p, "%lf", &dval) != 1) return hsb_seterr(HSB_E_ARG, "invalid resistivity\n");
        m->layers[i].k = 1.0 / dval;
        field = F_THICK;
        break;
      case F_THICK:
        if (sscanf(p, "%lf", &dval) != 1) return hsb_seterr(HSB_E_ARG, "invalid thickness\n");
        m->layers[i].thickness = dval;
        field = F_FLP;
        break;
      default: /* F_FLP */
        if (strstr(p, ".csv") && m->use_microchannels) {
          microchannel_config_t *u = calloc(1, sizeof(microchannel_config_t));
          const microchannel_config_t *d = m->default_microchannel_config;
          if (!u) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
          if (!d) return hsb_seterr(HSB_E_ARG, "microchannel layer without a microchannel configuration\n");
          m->layers[i].is_microchannel = 1;
          m->layers[i].microchannel_config = u;
          /* copy_microchannel (microchannel.c:573-583) */
          u->pumping_pressure = d->pumping_pressure;
          u->pump_internal_res = d->pump_internal_res;
          u->inlet_temperature = d->inlet_temperature;
          u->coolant_capac = d->coolant_capac;
          u->coolant_res = d->coolant_res;
          u->coolant_visc = d->coolant_visc;
          u->wall_capac = d->wall_capac;
          u->wall_res = d->wall_res;
          u->htc = d->htc;
          u->cell_width = m->width / m->cols;
          u->cell_height = m->height / m->rows;
          u->cell_thickness = m->layers[i].thickness;
          u->num_rows = m->rows;
          u->num_columns = m->cols;
          strncpy(u->network_file, p, HSB_STR_SIZE - 1);
          CHECK(hsb_uchan_build(u, &m->layers[i].flp));
        } else if (strstr(p, ".csv") && !m->use_microchannels) {
          return hsb_seterr(HSB_E_ARG, "Floorplan file has microchannel extension but use_microchannels = 0\n");
        } else {
          CHECK(hsb_read_flp_file(p, &m->layers[i].flp));
          m->layers[i].is_microchannel = 0;
        }
        owned(m)->own_flp[i] = 1;
        if (count < 7) {
          m->width = hsb_flp_width(m->layers[i].flp);
          m->height = hsb_flp_height(m->layers[i].flp);
        } else if (!hsb_eq(m->width, hsb_flp_width(m->layers[i].flp)) ||
                   !hsb_eq(m->height, hsb_flp_height(m->layers[i].flp))) {
          return hsb_seterr(HSB_E_ARG, "width and height differ across layers\n");
        }
        field = F_SNO;
        break;
    }
    count++;
  }
  for (i = base; i < base + inner; i++) {
    if (!m->layers[i].flp) return hsb_seterr(HSB_E_ARG, "layer %d has no floorplan\n", i);
    m->layers[i].b2gmap = new_b2gmap(m->rows, m->cols);
    m->layers[i].g2bmap = calloc(m->layers[i].flp->n_units, sizeof(glist_t));
    if (!m->layers[i].b2gmap || !m->layers[i].g2bmap) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
    owned(m)->own_b2g[i] = owned(m)->own_g2b[i] = 1;
  }
  return HSB_OK;
}

static int populate_layers(grid_model_t *m, flp_t *flp_default, const materials_list_t *ml)
{
  FILE *fp = NULL;
  int n = 0, rc = HSB_OK;
  if (m->has_lcf) {
    fp = !strcasecmp(m->config.grid_layer_file, "stdin") ? stdin : fopen(m->config.grid_layer_file, "r");
    if (!fp) return hsb_seterr(HSB_E_ARG, "Unable to open file %s\n", m->config.grid_layer_file);
    if ((rc = count_lcf_layers(fp, &n))) goto out;
    m->n_layers = n;
  } else {
    m->n_layers = HSB_DEFAULT_CHIP_LAYERS + (m->config.model_secondary ? HSB_SEC_CHIP_LAYERS : 0);
  }
  m->n_layers += HSB_DEFAULT_PACK_LAYERS + (m->config.model_secondary ? HSB_SEC_PACK_LAYERS : 0);
  if (m->n_layers > HSB_MAX_LAYERS) {
    rc = hsb_seterr(HSB_E_ARG, "at most %d layers are supported\n", HSB_MAX_LAYERS);
    goto out;
  }
  m->layers = calloc(m->n_layers, sizeof(layer_t));
  if (!m->layers) {
    rc = hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
    goto out;
  }
  if (m->has_lcf) rc = parse_lcf(m, fp, ml);
  else if (!flp_default) rc = hsb_seterr(HSB_E_ARG, "Either LCF or FLP file must be specified\n");
  else rc = default_layers(m, flp_default);
  if (!rc) rc = append_package_layers(m);
out:
  if (fp && fp != stdin) fclose(fp);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* conductances (find_res, temperature_grid.c:26-186)                        */
/* ------------------------------------------------------------------------ */
static double res3(grid_model_t *m, int n, int i, int j, int choice)
{
  const blist_t *b = m->layers[n].b2gmap ? m->layers[n].b2gmap[i][j] : NULL;
  const int has = b ? b->hasRes : 0;
  if (choice == 1) return has ? b->rx : m->layers[n].rx;
  if (choice == 2) return has ? b->ry : m->layers[n].ry;
  return has ? b->rz : m->layers[n].rz;
}

static int fluid_at(grid_model_t *m, int n, int i, int j)
{
  const microchannel_config_t *u = m->layers[n].microchannel_config;
  return m->layers[n].is_microchannel && FLUID_CELL_TYPE(u->cell_types[i][j]);
}

double hsb_find_res(grid_model_t *m, int n1, int i1, int j1, int n2, int i2, int j2)
{
  double htc = 0.0;
  const double cw = m->width / m->cols, ch = m->height / m->rows;
  int f1 = 0, f2 = 0;
  if (m->layers[n1].is_microchannel) {
    htc = m->layers[n1].microchannel_config->htc;
    f1 = fluid_at(m, n1, i1, j1);
  }
  if (m->layers[n2].is_microchannel) {
    htc = m->layers[n2].microchannel_config->htc;
    f2 = fluid_at(m, n2, i2, j2);
  }
  if ((f1 && !f2) || (!f1 && f2)) {
    if (n1 == 0) return res3(m, n1, i1, j1, 3) + (1.0 / (htc * ch * cw)) + 0;
    if (n2 == 0) return res3(m, n2, i2, j2, 3) + (1.0 / (htc * ch * cw)) + 0;
    if (n1 != n2 && i1 == i2 && j1 == j2)
      return f1 ? (res3(m, n2, i2, j2, 3) / 2.0) + (1.0 / (htc * ch * cw)) + 0
                : (res3(m, n1, i1, j1, 3) / 2.0) + (1.0 / (htc * ch * cw)) + 0;
    if (n1 == n2 && i1 != i2 && j1 == j2)
      return f1 ? (res3(m, n2, i2, j2, 1) / 2.0) + (1.0 / (htc * cw * m->layers[n1].thickness))
                : (res3(m, n1, i1, j1, 1) / 2.0) + (1.0 / (htc * cw * m->layers[n2].thickness));
    if (n1 == n2 && i1 == i2 && j1 != j2)
      return f1 ? (res3(m, n2, i2, j2, 2) / 2.0) + (1.0 / (htc * ch * m->layers[n1].thickness))
                : (res3(m, n1, i1, j1, 2) / 2.0) + (1.0 / (htc * ch * m->layers[n2].thickness));
    return -1.0;
  }
  if (m->config.detailed_3D_used == 1) {
    if (n1 == 0 && i1 == i2 && j1 == j2) return res3(m, n1, i1, j1, 3) + (res3(m, n2, i2, j2, 3) / 2.0);
    if (n2 == 0 && i1 == i2 && j1 == j2) return res3(m, n2, i2, j2, 3) + (res3(m, n1, i1, j1, 3) / 2.0);
    if (n1 != n2 && i1 == i2 && j1 == j2) return (res3(m, n1, i1, j1, 3) / 2.0) + (res3(m, n2, i2, j2, 3) / 2.0);
    if (n1 == n2 && i1 != i2 && j1 == j2) return (res3(m, n1, i1, j1, 1) / 2.0) + (res3(m, n2, i2, j2, 1) / 2.0);
    if (n1 == n2 && i1 == i2 && j1 != j2) return (res3(m, n1, i1, j1, 2) / 2.0) + (res3(m, n2, i2, j2, 2) / 2.0);
    return -1.0;
  }
  if (n1 < n2 && i1 == i2 && j1 == j2) return m->layers[n1].rz;
  if (n1 > n2 && i1 == i2 && j1 == j2) return m->layers[n2].rz;
  if (n1 == n2 && i1 != i2 && j1 == j2) return (m->layers[n1].rx / 2.0) + (m->layers[n2].rx / 2.0);
  if (n1 == n2 && i1 == i2 && j1 != j2) return (m->layers[n1].ry / 2.0) + (m->layers[n2].ry / 2.0);
  return -1.0;
}

static double cap3(grid_model_t *m, int n, int i, int j)
{
  const blist_t *b = m->layers[n].b2gmap ? m->layers[n].b2gmap[i][j] : NULL;
  return (b && b->lock == 1) ? b->capacitance : m->layers[n].c;
}

/* ------------------------------------------------------------------------ */
/* device upload                                                             */
/* ------------------------------------------------------------------------ */
static int upload_layers(grid_model_t *m)
{
  double rx[HSB_MAX_LAYERS], ry[HSB_MAX_LAYERS], rz[HSB_MAX_LAYERS], c[HSB_MAX_LAYERS];
  int n;
  for (n = 0; n < m->n_layers; n++) {
    rx[n] = m->layers[n].rx;
    ry[n] = m->layers[n].ry;
    rz[n] = m->layers[n].rz;
    c[n] = m->layers[n].c;
  }
  if (hsb_dev_set_layers(m->dev, rx, ry, rz, c, (const double *)&m->pack, m->config.ambient, m->width,
                         m->height, m->config.r_convec_sec * (m->config.s_pcb * m->config.s_pcb)))
    return hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error());
  return HSB_OK;
}

static int upload_maps(grid_model_t *m)
{
  const int nl = m->n_layers, nr = m->rows, nc = m->cols;
  const long long ncell = (long long)nl * nr * nc;
  long long nnz = 0, c;
  int n, i, j, u, base = 0, rc;
  int *ptr = malloc(sizeof(int) * (ncell + 1)), *blk, *g2b;
  double *occ, *area;
  if (!ptr) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  c = 0;
  for (n = 0; n < nl; n++)
    for (i = 0; i < nr; i++)
      for (j = 0; j < nc; j++, c++) {
        ptr[c] = (int)nnz;
        for (const blist_t *b = m->layers[n].b2gmap[i][j]; b; b = b->next) nnz++;
      }
  ptr[ncell] = (int)nnz;
  blk = malloc(sizeof(int) * (nnz + 1));
  occ = malloc(sizeof(double) * (nnz + 1));
  area = malloc(sizeof(double) * (nnz + 1));
  g2b = malloc(sizeof(int) * 5 * (m->total_n_blocks + 1));
  if (!blk || !occ || !area || !g2b) {
    free(ptr); free(blk); free(occ); free(area); free(g2b);
    return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  }
  c = 0;
  nnz = 0;
  for (n = 0; n < nl; n++) {
    const flp_t *f = m->layers[n].flp;
    for (i = 0; i < nr; i++)
      for (j = 0; j < nc; j++, c++)
        for (const blist_t *b = m->layers[n].b2gmap[i][j]; b; b = b->next, nnz++) {
          blk[nnz] = base + b->idx;
          occ[nnz] = b->occupancy;
          area[nnz] = f->units[b->idx].width * f->units[b->idx].height;
        }
    for (u = 0; u < f->n_units; u++) {
      int *g = g2b + 5 * (base + u);
      g[0] = n;
      g[1] = m->layers[n].g2bmap[u].i1;
      g[2] = m->layers[n].g2bmap[u].i2;
      g[3] = m->layers[n].g2bmap[u].j1;
      g[4] = m->layers[n].g2bmap[u].j2;
    }
    base += f->n_units;
  }
  rc = hsb_dev_set_maps(m->dev, ptr, blk, occ, area,
                        (m->width * m->height) / (m->cols * m->rows), g2b);
  free(ptr); free(blk); free(occ); free(area); free(g2b);
  return rc ? hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error()) : HSB_OK;
}

/* per-cell resistances as the slope/GS macros see them: find_res(neighbour, cell) */
static int upload_cells(grid_model_t *m, int with_cap)
{
  const int nl = m->n_layers, nr = m->rows, nc = m->cols;
  const size_t N = (size_t)nl * nr * nc;
  double *a = calloc(7 * N, sizeof(double));
  int n, i, j, rc;
  size_t c = 0;
  if (!a) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  for (n = 0; n < nl; n++)
    for (i = 0; i < nr; i++)
      for (j = 0; j < nc; j++, c++) {
        if (i > 0) a[c] = hsb_find_res(m, n, i - 1, j, n, i, j);
        if (i < nr - 1) a[N + c] = hsb_find_res(m, n, i + 1, j, n, i, j);
        if (j > 0) a[2 * N + c] = hsb_find_res(m, n, i, j - 1, n, i, j);
        if (j < nc - 1) a[3 * N + c] = hsb_find_res(m, n, i, j + 1, n, i, j);
        if (n > 0) a[4 * N + c] = hsb_find_res(m, n - 1, i, j, n, i, j);
        if (n < nl - 1) a[5 * N + c] = hsb_find_res(m, n + 1, i, j, n, i, j);
        a[6 * N + c] = with_cap ? cap3(m, n, i, j) : 1.0;
      }
  rc = hsb_dev_set_cells(m->dev, a, a + N, a + 2 * N, a + 3 * N, a + 4 * N, a + 5 * N, a + 6 * N);
  free(a);
  return rc ? hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error()) : HSB_OK;
}

/* microchannel advection per cell (slope_fn_grid, temperature_grid.c:3256-3590) */
static int upload_advection(grid_model_t *m)
{
  const int nl = m->n_layers, nr = m->rows, nc = m->cols;
  const size_t N = (size_t)nl * nr * nc;
  int n, i, j, any = 0, rc;
  double *a;
  for (n = 0; n < nl; n++) any |= m->layers[n].is_microchannel;
  if (!any) return HSB_OK;
  a = calloc(6 * N, sizeof(double));
  if (!a) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  for (n = 0; n < nl; n++) {
    const microchannel_config_t *u = m->layers[n].microchannel_config;
    if (!m->layers[n].is_microchannel) continue;
    for (i = 0; i < nr; i++)
      for (j = 0; j < nc; j++) {
        const size_t c = ((size_t)n * nr + i) * nc + j;
        const double Cv = u->coolant_capac;
#define FL(ii, jj) FLUID_CELL_TYPE(u->cell_types[ii][jj])
        if (!FL(i, j)) continue;
        if (i > 0 && FL(i - 1, j)) a[c] = Cv * hsb_uchan_flow(u, i - 1, j, i, j);
        if (i < nr - 1 && FL(i + 1, j)) a[N + c] = Cv * hsb_uchan_flow(u, i + 1, j, i, j);
        if (j > 0 && FL(i, j - 1)) a[2 * N + c] = Cv * hsb_uchan_flow(u, i, j - 1, i, j);
        if (j < nc - 1 && FL(i, j + 1)) a[3 * N + c] = Cv * hsb_uchan_flow(u, i, j + 1, i, j);
        if (u->cell_types[i][j] == HSB_INLET || u->cell_types[i][j] == HSB_OUTLET) {
          /* neighbour order per boundary side as :3318-3445 / :3460-3580 */
          double rate = 0;
          if (i == 0) {
            if (j > 0 && FL(i, j - 1)) rate += hsb_uchan_flow(u, i, j - 1, i, j);
            if (j < nc - 1 && FL(i, j + 1)) rate += hsb_uchan_flow(u, i, j + 1, i, j);
            if (i < nr - 1 && FL(i + 1, j)) rate += hsb_uchan_flow(u, i + 1, j, i, j);
          } else if (i == nr - 1) {
            if (j > 0 && FL(i, j - 1)) rate += hsb_uchan_flow(u, i, j - 1, i, j);
            if (j < nc - 1 && FL(i, j + 1)) rate += hsb_uchan_flow(u, i, j + 1, i, j);
            if (i > 0 && FL(i - 1, j)) rate += hsb_uchan_flow(u, i - 1, j, i, j);
          } else if (j == 0) {
            if (j < nc - 1 && FL(i, j + 1)) rate += hsb_uchan_flow(u, i, j + 1, i, j);
            if (i > 0 && FL(i - 1, j)) rate += hsb_uchan_flow(u, i - 1, j, i, j);
            if (i < nr - 1 && FL(i + 1, j)) rate += hsb_uchan_flow(u, i + 1, j, i, j);
          } else if (j == nc - 1) {
            if (j > 0 && FL(i, j - 1)) rate += hsb_uchan_flow(u, i, j - 1, i, j);
            if (i > 0 && FL(i - 1, j)) rate += hsb_uchan_flow(u, i - 1, j, i, j);
            if (i < nr - 1 && FL(i + 1, j)) rate += hsb_uchan_flow(u, i + 1, j, i, j);
          }
          rate *= -1;
          if (u->cell_types[i][j] == HSB_INLET) a[5 * N + c] = u->coolant_capac * rate * u->inlet_temperature;
          else a[4 * N + c] = u->coolant_capac * rate;
        }
#undef FL
      }
  }
  rc = hsb_dev_set_advection(m->dev, a, a + N, a + 2 * N, a + 3 * N, a + 4 * N, a + 5 * N);
  free(a);
  return rc ? hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error()) : HSB_OK;
}

/* ------------------------------------------------------------------------ */
/* status-returning implementations                                          */
/* ------------------------------------------------------------------------ */
static void free_model_host(grid_model_t *m)
{
  int i;
  if (!m) return;
  if (m->layers) {
    for (i = 0; i < m->n_layers; i++) {
      if (m->ext && owned(m)->own_b2g[i]) delete_b2gmap(m->layers[i].b2gmap, m->rows, m->cols);
      if (m->ext && owned(m)->own_g2b[i]) free(m->layers[i].g2bmap);
      if (m->ext && owned(m)->own_flp[i]) hsb_free_flp(m->layers[i].flp);
      if (m->layers[i].is_microchannel) hsb_uchan_free(m->layers[i].microchannel_config);
    }
    free(m->layers);
  }
  if (m->last_steady) {
    hsb_free_dcuboid(m->last_steady->cuboid);
    free(m->last_steady);
  }
  if (m->last_trans) {
    hsb_free_dcuboid(m->last_trans->cuboid);
    free(m->last_trans);
  }
  if (m->dev) hsb_dev_destroy(m->dev);
  free(m->ext);
  free(m);
}

int hsb_grid_alloc(grid_model_t **out, thermal_config_t *config, flp_t *flp_default,
                   microchannel_config_t *uconf, materials_list_t *ml, int do_detailed_3D,
                   int use_microchannels)
{
  grid_model_t *m;
  int i, rc;
  *out = NULL;
  if (!config) return hsb_seterr(HSB_E_ARG, "null configuration\n");
  if (config->grid_rows & (config->grid_rows - 1) || config->grid_cols & (config->grid_cols - 1) ||
      config->grid_rows <= 0 || config->grid_cols <= 0)
    return hsb_seterr(HSB_E_ARG, "grid rows and columns should both be powers of two\n");
  m = calloc(1, sizeof(grid_model_t));
  if (!m) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  m->ext = calloc(1, sizeof(ext_full));
  if (!m->ext) {
    free(m);
    return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  }
  default_opts(&m->ext->opts);
  m->config = *config;
  m->rows = config->grid_rows;
  m->cols = config->grid_cols;
  m->use_microchannels = use_microchannels;
  m->default_microchannel_config = uconf;
  if (do_detailed_3D) m->config.detailed_3D_used = 1;
  if (!strcasecmp(m->config.grid_map_mode, "avg")) m->map_mode = HSB_GRID_AVG;
  else if (!strcasecmp(m->config.grid_map_mode, "min")) m->map_mode = HSB_GRID_MIN;
  else if (!strcasecmp(m->config.grid_map_mode, "max")) m->map_mode = HSB_GRID_MAX;
  else if (!strcasecmp(m->config.grid_map_mode, "center")) m->map_mode = HSB_GRID_CENTER;
  else {
    free_model_host(m);
    return hsb_seterr(HSB_E_ARG, "unknown mapping mode\n");
  }
  if (strcmp(m->config.grid_layer_file, HSB_NULLFILE)) {
    m->has_lcf = 1;
  } else {
    m->has_lcf = 0;
    if (!flp_default) {
      free_model_host(m);
      return hsb_seterr(HSB_E_ARG, "Either LCF or FLP file must be specified\n");
    }
    m->base_n_units = flp_default->n_units;
  }
  if ((rc = populate_layers(m, flp_default, ml))) {
    free_model_host(m);
    return rc;
  }
  m->total_n_blocks = 0;
  for (i = 0; i < m->n_layers; i++) m->total_n_blocks += m->layers[i].flp->n_units;
  m->last_steady = calloc(1, sizeof(grid_model_vector_t));
  m->last_trans = calloc(1, sizeof(grid_model_vector_t));
  m->last_steady->cuboid = hsb_dcuboid_tail(m->rows, m->cols, m->n_layers, n_extra(m));
  m->last_trans->cuboid = hsb_dcuboid_tail(m->rows, m->cols, m->n_layers, n_extra(m));
  if (!m->last_steady->cuboid || !m->last_trans->cuboid) {
    free_model_host(m);
    return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  }
  m->last_steady->extra = m->last_steady->cuboid[0][0] + (size_t)m->rows * m->cols * m->n_layers;
  m->last_trans->extra = m->last_trans->cuboid[0][0] + (size_t)m->rows * m->cols * m->n_layers;
  {
    hsb_grid_desc d;
    int any_uc = 0;
    memset(&d, 0, sizeof(d));
    d.nl = m->n_layers;
    d.nr = m->rows;
    d.nc = m->cols;
    d.n_extra = n_extra(m);
    d.spidx = m->n_layers - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SP;
    d.hsidx = m->n_layers - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SINK;
    d.subidx = m->config.model_secondary ? HSB_LAYER_SUB : -1;
    d.solderidx = m->config.model_secondary ? HSB_LAYER_SOLDER : -1;
    d.pcbidx = m->config.model_secondary ? HSB_LAYER_PCB : -1;
    for (i = 0; i < m->n_layers; i++) any_uc |= m->layers[i].is_microchannel;
    d.field = m->config.detailed_3D_used || any_uc;
    d.map_mode = m->map_mode;
    d.total_n_blocks = m->total_n_blocks;
    d.ambient = m->config.ambient;
    if (hsb_dev_create(&m->dev, &d)) {
      rc = hsb_seterr(HSB_E_CUDA, "libhotspot_b200: %s\n", hsb_dev_last_error());
      free_model_host(m);
      return rc;
    }
  }
  *out = m;
  return HSB_OK;
}

static void silidx_info(const grid_model_t *m, int *base, int *inner, int *sil)
{
  const int nl = m->n_layers;
  if (m->config.model_secondary) {
    if (m->has_lcf) {
      *base = HSB_SEC_PACK_LAYERS;
      *inner = nl - HSB_DEFAULT_PACK_LAYERS - HSB_SEC_PACK_LAYERS;
      *sil = HSB_SEC_PACK_LAYERS + HSB_LAYER_SI;
    } else {
      *base = HSB_SEC_CHIP_LAYERS + HSB_SEC_PACK_LAYERS;
      *inner = nl - HSB_DEFAULT_PACK_LAYERS - HSB_SEC_PACK_LAYERS - HSB_SEC_CHIP_LAYERS;
      *sil = HSB_SEC_PACK_LAYERS + HSB_SEC_CHIP_LAYERS + HSB_LAYER_SI;
    }
  } else {
    *base = 0;
    *inner = nl - HSB_DEFAULT_PACK_LAYERS;
    *sil = HSB_LAYER_SI;
  }
}

/* populate_R_model_grid (temperature_grid.c:950-1062) */
int hsb_grid_populate_R(grid_model_t *m, flp_t *flp)
{
  int i, base, inner, sil, hs, ii, jj, any_uc = 0;
  double cw, ch;
  const int nl = m->n_layers;
  silidx_info(m, &base, &inner, &sil);
  if (m->has_lcf) {
    for (i = base; i < base + inner; i++) CHECK(set_bgmap(m, &m->layers[i]));
  } else {
    if (flp != m->layers[sil].flp) return hsb_seterr(HSB_E_ARG, "mismatch between the floorplan and the thermal model\n");
    m->width = hsb_flp_width(flp);
    m->height = hsb_flp_height(flp);
    CHECK(set_bgmap(m, &m->layers[sil]));
  }
  if (m->config.detailed_3D_used) {
    const int sp = nl - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SP;
    CHECK(set_bgmap(m, &m->layers[sp]));
    for (ii = 0; ii < m->rows; ii++)
      for (jj = 0; jj < m->cols; jj++)
        if (m->layers[sp].b2gmap[ii][jj]) {
          m->layers[sp].b2gmap[ii][jj]->hasRes = 0;
          m->layers[sp].b2gmap[ii][jj]->hasCap = 0;
          m->layers[sp].b2gmap[ii][jj]->lock = 0;
        }
    if (m->config.model_secondary) {
      CHECK(set_bgmap(m, &m->layers[HSB_LAYER_SUB]));
      for (ii = 0; ii < m->rows; ii++)
        for (jj = 0; jj < m->cols; jj++)
          if (m->layers[HSB_LAYER_SUB].b2gmap[ii][jj]) {
            m->layers[HSB_LAYER_SUB].b2gmap[ii][jj]->hasRes = 0;
            m->layers[HSB_LAYER_SUB].b2gmap[ii][jj]->hasCap = 0;
            m->layers[HSB_LAYER_SUB].b2gmap[ii][jj]->lock = 0;
          }
    }
  }
  if (m->width > m->config.s_sink || m->height > m->config.s_sink || m->width > m->config.s_spreader ||
      m->height > m->config.s_spreader)
    return hsb_seterr(HSB_E_ARG, "inordinate floorplan size!\n");
  cw = m->width / m->cols;
  ch = m->height / m->rows;
  hsb_package_R(&m->pack, &m->config, m->width, m->height);
  hs = nl - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SINK;
  for (i = 0; i < nl; i++) {
    layer_t *L = &m->layers[i];
    if (L->has_lateral) {
      L->rx = hsb_getr(L->k, cw, ch * L->thickness);
      L->ry = hsb_getr(L->k, ch, cw * L->thickness);
    } else {
      L->rx = HSB_LARGENUM;
      L->ry = HSB_LARGENUM;
    }
    L->rz = hsb_getr(L->k, L->thickness, cw * ch);
    if (i == hs) L->rz += m->config.r_convec * (m->config.s_sink * m->config.s_sink) / (cw * ch);
    any_uc |= L->is_microchannel;
  }
  m->r_ready = 1;
  CHECK(upload_layers(m));
  CHECK(upload_maps(m));
  if (m->config.detailed_3D_used || any_uc) CHECK(upload_cells(m, m->c_ready));
  CHECK(upload_advection(m));
  return HSB_OK;
}

/* populate_C_model_grid (temperature_grid.c:1065-1114) */
int hsb_grid_populate_C(grid_model_t *m, flp_t *flp)
{
  int i, base, inner, sil, any_uc = 0;
  const double cw = m->width / m->cols, ch = m->height / m->rows;
  const int nl = m->n_layers, hs = nl - HSB_DEFAULT_PACK_LAYERS + HSB_LAYER_SINK;
  silidx_info(m, &base, &inner, &sil);
  if (!m->r_ready) return hsb_seterr(HSB_E_ARG, "R model not ready\n");
  if (!m->has_lcf && flp != m->layers[sil].flp)
    return hsb_seterr(HSB_E_ARG, "different floorplans for R and C models!\n");
  hsb_package_C(&m->pack, &m->config, m->width, m->height);
  for (i = 0; i < nl; i++) {
    m->layers[i].c = hsb_getcap(m->layers[i].sp, m->layers[i].thickness, cw * ch);
    any_uc |= m->layers[i].is_microchannel;
  }
  m->layers[hs].c += HSB_C_FACTOR * m->config.c_convec * (cw * ch) / (m->config.s_sink * m->config.s_sink);
  if (m->config.model_secondary)
    m->layers[HSB_LAYER_PCB].c +=
        HSB_C_FACTOR * m->config.c_convec_sec * (cw * ch) / (m->config.s_pcb * m->config.s_pcb);
  m->c_ready = 1;
  CHECK(upload_layers(m));
  if (m->config.detailed_3D_used || any_uc) CHECK(upload_cells(m, 1));
  return HSB_OK;
}

/* set_internal_power_grid (temperature_grid.c:2018-2024): the caller's
 * package-node power entries are zeroed, as the reference does */
static void zero_internal_power(grid_model_t *m, double *power)
{
  memset(&power[m->total_n_blocks], 0, sizeof(double) * n_extra(m));
}

int hsb_grid_compute_temp(grid_model_t *m, double *power, double *temp, double time_elapsed)
{
  if (!m->r_ready || !m->c_ready) return hsb_seterr(HSB_E_ARG, "grid model not ready\n");
  zero_internal_power(m, power);
  if (temp) m->last_temp = temp;
  if (!m->last_temp)
    return hsb_seterr(HSB_E_ARG, "compute_temp: the first call must pass a temperature vector\n");
  memset(&m->ext->last, 0, sizeof(hsb_stats));
  if (hsb_dev_transient(m->dev, power, temp, time_elapsed, m->last_temp, &m->ext->opts, &m->ext->last))
    return hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error());
  m->ext->host_trans_valid = 0;
  return HSB_OK;
}

int hsb_grid_steady(grid_model_t *m, double *power, double *temp)
{
  if (!m->r_ready) return hsb_seterr(HSB_E_ARG, "R model not ready\n");
  zero_internal_power(m, power);
  memset(&m->ext->last, 0, sizeof(hsb_stats));
  if (hsb_dev_steady(m->dev, power, temp, &m->ext->opts, &m->ext->last))
    return hsb_seterr(HSB_E_NOCONV, "%s\n", hsb_dev_last_error());
  m->ext->host_steady_valid = 0;
  return HSB_OK;
}

int hsb_grid_steady_leakage(grid_model_t *m, double *power, double *temp, int *iterations)
{
  int k, j, base, rc;
  double *dims;
  if (!m->r_ready) return hsb_seterr(HSB_E_ARG, "R model not ready\n");
  if (m->config.leakage_mode)
    return hsb_seterr(HSB_E_ARG, "HotLeakage currently is not implemented in this release of HotSpot\n");
  /* the power blocks' heights and widths (0: a block of a layer without power) */
  dims = calloc(2 * (size_t)m->total_n_blocks, sizeof(double));
  if (!dims) return hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
  for (k = 0, base = 0; k < m->n_layers; k++) {
    if (m->layers[k].has_power)
      for (j = 0; j < m->layers[k].flp->n_units; j++) {
        dims[base + j] = m->layers[k].flp->units[j].height;
        dims[m->total_n_blocks + base + j] = m->layers[k].flp->units[j].width;
      }
    base += m->layers[k].flp->n_units;
  }
  zero_internal_power(m, power);
  memset(&m->ext->last, 0, sizeof(hsb_stats));
  rc = hsb_dev_steady_leakage(m->dev, power, dims, dims + m->total_n_blocks, temp, &m->ext->opts, iterations,
                              &m->ext->last);
  free(dims);
  if (rc) return hsb_seterr(rc, "%s\n", hsb_dev_last_error());
  m->ext->host_steady_valid = 0;
  return HSB_OK;
}

/* ------------------------------------------------------------------------ */
/* exported: temperature_grid.h interface                                    */
/* ------------------------------------------------------------------------ */
grid_model_t *alloc_grid_model(thermal_config_t *config, flp_t *flp_default,
                               microchannel_config_t *microchannel_config,
                               materials_list_t *materials_list, int do_detailed_3D,
                               int use_microchannels)
{
  grid_model_t *m;
  OR_DIE(hsb_grid_alloc(&m, config, flp_default, microchannel_config, materials_list, do_detailed_3D,
                        use_microchannels));
  return m;
}

void delete_grid_model(grid_model_t *model) { free_model_host(model); }

void populate_R_model_grid(grid_model_t *model, flp_t *flp) { OR_DIE(hsb_grid_populate_R(model, flp)); }

void populate_C_model_grid(grid_model_t *model, flp_t *flp) { OR_DIE(hsb_grid_populate_C(model, flp)); }

void steady_state_temp_grid(grid_model_t *model, double *power, double *temp)
{
  OR_DIE(hsb_grid_steady(model, power, temp));
}

void compute_temp_grid(grid_model_t *model, double *power, double *temp, double time_elapsed)
{
  OR_DIE(hsb_grid_compute_temp(model, power, temp, time_elapsed));
}

double *hotspot_vector_grid(grid_model_t *model)
{
  double *v;
  if (model->total_n_blocks <= 0) {
    hsb_seterr(HSB_E_ARG, "total_n_blocks is not greater than zero\n");
    hsb_die();
  }
  v = calloc(model->total_n_blocks + n_extra(model), sizeof(double));
  if (!v) {
    hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
    hsb_die();
  }
  return v;
}

void trim_hotspot_vector_grid(grid_model_t *model, double *dst, double *src, int at, int size)
{
  int i;
  const int total = model->total_n_blocks + n_extra(model);
  if (model->has_lcf) {
    hsb_seterr(HSB_E_ARG, "trim_hotspot_vector_grid called with lcf file\n");
    hsb_die();
  }
  for (i = 0; i < at && i < total; i++) dst[i] = src[i];
  for (i = at + size; i < total; i++) dst[i - size] = src[i];
}

void resize_thermal_model_grid(grid_model_t *model, int n_units)
{
  int i;
  if (model->has_lcf) {
    hsb_seterr(HSB_E_ARG, "resize_thermal_model_grid called with lcf file\n");
    hsb_die();
  }
  if (n_units > model->base_n_units) {
    hsb_seterr(HSB_E_ARG, "resizing grid model to more than the allocated space\n");
    hsb_die();
  }
  model->total_n_blocks = 0;
  for (i = 0; i < model->n_layers; i++) model->total_n_blocks += model->layers[i].flp->n_units;
}

void set_temp_grid(grid_model_t *model, double *temp, double val)
{
  int i;
  const int total = model->total_n_blocks + n_extra(model);
  if (model->total_n_blocks <= 0) {
    hsb_seterr(HSB_E_ARG, "total_n_blocks is not greater than zero\n");
    hsb_die();
  }
  for (i = 0; i < total; i++) temp[i] = val;
}

void copy_temp_grid(grid_model_t *model, double *dst, double *src)
{
  memcpy(dst, src, sizeof(double) * (model->total_n_blocks + n_extra(model)));
}

grid_model_vector_t *new_grid_model_vector(grid_model_t *model)
{
  grid_model_vector_t *v = calloc(1, sizeof(grid_model_vector_t));
  if (!v || !(v->cuboid = hsb_dcuboid_tail(model->rows, model->cols, model->n_layers, n_extra(model)))) {
    hsb_seterr(HSB_E_NOMEM, "memory allocation error\n");
    hsb_die();
  }
  v->extra = v->cuboid[0][0] + (size_t)model->rows * model->cols * model->n_layers;
  return v;
}

void free_grid_model_vector(grid_model_vector_t *v)
{
  if (!v) return;
  hsb_free_dcuboid(v->cuboid);
  free(v);
}

/* host-side translation between block and grid vectors
 * (xlate_vector_b2g / xlate_temp_g2b, temperature_grid.c:1888-2015) */
void xlate_vector_b2g(grid_model_t *model, double *b, grid_model_vector_t *g, int type)
{
  int i, j, n, base = 0;
  const double area = (model->width * model->height) / (model->cols * model->rows);
  for (n = 0; n < model->n_layers; n++) {
    const flp_t *f = model->layers[n].flp;
    for (i = 0; i < model->rows; i++)
      for (j = 0; j < model->cols; j++) {
        double val = 0.0;
        for (const blist_t *p = model->layers[n].b2gmap[i][j]; p; p = p->next) {
          if (type == HSB_V_POWER)
            val += p->occupancy * b[base + p->idx] / (f->units[p->idx].width * f->units[p->idx].height);
          else
            val += p->occupancy * b[base + p->idx];
        }
        g->cuboid[n][i][j] = type == HSB_V_POWER ? val * area : val;
      }
    base += f->n_units;
  }
  for (i = 0; i < n_extra(model); i++) g->extra[i] = b[base + i];
}

void xlate_temp_g2b(grid_model_t *model, double *b, grid_model_vector_t *g)
{
  int i, j, n, u, base = 0, count;
  for (n = 0; n < model->n_layers; n++) {
    for (u = 0; u < model->layers[n].flp->n_units; u++) {
      const glist_t *G = &model->layers[n].g2bmap[u];
      const int i1 = G->i1, i2 = G->i2, j1 = G->j1, j2 = G->j2;
      double mn, mx, avg = 0.0;
      if (model->map_mode == HSB_GRID_CENTER) {
        const int ci1 = (i1 + i2) / 2, cj1 = (j1 + j2) / 2;
        const int ci2 = ci1 - !((i2 - i1) % 2), cj2 = cj1 - !((j2 - j1) % 2);
        b[base + u] = (g->cuboid[n][ci1][cj1] + g->cuboid[n][ci2][cj1] + g->cuboid[n][ci1][cj2] +
                       g->cuboid[n][ci2][cj2]) / 4;
        continue;
      }
      count = 0;
      mn = mx = g->cuboid[n][i1][j1];
      for (i = i1; i < i2; i++)
        for (j = j1; j < j2; j++) {
          avg += g->cuboid[n][i][j];
          if (g->cuboid[n][i][j] < mn) mn = g->cuboid[n][i][j];
          if (g->cuboid[n][i][j] > mx) mx = g->cuboid[n][i][j];
          count++;
        }
      b[base + u] = model->map_mode == HSB_GRID_AVG ? avg / count : model->map_mode == HSB_GRID_MIN ? mn : mx;
    }
    base += model->layers[n].flp->n_units;
  }
  for (i = 0; i < n_extra(model); i++) b[base + i] = g->extra[i];
}

double find_res_3D(int n, int i, int j, grid_model_t *model, int choice) { return res3(model, n, i, j, choice); }

double find_cap_3D(int n, int i, int j, grid_model_t *model) { return cap3(model, n, i, j); }

/* ------------------------------------------------------------------------ */
/* host copies of the device-resident grid state                             */
/* ------------------------------------------------------------------------ */
int hsb_grid_sync_host(grid_model_t *m)
{
  if (!m->ext->host_trans_valid) {
    if (hsb_dev_get_state(m->dev, 0, m->last_trans->cuboid[0][0]))
      return hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error());
    m->ext->host_trans_valid = 1;
  }
  if (!m->ext->host_steady_valid) {
    if (hsb_dev_get_state(m->dev, 1, m->last_steady->cuboid[0][0]))
      return hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error());
    m->ext->host_steady_valid = 1;
  }
  return HSB_OK;
}

int hsb_grid_get_state(grid_model_t *m, int which, double *out)
{
  if (hsb_dev_get_state(m->dev, which, out)) return hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error());
  return HSB_OK;
}

int hsb_grid_set_state(grid_model_t *m, int which, const double *in)
{
  if (hsb_dev_set_state(m->dev, which, in)) return hsb_seterr(HSB_E_CUDA, "%s\n", hsb_dev_last_error());
  if (which) m->ext->host_steady_valid = 0;
  else m->ext->host_trans_valid = 0;
  return HSB_OK;
}

int hsb_grid_set_solver(grid_model_t *m, int form, int steady_method, double steady_tol, int max_iters)
{
  if (form != HSB_FORM_PARITY && form != HSB_FORM_FAST && form != HSB_FORM_FAST_STAGES &&
      form != HSB_FORM_FAST_PASSES && form != HSB_FORM_FP64_BLOCKED && form != HSB_FORM_FAST_BLOCKED)
    return hsb_seterr(HSB_E_ARG, "unknown form %d\n", form);
  m->ext->opts.form = form;
  m->ext->opts.steady_method = steady_method;
  m->ext->opts.steady_tol = steady_tol;
  m->ext->opts.max_iters = max_iters;
  return HSB_OK;
}

int hsb_grid_get_stats(grid_model_t *m, hsb_stats *out)
{
  *out = m->ext->last;
  return HSB_OK;
}

struct hsb_dev_model *hsb_grid_device(grid_model_t *m) { return m->dev; }

const char *hsb_last_error(void) { return hsb_errmsg(); }
