/* host_internal.h -- private declarations of libhotspot_b200's C host code. */
#ifndef HSB_HOST_INTERNAL_H
#define HSB_HOST_INTERNAL_H

#include <stdio.h>
#include "hotspot_b200_types.h"
#include "hsb_device.h"

#define HSB_HIDDEN __attribute__((visibility("hidden")))

#define HSB_DELTA     1.0e-6    /* util.h:18 */
#define HSB_LARGENUM  1.0e100   /* util.h:19 */
#define HSB_NULLFILE  "(null)"  /* util.h:20 */
#define HSB_C_FACTOR  0.333     /* temperature.h:116 */
#define HSB_OCCUPANCY_THRESHOLD 0.95  /* temperature_grid.h:58 */

/* layer bookkeeping (temperature_grid.h:36-54) */
#define HSB_DEFAULT_CHIP_LAYERS 2
#define HSB_LAYER_SI  0
#define HSB_LAYER_INT 1
#define HSB_SEC_CHIP_LAYERS 2
#define HSB_LAYER_C4 0
#define HSB_LAYER_METAL 1
#define HSB_DEFAULT_PACK_LAYERS 2
#define HSB_LAYER_SP 0
#define HSB_LAYER_SINK 1
#define HSB_SEC_PACK_LAYERS 3
#define HSB_LAYER_PCB 0
#define HSB_LAYER_SOLDER 1
#define HSB_LAYER_SUB 2

/* secondary-path material constants (temperature.h:91-112) */
#define HSB_K_METAL (1.0 / 0.0025)
#define HSB_K_C4 (1.0 / 0.8)
#define HSB_K_SUB (1.0 / 0.5)
#define HSB_K_SOLDER (1.0 / 0.06)
#define HSB_K_PCB (1.0 / 0.333)
#define HSB_SPEC_HEAT_METAL 3.55e6
#define HSB_SPEC_HEAT_C4 1.65e6
#define HSB_SPEC_HEAT_SUB 1.6e6
#define HSB_SPEC_HEAT_SOLDER 2.1e6
#define HSB_SPEC_HEAT_PCB 1.32e6

#define FLUID_CELL_TYPE(t) ((t) == HSB_FLUID || (t) == HSB_INLET || (t) == HSB_OUTLET)

#define HSB_MAX(x, y) (((x) > (y)) ? (x) : (y))
#define HSB_MIN(x, y) (((x) < (y)) ? (x) : (y))

/* errors: internal functions return 0 / HSB_E_*; the message is kept per thread */
HSB_HIDDEN int hsb_seterr(int code, const char *fmt, ...);
HSB_HIDDEN const char *hsb_errmsg(void);
/* the reference's fatal(): "error: <msg>" on stderr, exit(1) (util.c:32-36) */
HSB_HIDDEN void hsb_die(void) __attribute__((noreturn));
HSB_HIDDEN void hsb_warn(const char *msg);

HSB_HIDDEN int hsb_eq(double x, double y);
HSB_HIDDEN int hsb_tolerant_ceil(double v);
HSB_HIDDEN int hsb_tolerant_floor(double v);
HSB_HIDDEN double hsb_getr(double k, double thickness, double area);
HSB_HIDDEN double hsb_getcap(double sp, double thickness, double area);
HSB_HIDDEN double ***hsb_dcuboid_tail(int nr, int nc, int nl, int xtra);
HSB_HIDDEN void hsb_free_dcuboid(double ***m);

/* floorplans (flp.c:1004-1230 semantics) */
HSB_HIDDEN int hsb_read_flp_file(const char *file, flp_t **out);
HSB_HIDDEN int hsb_read_flp_text(const char *text, const char *what, flp_t **out);
HSB_HIDDEN void hsb_free_flp(flp_t *flp);
HSB_HIDDEN double hsb_flp_width(const flp_t *flp);
HSB_HIDDEN double hsb_flp_height(const flp_t *flp);
HSB_HIDDEN int hsb_flp_index(const flp_t *flp, const char *name);

/* materials (materials.c:162-205 semantics) */
HSB_HIDDEN double hsb_material_k(const materials_list_t *ml, const char *name);
HSB_HIDDEN double hsb_material_cv(const materials_list_t *ml, const char *name);

/* package R/C (temperature.c:458-569) */
HSB_HIDDEN void hsb_package_R(package_RC_t *p, const thermal_config_t *c, double w, double h);
HSB_HIDDEN void hsb_package_C(package_RC_t *p, const thermal_config_t *c, double w, double h);

/* microchannel network (microchannel.c:258-571 semantics) */
HSB_HIDDEN int hsb_uchan_build(microchannel_config_t *u, flp_t **flp_out);
HSB_HIDDEN double hsb_uchan_hydroC(const microchannel_config_t *u);
HSB_HIDDEN double hsb_uchan_flow(const microchannel_config_t *u, int i1, int j1, int i2, int j2);
HSB_HIDDEN void hsb_uchan_free(microchannel_config_t *u);

/* model pieces */
HSB_HIDDEN double hsb_find_res(grid_model_t *m, int n1, int i1, int j1, int n2, int i2, int j2);

/* per-model host state hung off grid_model_t.dev's companion */
typedef struct hsb_host_ext {
  hsb_solver_opts opts;
  hsb_stats last;
  int host_trans_valid;   /* host copy of last_trans is current */
  int host_steady_valid;
  int dev_ready_r;        /* device has current conductances */
} hsb_host_ext;

#define hsb_ext(m) ((m)->ext)

#endif
