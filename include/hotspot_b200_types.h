/*
 * hotspot_b200_types.h -- data layouts shared with HotSpot's C model API.
 *
 * libhotspot_b200 is a drop-in for HotSpot's grid thermal model, so every
 * struct that crosses its boundary keeps the reference's memory layout field
 * for field: callers compiled against the reference headers (hotspot.c,
 * temperature.c, sim-template.c, external cycle simulators) read these
 * structs directly (e.g. hotspot.c:547-549 reads model->grid->n_layers,
 * layers[i].has_power and layers[i].flp->n_units).  The layouts follow:
 *
 *   thermal_config_t       temperature.h:141-221
 *   package_RC_t           temperature.h:237-334
 *   RC_model_t             temperature.h:347-357
 *   unit_t, flp_t          flp.h:122-144
 *   str_pair               util.h:92-96
 *   material_t, materials_list_t   materials.h:9-25
 *   microchannel_config_t  microchannel.h:29-90
 *   blist_t, glist_t       temperature_grid.h:63-96
 *   layer_t                temperature_grid.h:101-126
 *   grid_model_vector_t    temperature_grid.h:129-135
 *   grid_model_t           temperature_grid.h:138-191 (SUPERLU=0 layout),
 *                          with one field appended at the end (`dev`), which
 *                          callers never touch: they only hold pointers to a
 *                          grid_model_t that this library allocates.
 *
 * The constants (EXTRA, SP_W ... PCB_S, LCF_*, V_POWER, GRID_*) are the
 * reference's values, because they index caller-visible vectors.
 */
#ifndef HOTSPOT_B200_TYPES_H
#define HOTSPOT_B200_TYPES_H

#ifdef __cplusplus
extern "C" {
#endif

#define HSB_STR_SIZE   512      /* util.h:28 STR_SIZE */
#define HSB_LINE_SIZE  65536    /* util.h:29 LINE_SIZE */
#define HSB_MAX_UNITS  8192     /* flp.h:6 MAX_UNITS */

/* package nodes (temperature.h:38-76) */
#define HSB_EXTRA      12
#define HSB_EXTRA_SEC  16
enum {
  HSB_SP_W = 0, HSB_SP_E, HSB_SP_N, HSB_SP_S,
  HSB_SINK_C_W, HSB_SINK_C_E, HSB_SINK_C_N, HSB_SINK_C_S,
  HSB_SINK_W, HSB_SINK_E, HSB_SINK_N, HSB_SINK_S,
  HSB_SUB_W, HSB_SUB_E, HSB_SUB_N, HSB_SUB_S,
  HSB_SOLDER_W, HSB_SOLDER_E, HSB_SOLDER_N, HSB_SOLDER_S,
  HSB_PCB_C_W, HSB_PCB_C_E, HSB_PCB_C_N, HSB_PCB_C_S,
  HSB_PCB_W, HSB_PCB_E, HSB_PCB_N, HSB_PCB_S
};

/* grid-to-block mapping modes (temperature.h:19-22) */
#define HSB_GRID_AVG     0
#define HSB_GRID_MIN     1
#define HSB_GRID_MAX     2
#define HSB_GRID_CENTER  3

/* vector types (temperature_grid.h:30-31) */
#define HSB_V_POWER 0
#define HSB_V_TEMP  1

typedef struct hsb_thermal_config_st {
  double t_chip, k_chip, p_chip, thermal_threshold;
  double c_convec, r_convec, s_sink, t_sink, k_sink, p_sink;
  double s_spreader, t_spreader, k_spreader, p_spreader;
  double t_interface, k_interface, p_interface;
  int model_secondary;
  double r_convec_sec, c_convec_sec;
  int n_metal;
  double t_metal, t_c4, s_c4;
  int n_c4;
  double s_sub, t_sub, s_solder, t_solder, s_pcb, t_pcb;
  double ambient;
  char init_file[HSB_STR_SIZE];
  double init_temp;
  char steady_file[HSB_STR_SIZE];
  double sampling_intvl;
  double base_proc_freq;
  int dtm_used;
  char model_type[HSB_STR_SIZE];
  int leakage_used;
  int leakage_mode;
  int package_model_used;
  char package_config_file[HSB_STR_SIZE];
  int block_omit_lateral;
  int grid_rows;
  int grid_cols;
  char grid_layer_file[HSB_STR_SIZE];
  char grid_steady_file[HSB_STR_SIZE];
  char grid_map_mode[HSB_STR_SIZE];
  char grid_transient_file[HSB_STR_SIZE];
  int detailed_3D_used;
} thermal_config_t;

typedef struct hsb_package_RC_st {
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
} package_RC_t;

typedef struct hsb_unit_st {
  char name[HSB_STR_SIZE];
  double width, height, leftx, bottomy;
  double specificheat, resistivity;
  int hasRes, hasSh;
} unit_t;

typedef struct hsb_flp_st {
  unit_t *units;
  int n_units;
  double **wire_density;
} flp_t;

typedef struct hsb_str_pair_st {
  char name[HSB_STR_SIZE];
  char value[HSB_STR_SIZE];
} str_pair;

typedef struct hsb_material_st {
  int material_type;
  double thermal_conductivity;
  double volumetric_heat_capacity;
  double dynamic_viscosity;
} material_t;

typedef struct hsb_materials_list_st {
  int size;
  char **names;
  material_t *material_properties;
} materials_list_t;

/* microchannel cell types (microchannel.h:11-15) */
#define HSB_TSV    -1
#define HSB_SOLID   0
#define HSB_FLUID   1
#define HSB_INLET   2
#define HSB_OUTLET  3

typedef struct hsb_microchannel_config_st {
  double cell_width, cell_height, cell_thickness;
  double pumping_pressure, pump_internal_res, inlet_temperature;
  double coolant_capac, coolant_res, coolant_visc;
  double wall_capac, wall_res, htc;
  char network_file[HSB_STR_SIZE];
  char floorplan_file[HSB_STR_SIZE + 3];
  int num_rows, num_columns, n_fluid_cells;
  int **cell_types;
  int **mapping;
  double **A;      /* unused here: the pressure network is solved sparsely */
  double *b;       /* pressure of each fluid cell (indexed through mapping) */
  int nnz;
} microchannel_config_t;

typedef struct hsb_blist_st {
  int idx;
  double occupancy;
  struct hsb_blist_st *next;
  int lock, hasRes, hasCap;
  double rx, ry, rz;
  double capacitance;
} blist_t;

typedef struct hsb_glist_st {
  int i1, i2, j1, j2;
} glist_t;

typedef struct hsb_layer_st {
  flp_t *flp;
  int no, has_lateral, has_power;
  double k, thickness, sp;
  int is_microchannel;
  microchannel_config_t *microchannel_config;
  double rx, ry, rz;
  double c;
  blist_t ***b2gmap;
  glist_t *g2bmap;
} layer_t;

typedef struct hsb_grid_model_vector_st {
  double ***cuboid;
  double *extra;
} grid_model_vector_t;

struct hsb_dev_model;   /* device-resident state; opaque to callers */
struct hsb_host_ext;    /* host-side solver settings; opaque to callers */

typedef struct grid_model_t_st {
  thermal_config_t config;
  layer_t *layers;
  int n_layers;
  int rows, cols;
  double width, height;
  package_RC_t pack;
  int total_n_blocks;
  int map_mode;
  int r_ready, c_ready, has_lcf;
  grid_model_vector_t *last_steady;
  grid_model_vector_t *last_trans;
  double *last_temp;
  int base_n_units;
  int use_microchannels;
  microchannel_config_t *default_microchannel_config;
  /* ---- appended by libhotspot_b200 (not in the reference layout) ---- */
  struct hsb_dev_model *dev;     /* device-resident state and kernels */
  struct hsb_host_ext *ext;      /* solver options and statistics */
} grid_model_t;

#ifdef __cplusplus
}
#endif
#endif
