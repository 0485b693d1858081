/*
 * hotspot_b200.h -- public C-ABI of libhotspot_b200.so, a B200 (sm_100a)
 * implementation of HotSpot's grid thermal model.
 *
 * Part 1 is HotSpot's own grid-model interface, same names, signatures,
 * argument meaning and error behaviour (fatal(): "error: <msg>" on stderr,
 * exit(1)), so the reference's model-API dispatch (temperature.c:616-938)
 * and its callers (hotspot.c, sim-template.c, cycle simulators) link against
 * this library in place of temperature_grid.o.  Each entry replaces the
 * reference function cited beside it (file:line in the HotSpot sources).
 *
 * Part 2 are additions of this library: solver selection, statistics,
 * access to the device-resident state, and status-returning variants of the
 * Part 1 calls for callers that must not exit (the serving loop).
 */
#ifndef HOTSPOT_B200_H
#define HOTSPOT_B200_H

#include "hotspot_b200_types.h"
#include "hsb_device.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- Part 1: temperature_grid.h:194-254 ------------------------------- */

/* temperature_grid.c:144 */
double find_res_3D(int n, int i, int j, grid_model_t *model, int choice);
/* temperature_grid.c:176 */
double find_cap_3D(int n, int i, int j, grid_model_t *model);
/* temperature_grid.c:896 -- also creates the device model (fails loudly when
 * no CUDA device is visible) */
grid_model_t *alloc_grid_model(thermal_config_t *config, flp_t *flp_default,
                               microchannel_config_t *microchannel_config,
                               materials_list_t *materials_list, int do_detailed_3D,
                               int use_microchannels);
/* temperature_grid.c:1117 */
void delete_grid_model(grid_model_t *model);
/* temperature_grid.c:950 -- builds maps and conductances, uploads them */
void populate_R_model_grid(grid_model_t *model, flp_t *flp);
/* temperature_grid.c:1065 */
void populate_C_model_grid(grid_model_t *model, flp_t *flp);
/* temperature_grid.c:2799 -- the steady state stays resident on the device;
 * the default form replays the reference's nested-iteration Gauss-Seidel */
void steady_state_temp_grid(grid_model_t *model, double *power, double *temp);
/* temperature_grid.c:3603 -- RK4 on the device; the grid state stays
 * resident between calls; `temp` is remembered as in the reference */
void compute_temp_grid(grid_model_t *model, double *power, double *temp, double time_elapsed);
/* temperature_grid.c:1182 */
double *hotspot_vector_grid(grid_model_t *model);
/* temperature_grid.c:1203 */
void trim_hotspot_vector_grid(grid_model_t *model, double *dst, double *src, int at, int size);
/* temperature_grid.c:1223 */
void resize_thermal_model_grid(grid_model_t *model, int n_units);
/* temperature_grid.c:1245 */
void set_temp_grid(grid_model_t *model, double *temp, double val);
/* temperature_grid.c:1262 (reads the device-resident steady state) */
void dump_steady_temp_grid(grid_model_t *model, char *file);
/* temperature_grid.c:1322 */
void dump_temp_grid(grid_model_t *model, double *temp, char *file);
/* temperature_grid.c:1297 (reads the device-resident transient state) */
void dump_transient_temp_grid(grid_model_t *model, int trace_num, double sampling_intvl, char *filename);
/* temperature_grid.c:1449 */
void copy_temp_grid(grid_model_t *model, double *dst, double *src);
/* temperature_grid.c:1462 */
void read_temp_grid(grid_model_t *model, double *temp, char *file, int clip);
/* temperature_grid.c:1645 */
void dump_power_grid(grid_model_t *model, double *power, char *file);
/* temperature_grid.c:1684 */
void read_power_grid(grid_model_t *model, double *power, char *file);
/* temperature_grid.c:1766 */
double find_max_temp_grid(grid_model_t *model, double *temp);
/* temperature_grid.c:1792 */
double find_avg_temp_grid(grid_model_t *model, double *temp);
/* temperature_grid.c:1816 */
double calc_sink_temp_grid(grid_model_t *model, double *temp, thermal_config_t *config);
/* temperature_grid.c:1861 */
grid_model_vector_t *new_grid_model_vector(grid_model_t *model);
/* temperature_grid.c:1881 */
void free_grid_model_vector(grid_model_vector_t *v);
/* temperature_grid.c:1888 (host vectors) */
void xlate_vector_b2g(grid_model_t *model, double *b, grid_model_vector_t *g, int type);
/* temperature_grid.c:1932 (host vectors) */
void xlate_temp_g2b(grid_model_t *model, double *b, grid_model_vector_t *g);
/* temperature_grid.c:3792 */
void debug_print_grid(grid_model_t *model);

/* ---- Part 2: additions (no counterpart in the reference) --------------- */

/* Solver form for later compute/steady calls: HSB_FORM_PARITY (default, or
 * env HOTSPOT_B200_FORM=fast) replays the reference in FP64;
 * HSB_FORM_FAST computes stencils in FP32 with FP64 state and refinement.
 * steady_method: HSB_STEADY_*; steady_tol: FP64 residual target in K
 * (0 = default); max_iters: iteration cap (0 = default). */
int hsb_grid_set_solver(grid_model_t *model, int form, int steady_method, double steady_tol,
                        int max_iters);
/* statistics of the last compute/steady call */
int hsb_grid_get_stats(grid_model_t *model, hsb_stats *out);
/* the full grid vector (nl*nr*nc cells + package nodes), which = 0 for the
 * transient state, 1 for the steady state */
int hsb_grid_get_state(grid_model_t *model, int which, double *out);
int hsb_grid_set_state(grid_model_t *model, int which, const double *in);
/* refresh model->last_trans / last_steady host copies from the device */
int hsb_grid_sync_host(grid_model_t *model);
/* Binary checkpoint of the grid state: both grid vectors (transient and
 * steady) with the grid's dimensions, so that a run can stop and resume on
 * another model of the same grid.  No counterpart in the reference (its
 * only state output is the text dumps below).  Load refuses a checkpoint
 * whose dimensions differ from the model's. */
int hsb_grid_save_state(grid_model_t *model, const char *path);
int hsb_grid_load_state(grid_model_t *model, const char *path);
/* The rows "%d\t%.2f\n" (index, value) of n grid cells, as the grid dumps
 * print them (dump_steady_temp_grid / dump_transient_temp_grid,
 * temperature_grid.c:1262-1319), byte for byte, without a printf per value;
 * out must hold 400 bytes per cell.  Returns the bytes written or HSB_E_ARG. */
long long hsb_format_grid_rows(const double *values, long long n, char *out, long long cap);
/* status-returning forms of alloc / populate / compute / steady */
int hsb_grid_alloc(grid_model_t **out, thermal_config_t *config, flp_t *flp_default,
                   microchannel_config_t *uconf, materials_list_t *ml, int do_detailed_3D,
                   int use_microchannels);
int hsb_grid_populate_R(grid_model_t *model, flp_t *flp);
int hsb_grid_populate_C(grid_model_t *model, flp_t *flp);
int hsb_grid_compute_temp(grid_model_t *model, double *power, double *temp, double time_elapsed);
int hsb_grid_steady(grid_model_t *model, double *power, double *temp);
/* the temperature-leakage fixed point of steady_state_temp with leakage_used
 * (temperature.c:706-746; calc_leakage, temperature.c:910-927) with the
 * block vectors on the device between iterations: temp holds the starting
 * temperatures and receives the result; *iterations (may be NULL) the
 * steady solves it took.  HSB_E_NOCONV on thermal runaway or when the loop
 * does not converge, as the reference's fatal() cases */
int hsb_grid_steady_leakage(grid_model_t *model, double *power, double *temp, int *iterations);
/* the device model behind a grid model (for the batch and serving layers) */
struct hsb_dev_model *hsb_grid_device(grid_model_t *model);
/* floorplan reader with flp.c's format (read_flp, flp.c:1175), for callers
 * without the reference's flp.c */
flp_t *hsb_read_flp(const char *file);
void hsb_free_flp_public(flp_t *flp);
/* message of the last failed hsb_* call on this thread */
const char *hsb_last_error(void);
/* sizeof of the boundary structs, in the order thermal_config_t, unit_t,
 * flp_t, materials_list_t, microchannel_config_t, package_RC_t, layer_t,
 * grid_model_vector_t, grid_model_t, hsb_stats; returns how many exist */
int hsb_abi_sizes(long long *out, int n);

#ifdef __cplusplus
}
#endif
#endif
