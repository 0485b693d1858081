"""ctypes view of libhotspot_b200.so: the struct layouts of
``include/hotspot_b200_types.h`` and the entry points of
``include/hotspot_b200.h`` / ``include/hsb_device.h``.

The library is built in-tree (``make -C hotspot_b200/csrc`` or
``__graft_entry__.build()``).  Loading fails loudly when it is missing: there
is no CPU fallback anywhere in this package.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhotspot_b200.so")

STR = 512
EXTRA, EXTRA_SEC = 12, 16

# solver forms / methods (hsb_device.h)
FORM_PARITY, FORM_FAST, FORM_FAST_STAGES, FORM_FAST_PASSES, FORM_FP64_BLOCKED, FORM_FAST_BLOCKED = 0, 1, 2, 3, 4, 5
STEADY_AUTO, STEADY_GS_REPLAY, STEADY_MG, STEADY_BICGSTAB = 0, 1, 2, 3


class ThermalConfig(C.Structure):
    """thermal_config_t (temperature.h:141-221)."""
    _fields_ = [
        ("t_chip", C.c_double), ("k_chip", C.c_double), ("p_chip", C.c_double),
        ("thermal_threshold", C.c_double),
        ("c_convec", C.c_double), ("r_convec", C.c_double), ("s_sink", C.c_double),
        ("t_sink", C.c_double), ("k_sink", C.c_double), ("p_sink", C.c_double),
        ("s_spreader", C.c_double), ("t_spreader", C.c_double), ("k_spreader", C.c_double),
        ("p_spreader", C.c_double),
        ("t_interface", C.c_double), ("k_interface", C.c_double), ("p_interface", C.c_double),
        ("model_secondary", C.c_int), ("r_convec_sec", C.c_double), ("c_convec_sec", C.c_double),
        ("n_metal", C.c_int), ("t_metal", C.c_double), ("t_c4", C.c_double), ("s_c4", C.c_double),
        ("n_c4", C.c_int), ("s_sub", C.c_double), ("t_sub", C.c_double), ("s_solder", C.c_double),
        ("t_solder", C.c_double), ("s_pcb", C.c_double), ("t_pcb", C.c_double),
        ("ambient", C.c_double), ("init_file", C.c_char * STR), ("init_temp", C.c_double),
        ("steady_file", C.c_char * STR), ("sampling_intvl", C.c_double),
        ("base_proc_freq", C.c_double), ("dtm_used", C.c_int), ("model_type", C.c_char * STR),
        ("leakage_used", C.c_int), ("leakage_mode", C.c_int), ("package_model_used", C.c_int),
        ("package_config_file", C.c_char * STR), ("block_omit_lateral", C.c_int),
        ("grid_rows", C.c_int), ("grid_cols", C.c_int), ("grid_layer_file", C.c_char * STR),
        ("grid_steady_file", C.c_char * STR), ("grid_map_mode", C.c_char * STR),
        ("grid_transient_file", C.c_char * STR), ("detailed_3D_used", C.c_int),
    ]


class Unit(C.Structure):
    """unit_t (flp.h:122-135)."""
    _fields_ = [("name", C.c_char * STR), ("width", C.c_double), ("height", C.c_double),
                ("leftx", C.c_double), ("bottomy", C.c_double), ("specificheat", C.c_double),
                ("resistivity", C.c_double), ("hasRes", C.c_int), ("hasSh", C.c_int)]


class Flp(C.Structure):
    """flp_t (flp.h:138-144)."""
    _fields_ = [("units", C.POINTER(Unit)), ("n_units", C.c_int),
                ("wire_density", C.POINTER(C.POINTER(C.c_double)))]


class Material(C.Structure):
    _fields_ = [("material_type", C.c_int), ("thermal_conductivity", C.c_double),
                ("volumetric_heat_capacity", C.c_double), ("dynamic_viscosity", C.c_double)]


class MaterialsList(C.Structure):
    """materials_list_t (materials.h:17-25)."""
    _fields_ = [("size", C.c_int), ("names", C.POINTER(C.c_char_p)),
                ("material_properties", C.POINTER(Material))]


class MicrochannelConfig(C.Structure):
    """microchannel_config_t (microchannel.h:29-90)."""
    _fields_ = [
        ("cell_width", C.c_double), ("cell_height", C.c_double), ("cell_thickness", C.c_double),
        ("pumping_pressure", C.c_double), ("pump_internal_res", C.c_double),
        ("inlet_temperature", C.c_double), ("coolant_capac", C.c_double),
        ("coolant_res", C.c_double), ("coolant_visc", C.c_double), ("wall_capac", C.c_double),
        ("wall_res", C.c_double), ("htc", C.c_double), ("network_file", C.c_char * STR),
        ("floorplan_file", C.c_char * (STR + 3)), ("num_rows", C.c_int), ("num_columns", C.c_int),
        ("n_fluid_cells", C.c_int), ("cell_types", C.POINTER(C.POINTER(C.c_int))),
        ("mapping", C.POINTER(C.POINTER(C.c_int))), ("A", C.POINTER(C.POINTER(C.c_double))),
        ("b", C.POINTER(C.c_double)), ("nnz", C.c_int),
    ]


class PackageRC(C.Structure):
    """package_RC_t (temperature.h:237-334): 52 doubles."""
    _fields_ = [(f"f{i}", C.c_double) for i in range(52)]


class Layer(C.Structure):
    """layer_t (temperature_grid.h:101-126)."""
    _fields_ = [
        ("flp", C.POINTER(Flp)), ("no", C.c_int), ("has_lateral", C.c_int), ("has_power", C.c_int),
        ("k", C.c_double), ("thickness", C.c_double), ("sp", C.c_double),
        ("is_microchannel", C.c_int), ("microchannel_config", C.POINTER(MicrochannelConfig)),
        ("rx", C.c_double), ("ry", C.c_double), ("rz", C.c_double), ("c", C.c_double),
        ("b2gmap", C.c_void_p), ("g2bmap", C.c_void_p),
    ]


class GridVector(C.Structure):
    _fields_ = [("cuboid", C.c_void_p), ("extra", C.POINTER(C.c_double))]


class GridModel(C.Structure):
    """grid_model_t (temperature_grid.h:138-191) + the two appended fields."""
    _fields_ = [
        ("config", ThermalConfig), ("layers", C.POINTER(Layer)), ("n_layers", C.c_int),
        ("rows", C.c_int), ("cols", C.c_int), ("width", C.c_double), ("height", C.c_double),
        ("pack", PackageRC), ("total_n_blocks", C.c_int), ("map_mode", C.c_int),
        ("r_ready", C.c_int), ("c_ready", C.c_int), ("has_lcf", C.c_int),
        ("last_steady", C.POINTER(GridVector)), ("last_trans", C.POINTER(GridVector)),
        ("last_temp", C.POINTER(C.c_double)), ("base_n_units", C.c_int),
        ("use_microchannels", C.c_int),
        ("default_microchannel_config", C.POINTER(MicrochannelConfig)),
        ("dev", C.c_void_p), ("ext", C.c_void_p),
    ]


class Stats(C.Structure):
    """hsb_stats (hsb_device.h)."""
    _fields_ = [("rk4_steps", C.c_longlong), ("rk4_attempts", C.c_longlong),
                ("slope_evals", C.c_longlong), ("sweeps", C.c_longlong),
                ("cycles", C.c_longlong), ("refinements", C.c_longlong),
                ("residual", C.c_double), ("sim_time", C.c_double), ("device_ms", C.c_double),
                ("kernel_ms", C.c_double), ("launches", C.c_longlong), ("fallbacks", C.c_longlong)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class Request(C.Structure):
    """hsb_request (hsb_device.h)."""
    _fields_ = [("model", C.c_int), ("kind", C.c_int), ("steps", C.c_int), ("dt", C.c_double),
                ("power", C.c_void_p), ("temp_in", C.c_void_p), ("out", C.c_void_p),
                ("arrival", C.c_double), ("start", C.c_double), ("finish", C.c_double),
                ("status", C.c_int), ("worker", C.c_int)]


REQ_STEADY, REQ_TRANSIENT = 0, 1


class GridDesc(C.Structure):
    """hsb_grid_desc (hsb_device.h)."""
    _fields_ = [("nl", C.c_int), ("nr", C.c_int), ("nc", C.c_int), ("n_extra", C.c_int),
                ("spidx", C.c_int), ("hsidx", C.c_int), ("subidx", C.c_int), ("solderidx", C.c_int),
                ("pcbidx", C.c_int), ("field", C.c_int), ("map_mode", C.c_int), ("total_n_blocks", C.c_int),
                ("ambient", C.c_double), ("width", C.c_double), ("height", C.c_double),
                ("pcb_amb_num", C.c_double),
                ("layer_rx", C.POINTER(C.c_double)), ("layer_ry", C.POINTER(C.c_double)),
                ("layer_rz", C.POINTER(C.c_double)), ("layer_c", C.POINTER(C.c_double)),
                ("pack", C.POINTER(C.c_double))]


class SolverOpts(C.Structure):
    """hsb_solver_opts (hsb_device.h)."""
    _fields_ = [("form", C.c_int), ("steady_method", C.c_int), ("steady_tol", C.c_double),
                ("max_iters", C.c_int)]


_lib = None

# entry points and their ctypes signatures (include/hotspot_b200.h)
_GM = C.POINTER(GridModel)
_D = C.POINTER(C.c_double)
_SIGS = {
    "alloc_grid_model": (_GM, [C.POINTER(ThermalConfig), C.POINTER(Flp), C.POINTER(MicrochannelConfig),
                               C.POINTER(MaterialsList), C.c_int, C.c_int]),
    "delete_grid_model": (None, [_GM]),
    "populate_R_model_grid": (None, [_GM, C.POINTER(Flp)]),
    "populate_C_model_grid": (None, [_GM, C.POINTER(Flp)]),
    "steady_state_temp_grid": (None, [_GM, _D, _D]),
    "compute_temp_grid": (None, [_GM, _D, _D, C.c_double]),
    "hotspot_vector_grid": (_D, [_GM]),
    "trim_hotspot_vector_grid": (None, [_GM, _D, _D, C.c_int, C.c_int]),
    "resize_thermal_model_grid": (None, [_GM, C.c_int]),
    "set_temp_grid": (None, [_GM, _D, C.c_double]),
    "dump_steady_temp_grid": (None, [_GM, C.c_char_p]),
    "dump_temp_grid": (None, [_GM, _D, C.c_char_p]),
    "dump_transient_temp_grid": (None, [_GM, C.c_int, C.c_double, C.c_char_p]),
    "copy_temp_grid": (None, [_GM, _D, _D]),
    "read_temp_grid": (None, [_GM, _D, C.c_char_p, C.c_int]),
    "dump_power_grid": (None, [_GM, _D, C.c_char_p]),
    "read_power_grid": (None, [_GM, _D, C.c_char_p]),
    "find_max_temp_grid": (C.c_double, [_GM, _D]),
    "find_avg_temp_grid": (C.c_double, [_GM, _D]),
    "calc_sink_temp_grid": (C.c_double, [_GM, _D, C.POINTER(ThermalConfig)]),
    "new_grid_model_vector": (C.POINTER(GridVector), [_GM]),
    "free_grid_model_vector": (None, [C.POINTER(GridVector)]),
    "xlate_vector_b2g": (None, [_GM, _D, C.POINTER(GridVector), C.c_int]),
    "xlate_temp_g2b": (None, [_GM, _D, C.POINTER(GridVector)]),
    "debug_print_grid": (None, [_GM]),
    "find_res_3D": (C.c_double, [C.c_int, C.c_int, C.c_int, _GM, C.c_int]),
    "find_cap_3D": (C.c_double, [C.c_int, C.c_int, C.c_int, _GM]),
    "hsb_grid_set_solver": (C.c_int, [_GM, C.c_int, C.c_int, C.c_double, C.c_int]),
    "hsb_grid_get_stats": (C.c_int, [_GM, C.POINTER(Stats)]),
    "hsb_grid_get_state": (C.c_int, [_GM, C.c_int, _D]),
    "hsb_grid_set_state": (C.c_int, [_GM, C.c_int, _D]),
    "hsb_grid_save_state": (C.c_int, [_GM, C.c_char_p]),
    "hsb_grid_load_state": (C.c_int, [_GM, C.c_char_p]),
    "hsb_format_grid_rows": (C.c_longlong, [_D, C.c_longlong, C.c_char_p, C.c_longlong]),
    "hsb_grid_sync_host": (C.c_int, [_GM]),
    "hsb_grid_alloc": (C.c_int, [C.POINTER(_GM), C.POINTER(ThermalConfig), C.POINTER(Flp),
                                 C.POINTER(MicrochannelConfig), C.POINTER(MaterialsList), C.c_int, C.c_int]),
    "hsb_grid_populate_R": (C.c_int, [_GM, C.POINTER(Flp)]),
    "hsb_grid_populate_C": (C.c_int, [_GM, C.POINTER(Flp)]),
    "hsb_grid_compute_temp": (C.c_int, [_GM, _D, _D, C.c_double]),
    "hsb_grid_steady": (C.c_int, [_GM, _D, _D]),
    "hsb_grid_steady_leakage": (C.c_int, [_GM, _D, _D, C.POINTER(C.c_int)]),
    "hsb_grid_device": (C.c_void_p, [_GM]),
    "hsb_read_flp": (C.POINTER(Flp), [C.c_char_p]),
    "hsb_free_flp_public": (None, [C.POINTER(Flp)]),
    "hsb_last_error": (C.c_char_p, []),
    "hsb_dev_last_error": (C.c_char_p, []),
    "hsb_dev_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(GridDesc)]),
    "hsb_dev_destroy": (None, [C.c_void_p]),
    "hsb_dev_set_layers": (C.c_int, [C.c_void_p, _D, _D, _D, _D, _D, C.c_double, C.c_double, C.c_double,
                                     C.c_double]),
    "hsb_dev_set_cells": (C.c_int, [C.c_void_p, _D, _D, _D, _D, _D, _D, _D]),
    "hsb_dev_set_advection": (C.c_int, [C.c_void_p, _D, _D, _D, _D, _D, _D]),
    "hsb_dev_set_maps": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), _D, _D, C.c_double,
                                   C.POINTER(C.c_int)]),
    "hsb_dev_transient": (C.c_int, [C.c_void_p, _D, _D, C.c_double, _D, C.POINTER(SolverOpts),
                                    C.POINTER(Stats)]),
    "hsb_dev_steady": (C.c_int, [C.c_void_p, _D, _D, C.POINTER(SolverOpts), C.POINTER(Stats)]),
    "hsb_dev_transient_trace": (C.c_int, [C.c_void_p, _D, C.c_int, _D, C.c_double, _D, C.POINTER(SolverOpts),
                                          C.POINTER(Stats)]),
    "hsb_dev_get_state": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "hsb_dev_workspaces": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "hsb_dev_transient_kernel": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "hsb_dev_steady_leakage": (C.c_int, [C.c_void_p, _D, _D, _D, _D, C.c_void_p, C.POINTER(C.c_int), C.c_void_p]),
    "hsb_dev_set_tile": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "hsb_dev_set_state": (C.c_int, [C.c_void_p, C.c_int, _D]),
    "hsb_abi_sizes": (C.c_int, [C.POINTER(C.c_longlong), C.c_int]),
    "hsb_dev_transient_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_double,
                                            C.POINTER(Stats)]),
    "hsb_batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(C.c_void_p), C.c_int]),
    "hsb_batch_destroy": (None, [C.c_void_p]),
    "hsb_batch_transient": (C.c_int, [C.c_void_p, _D, C.c_double, C.POINTER(Stats)]),
    "hsb_batch_transient_trace": (C.c_int, [C.c_void_p, _D, C.c_int, C.c_double, C.POINTER(Stats)]),
    "hsb_batch_chip_tile": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]),
    "hsb_batch_set_ctas": (C.c_int, [C.c_void_p, C.c_int]),
    "hsb_batch_run_subset": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.c_int, _D, C.c_int, C.c_double,
                                       C.POINTER(Stats)]),
    "hsb_batch_offsets": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "hsb_batch_set_schedule": (C.c_int, [C.c_void_p, C.c_int, C.c_double]),
    "hsb_batch_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_longlong),
                                 C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "hsb_batch_chip_steps": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "hsb_batch_autotune": (C.c_int, [C.c_void_p, C.c_int]),
    "hsb_server_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.c_longlong]),
    "hsb_server_destroy": (None, [C.c_void_p]),
    "hsb_server_add_model": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_longlong]),
    "hsb_server_add_replica": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p]),
    "hsb_server_run": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int]),
    "hsb_server_set_priority": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "hsb_server_set_batching": (C.c_int, [C.c_void_p, C.c_int]),
    "hsb_server_batch_stats": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong), C.POINTER(C.c_longlong),
                                         C.POINTER(C.c_longlong)]),
    "hsb_dev_set_priority": (C.c_int, [C.c_void_p, C.c_int]),
    "hsb_batch_tuning": (C.c_int, [C.c_void_p, _D, C.c_int]),
}


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libhotspot_b200.so is not built ({LIB_PATH}); run "
                               "`python -c 'import __graft_entry__ as g; g.build()'` "
                               "or `make -C hotspot_b200/csrc`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def dptr(a):
    """double* view of a C-contiguous float64 numpy array."""
    return a.ctypes.data_as(_D)


class HotspotError(RuntimeError):
    pass


def check(rc: int):
    if rc != 0:
        raise HotspotError(lib().hsb_last_error().decode(errors="replace").strip())
