"""Python mirror of HotSpot's model API for the grid model, over the C-ABI.

Names, argument meaning and order follow the reference's C API
(temperature.h:224-391, microchannel.h:92-101, materials.h:27-35,
flp.h ``read_flp``) so that code driving the reference reads the same here:

    cfg = default_thermal_config()
    thermal_config_add_from_strs(cfg, materials, {"model_type": "grid", ...})
    flp = read_flp("chip.flp")
    model = alloc_RC_model(cfg, flp, None, materials, 0, 0)
    populate_R_model(model, flp); populate_C_model(model, flp)
    temp = hotspot_vector(model); set_temp(model, temp, cfg.init_temp)
    compute_temp(model, power, temp, cfg.sampling_intvl)
    steady_state_temp(model, power, steady)

Everything runs in libhotspot_b200.so on the GPU; this module only builds the
C structs and holds references so their memory outlives the model.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import check, dptr, lib

NULLFILE = b"(null)"


# ---------------------------------------------------------------------------
# configuration (temperature.c:19-109, :115-339; microchannel.c:17-108)
# ---------------------------------------------------------------------------
def default_thermal_config() -> _abi.ThermalConfig:
    c = _abi.ThermalConfig()
    c.t_chip, c.k_chip, c.p_chip = 0.15e-3, 100.0, 1.75e6
    c.thermal_threshold = 81.8 + 273.15
    c.c_convec, c.r_convec, c.s_sink, c.t_sink = 140.4, 0.1, 60e-3, 6.9e-3
    c.k_sink, c.p_sink = 400.0, 3.55e6
    c.s_spreader, c.t_spreader, c.k_spreader, c.p_spreader = 30e-3, 1e-3, 400.0, 3.55e6
    c.t_interface, c.k_interface, c.p_interface = 20e-6, 4.0, 4.0e6
    c.model_secondary, c.r_convec_sec, c.c_convec_sec = 0, 1.0, 140.4
    c.n_metal, c.t_metal, c.t_c4, c.s_c4, c.n_c4 = 8, 10.0e-6, 0.0001, 20.0e-6, 400
    c.s_sub, c.t_sub, c.s_solder, c.t_solder = 0.021, 0.001, 0.021, 0.00094
    c.s_pcb, c.t_pcb = 0.1, 0.002
    c.ambient = 45 + 273.15
    c.init_file = NULLFILE
    c.init_temp = 60 + 273.15
    c.steady_file = NULLFILE
    c.grid_transient_file = NULLFILE
    c.sampling_intvl = 3.333e-6
    c.base_proc_freq = 3e9
    c.dtm_used = 0
    c.leakage_used = c.leakage_mode = 0
    c.package_model_used = 0
    c.package_config_file = NULLFILE
    c.model_type = b"block"
    c.block_omit_lateral = 0
    c.grid_rows = c.grid_cols = 64
    c.grid_layer_file = NULLFILE
    c.grid_steady_file = NULLFILE
    c.grid_map_mode = b"center"
    c.detailed_3D_used = 0
    return c


def _set_field(obj, name: str, value: str):
    ftype = dict(obj._fields_)[name]
    if ftype is C.c_double:
        setattr(obj, name, float(value))
    elif ftype is C.c_int:
        setattr(obj, name, int(value))
    else:
        setattr(obj, name, str(value).encode())


_MATERIAL_KEYS = {"material_chip": ("k_chip", "p_chip"), "material_sink": ("k_sink", "p_sink"),
                  "material_spreader": ("k_spreader", "p_spreader"),
                  "material_interface": ("k_interface", "p_interface")}


def thermal_config_add_from_strs(cfg: _abi.ThermalConfig, materials: "Materials | None",
                                 table: dict):
    """Set configuration fields from name/value strings, as the reference's
    parser does for its option names (the struct field names plus material_*)."""
    fields = dict(cfg._fields_)
    for k, v in table.items():
        if k in fields:
            _set_field(cfg, k, v)
        elif k in _MATERIAL_KEYS:
            kk, pp = _MATERIAL_KEYS[k]
            if materials is None or v not in materials.props:
                raise ValueError(f"material name specified in configuration parameter {k} not found")
            setattr(cfg, kk, materials.props[v][0])
            setattr(cfg, pp, materials.props[v][1])


def default_microchannel_config() -> _abi.MicrochannelConfig:
    u = _abi.MicrochannelConfig()
    u.cell_width = u.cell_height = u.cell_thickness = 100e-6
    u.pumping_pressure, u.pump_internal_res, u.inlet_temperature = 5000, 0, 300
    u.coolant_capac, u.coolant_res, u.coolant_visc = 4172638, 1.647717911, 0.000889
    u.wall_capac, u.wall_res, u.htc = 1635660, 0.0076923077, 27132
    u.num_rows = u.num_columns = u.n_fluid_cells = -1
    return u


def microchannel_config_add_from_strs(u: _abi.MicrochannelConfig, materials: "Materials | None",
                                      table: dict):
    for k in ("pumping_pressure", "pump_internal_res", "inlet_temperature", "coolant_capac",
              "coolant_res", "coolant_visc", "wall_capac", "wall_res", "htc", "network_file"):
        if k in table:
            _set_field(u, k, table[k])
    if "wall_material" in table:
        k, cv, _ = materials.props[table["wall_material"]]
        u.wall_res, u.wall_capac = 1.0 / k, cv
    if "coolant_material" in table:
        k, cv, mu = materials.props[table["coolant_material"]]
        u.coolant_res, u.coolant_capac, u.coolant_visc = 1.0 / k, cv, mu


class Materials:
    """materials_list_t built from a materials file (format of materials.c:17-150)."""

    def __init__(self, path: str | None = None):
        self.props: dict[str, tuple[float, float, float]] = {}
        if path:
            toks = []
            for line in open(path):
                t = line.split()
                if t and not t[0].startswith("#"):
                    toks.append(t[0])
            i = 0
            while i < len(toks):
                name, kind = toks[i], toks[i + 1]
                k, cv = float(toks[i + 2]), float(toks[i + 3])
                mu = float(toks[i + 4]) if kind == "fluid" else 0.0
                self.props[name] = (k, cv, mu)
                i += 5 if kind == "fluid" else 4
        n = len(self.props)
        self._names = (C.c_char_p * max(n, 1))(*[k.encode() for k in self.props])
        self._mats = (_abi.Material * max(n, 1))()
        for i, (k, (kk, cv, mu)) in enumerate(self.props.items()):
            self._mats[i].material_type = 1 if mu else 0
            self._mats[i].thermal_conductivity = kk
            self._mats[i].volumetric_heat_capacity = cv
            self._mats[i].dynamic_viscosity = mu
        self.c = _abi.MaterialsList(n, C.cast(self._names, C.POINTER(C.c_char_p)),
                                    C.cast(self._mats, C.POINTER(_abi.Material)))


def read_flp(path: str):
    """Floorplan reader with the reference's format (flp.c:1175)."""
    f = lib().hsb_read_flp(path.encode())
    if not f:
        raise _abi.HotspotError(lib().hsb_last_error().decode().strip())
    return f


# ---------------------------------------------------------------------------
# the model (temperature.c:616-938 dispatch, grid model only)
# ---------------------------------------------------------------------------
class RCModel:
    """A grid model allocated by libhotspot_b200 (mirrors RC_model_t, type grid)."""

    def __init__(self, ptr, keep):
        self.ptr = ptr
        self._keep = keep
        g = ptr.contents
        self.n_layers, self.rows, self.cols = g.n_layers, g.rows, g.cols
        self.total_n_blocks = g.total_n_blocks
        self.n_extra = _abi.EXTRA + (_abi.EXTRA_SEC if g.config.model_secondary else 0)
        self.layer_units = [g.layers[i].flp.contents.n_units for i in range(self.n_layers)]
        self.layer_power = [bool(g.layers[i].has_power) for i in range(self.n_layers)]
        self.n_cells = self.n_layers * self.rows * self.cols

    @property
    def config(self) -> _abi.ThermalConfig:
        return self.ptr.contents.config

    def vector(self, fill: float = 0.0) -> np.ndarray:
        return np.full(self.total_n_blocks + self.n_extra, fill, dtype=np.float64)

    def unit_names(self, l: int) -> list[str]:
        f = self.ptr.contents.layers[l].flp.contents
        return [f.units[u].name.decode() for u in range(f.n_units)]

    def block_dims(self) -> tuple[np.ndarray, np.ndarray]:
        """Height and width (m) of every block; 0 for blocks of layers without power."""
        h, w = np.zeros(self.total_n_blocks), np.zeros(self.total_n_blocks)
        base = 0
        for l in range(self.n_layers):
            f = self.ptr.contents.layers[l].flp.contents
            if self.layer_power[l]:
                for u in range(f.n_units):
                    h[base + u], w[base + u] = f.units[u].height, f.units[u].width
            base += self.layer_units[l]
        return h, w

    def steady_leakage(self, power: np.ndarray, temp: np.ndarray) -> int:
        """The temperature-leakage fixed point of the steady solve on the device
        (steady_state_temp with leakage_used); temp: start in, result out.
        Returns the number of steady solves."""
        it = C.c_int()
        check(lib().hsb_grid_steady_leakage(self.ptr, dptr(power), dptr(temp), C.byref(it)))
        return it.value

    def power_vector(self, row) -> np.ndarray:
        """Scatter one trace row (power layers' blocks, floorplan order) into a block vector."""
        p = self.vector()
        base = k = 0
        for l in range(self.n_layers):
            n = self.layer_units[l]
            if self.layer_power[l]:
                p[base:base + n] = row[k:k + n]
                k += n
            base += n
        return p

    def set_solver(self, form: int = _abi.FORM_PARITY, steady_method: int = _abi.STEADY_AUTO,
                   steady_tol: float = 0.0, max_iters: int = 0):
        check(lib().hsb_grid_set_solver(self.ptr, form, steady_method, steady_tol, max_iters))

    def set_tile(self, rows: int, cols: int):
        """Own-tile shape of the temporally blocked transient kernel (0, 0: automatic)."""
        if lib().hsb_dev_set_tile(lib().hsb_grid_device(self.ptr), int(rows), int(cols)) != 0:
            raise _abi.HotspotError(lib().hsb_dev_last_error().decode(errors="replace").strip())

    def transient_kernel(self) -> str:
        """The kernel the fast transient runs for this model: "blocked",
        "blocked_fp64", "passes", or "" before its first fast interval."""
        k = C.c_int()
        if lib().hsb_dev_transient_kernel(lib().hsb_grid_device(self.ptr), C.byref(k)) != 0:
            raise _abi.HotspotError(lib().hsb_dev_last_error().decode(errors="replace").strip())
        return {0: "", 1: "blocked", 2: "blocked_fp64", 3: "passes"}[k.value]

    def stats(self) -> dict:
        s = _abi.Stats()
        check(lib().hsb_grid_get_stats(self.ptr, C.byref(s)))
        return s.as_dict()

    def grid(self, which: str = "trans") -> np.ndarray:
        out = np.empty(self.n_cells + self.n_extra)
        check(lib().hsb_grid_get_state(self.ptr, 0 if which == "trans" else 1, dptr(out)))
        return out

    def save_state(self, path: str):
        """Binary checkpoint of both grid vectors (hsb_grid_save_state)."""
        check(lib().hsb_grid_save_state(self.ptr, str(path).encode()))

    def load_state(self, path: str):
        """Restore a checkpoint written by save_state on a model of the same grid."""
        check(lib().hsb_grid_load_state(self.ptr, str(path).encode()))

    def dump_transient(self, trace_num: int, sampling_intvl: float, path: str):
        """Append the transient grid as dump_transient_temp_grid does."""
        lib().dump_transient_temp_grid(self.ptr, int(trace_num), float(sampling_intvl), str(path).encode())

    def set_grid(self, which: str, v: np.ndarray):
        v = np.ascontiguousarray(v, dtype=np.float64)
        check(lib().hsb_grid_set_state(self.ptr, 0 if which == "trans" else 1, dptr(v)))

    # status-returning forms (raise HotspotError instead of exiting)
    def compute_temp(self, power: np.ndarray, temp: np.ndarray | None, dt: float):
        self._last_temp = temp if temp is not None else getattr(self, "_last_temp", None)
        check(lib().hsb_grid_compute_temp(self.ptr, dptr(power), dptr(temp) if temp is not None else None, dt))

    def steady(self, power: np.ndarray, temp: np.ndarray):
        check(lib().hsb_grid_steady(self.ptr, dptr(power), dptr(temp)))

    def compute_trace(self, powers: np.ndarray, temp_in: np.ndarray | None, dt: float,
                      form: int = _abi.FORM_FAST) -> tuple[np.ndarray, dict]:
        """K consecutive intervals (rows of ``powers``) in one call; returns the
        block temperatures after the last interval and the call's statistics."""
        p = np.ascontiguousarray(powers, dtype=np.float64)
        out = self.vector()
        opts = _abi.SolverOpts(form, _abi.STEADY_AUTO, 0.0, 0)
        st = _abi.Stats()
        rc = lib().hsb_dev_transient_trace(lib().hsb_grid_device(self.ptr), dptr(p), int(p.shape[0]),
                                           dptr(temp_in) if temp_in is not None else None, dt, dptr(out),
                                           C.byref(opts), C.byref(st))
        if rc != 0:
            raise _abi.HotspotError(lib().hsb_dev_last_error().decode(errors="replace").strip())
        return out, st.as_dict()

    def close(self):
        if self.ptr:
            lib().delete_grid_model(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def alloc_RC_model(config: _abi.ThermalConfig, flp, microchannel_config, materials,
                   do_detailed_3D: int, use_microchannels: int) -> RCModel:
    """alloc_RC_model (temperature.c:616) for model_type "grid"."""
    if config.model_type.decode().lower() != "grid":
        raise ValueError("libhotspot_b200 implements the grid model (model_type grid) only")
    out = C.POINTER(_abi.GridModel)()
    mats = materials.c if materials is not None else None
    check(lib().hsb_grid_alloc(C.byref(out), C.byref(config), flp,
                               C.byref(microchannel_config) if microchannel_config is not None else None,
                               C.byref(mats) if mats is not None else None,
                               int(do_detailed_3D), int(use_microchannels)))
    return RCModel(out, (config, flp, microchannel_config, materials))


def populate_R_model(model: RCModel, flp):
    model._flp = flp
    check(lib().hsb_grid_populate_R(model.ptr, flp))


def populate_C_model(model: RCModel, flp):
    check(lib().hsb_grid_populate_C(model.ptr, flp))


def hotspot_vector(model: RCModel) -> np.ndarray:
    return model.vector()


def set_temp(model: RCModel, temp: np.ndarray, val: float):
    temp[:] = val


def compute_temp(model: RCModel, power: np.ndarray, temp: np.ndarray | None, time_elapsed: float):
    model.compute_temp(power, temp, time_elapsed)


def steady_state_temp(model: RCModel, power: np.ndarray, temp: np.ndarray):
    model.steady(power, temp)


def delete_RC_model(model: RCModel):
    model.close()


def from_scenario(sc, populate_c: bool = True) -> RCModel:
    """Build and populate a model from a :class:`hotspot_b200.workloads.Scenario`."""
    mats = Materials(sc.materials) if sc.materials else Materials()
    cfg = default_thermal_config()
    thermal_config_add_from_strs(cfg, mats, sc.config)
    uc = None
    if sc.use_microchannels:
        uc = default_microchannel_config()
        microchannel_config_add_from_strs(uc, mats, sc.config)
    flp = None if sc.lcf else read_flp(sc.flp)
    m = alloc_RC_model(cfg, flp, uc, mats, int(sc.detailed_3D), int(sc.use_microchannels))
    m._keep = (cfg, flp, uc, mats)
    populate_R_model(m, flp)
    if populate_c:
        populate_C_model(m, flp)
    return m
