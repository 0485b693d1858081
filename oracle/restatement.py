"""CPU restatement of HotSpot's grid model -- TEST INFRASTRUCTURE ONLY.

The test oracle of libhotspot_b200: only ``tests/``, ``__graft_entry__.smoke``
and ``bench.py``'s CPU-baseline leg import this module, never the product.

Model set-up runs here in Python (executed once per model, small sizes): the
floorplan/LCF readers, layer stack, block<->grid occupancy lists, R/C values,
package R/C and microchannel flow rates, each restating the reference
function cited at its definition with the same IEEE-double operations.  The
hot loops (slope, RK4, Gauss-Seidel, nested multigrid) run in
``oracle/grid_oracle.c`` (built by ``make -C oracle restatement``).  The
microchannel steady state, which the reference can only solve through
SuperLU (absent), is restated as the sparse system G T = P of
``build_transient_grid_matrix`` / ``build_transient_power_vector``
(temperature_grid.c:5196-6694) and solved by ``scipy.sparse.linalg.splu``
(FP64 direct).
"""
from __future__ import annotations

import contextlib
import ctypes as C
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libgrid_oracle.so")

DELTA = 1.0e-6
LARGENUM = 1.0e100
C_FACTOR = 0.333
EXTRA, EXTRA_SEC = 12, 16
(SP_W, SP_E, SP_N, SP_S, SINK_C_W, SINK_C_E, SINK_C_N, SINK_C_S, SINK_W, SINK_E, SINK_N, SINK_S) = range(12)
TSV, SOLID, FLUID, INLET, OUTLET = -1, 0, 1, 2, 3

# secondary-path constants (temperature.h:91-112)
K_SUB, K_SOLDER, K_PCB, K_METAL, K_C4 = 1.0 / 0.5, 1.0 / 0.06, 1.0 / 0.333, 1.0 / 0.0025, 1.0 / 0.8
SH_SUB, SH_SOLDER, SH_PCB, SH_METAL, SH_C4 = 1.6e6, 2.1e6, 1.32e6, 3.55e6, 1.65e6

PACK_FIELDS = [
    "r_sp1_x", "r_sp1_y", "r_hs1_x", "r_hs1_y", "r_hs2_x", "r_hs2_y", "r_hs",
    "r_sp_per_x", "r_sp_per_y", "r_hs_c_per_x", "r_hs_c_per_y", "r_hs_per",
    "c_sp_per_x", "c_sp_per_y", "c_hs_c_per_x", "c_hs_c_per_y", "c_hs_per",
    "r_amb_c_per_x", "c_amb_c_per_x", "r_amb_c_per_y", "c_amb_c_per_y", "r_amb_per", "c_amb_per",
    "r_sub1_x", "r_sub1_y", "r_solder1_x", "r_solder1_y", "r_pcb1_x", "r_pcb1_y", "r_pcb2_x",
    "r_pcb2_y", "r_pcb", "r_sub_per_x", "r_sub_per_y", "r_solder_per_x", "r_solder_per_y",
    "r_pcb_c_per_x", "r_pcb_c_per_y", "r_pcb_per", "c_sub_per_x", "c_sub_per_y", "c_solder_per_x",
    "c_solder_per_y", "c_pcb_c_per_x", "c_pcb_c_per_y", "c_pcb_per", "r_amb_sec_c_per_x",
    "c_amb_sec_c_per_x", "r_amb_sec_c_per_y", "c_amb_sec_c_per_y", "r_amb_sec_per", "c_amb_sec_per",
]

# default_thermal_config (temperature.c:19-109)
DEFAULT_CONFIG = dict(
    t_chip=0.15e-3, k_chip=100.0, p_chip=1.75e6, thermal_threshold=81.8 + 273.15,
    c_convec=140.4, r_convec=0.1, s_sink=60e-3, t_sink=6.9e-3, k_sink=400.0, p_sink=3.55e6,
    s_spreader=30e-3, t_spreader=1e-3, k_spreader=400.0, p_spreader=3.55e6,
    t_interface=20e-6, k_interface=4.0, p_interface=4.0e6, model_secondary=0, r_convec_sec=1.0,
    c_convec_sec=140.4, n_metal=8, t_metal=10.0e-6, t_c4=0.0001, s_c4=20.0e-6, n_c4=400,
    s_sub=0.021, t_sub=0.001, s_solder=0.021, t_solder=0.00094, s_pcb=0.1, t_pcb=0.002,
    ambient=45 + 273.15, init_temp=60 + 273.15, sampling_intvl=3.333e-6, grid_rows=64,
    grid_cols=64, grid_layer_file="(null)", grid_map_mode="center", model_type="block",
)
# default_microchannel_config (microchannel.c:17-45)
DEFAULT_UCHAN = dict(pumping_pressure=5000.0, pump_internal_res=0.0, inlet_temperature=300.0,
                     coolant_capac=4172638.0, coolant_res=1.647717911, coolant_visc=0.000889,
                     wall_capac=1635660.0, wall_res=0.0076923077, htc=27132.0)


def eq(x, y):
    return abs(x - y) < DELTA


def tolerant_ceil(v):            # util.c:57-66
    nearest = math.floor(v + 0.5)
    return int(nearest) if eq(v, nearest) else int(math.ceil(v))


def tolerant_floor(v):           # util.c:68-77
    nearest = math.floor(v + 0.5)
    return int(nearest) if eq(v, nearest) else int(math.floor(v))


def getr(k, t, a):               # RCutil.c:20-23
    return t / (k * a)


def getcap(sp, t, a):            # RCutil.c:26-31
    return C_FACTOR * sp * t * a


# ---------------------------------------------------------------------------
# floorplans (flp.c:1004-1230)
# ---------------------------------------------------------------------------
class Unit:
    __slots__ = ("name", "w", "h", "x", "y", "cp", "res", "has")

    def __init__(self, name, w, h, x, y, cp=0.0, res=0.0, has=False):
        self.name, self.w, self.h, self.x, self.y = name, w, h, x, y
        self.cp, self.res, self.has = cp, res, has


def _num(tok):
    try:
        return float(tok)
    except ValueError:
        return None


def parse_flp_text(text: str) -> list[Unit]:
    units = []
    for line in text.splitlines():
        t = line.split()
        if not t or t[0].startswith("#"):
            continue
        nums = []
        for tok in t[1:]:
            v = _num(tok)
            if v is None:
                break
            nums.append(v)
        if len(nums) >= 6:
            units.append(Unit(t[0], nums[0], nums[1], nums[2], nums[3], nums[4], nums[5], True))
        elif len(nums) >= 4:
            units.append(Unit(t[0], nums[0], nums[1], nums[2], nums[3]))
    minx = min(u.x for u in units)
    miny = min(u.y for u in units)
    for u in units:            # flp_translate (flp.c:334-350)
        u.x += (0 - minx)
        u.y += (0 - miny)
    return units


def flp_width(units):
    mn = units[0].x
    mx = units[0].x + units[0].w
    for u in units[1:]:
        mn = min(mn, u.x) if u.x < mn else mn
        if u.x + u.w > mx:
            mx = u.x + u.w
    return mx - mn


def flp_height(units):
    mn = units[0].y
    mx = units[0].y + units[0].h
    for u in units[1:]:
        if u.y < mn:
            mn = u.y
        if u.y + u.h > mx:
            mx = u.y + u.h
    return mx - mn


def read_materials(path):
    props = {}
    if not path:
        return props
    toks = [l.split()[0] for l in open(path) if l.split() and not l.split()[0].startswith("#")]
    i = 0
    while i < len(toks):
        name, kind = toks[i], toks[i + 1]
        k, cv = float(toks[i + 2]), float(toks[i + 3])
        mu = float(toks[i + 4]) if kind == "fluid" else 0.0
        props[name] = (k, cv, mu)
        i += 5 if kind == "fluid" else 4
    return props


# ---------------------------------------------------------------------------
# the restated model
# ---------------------------------------------------------------------------
class Layer:
    def __init__(self, no, lateral, power, k, t, sp, flp):
        self.no, self.lateral, self.power, self.k, self.t, self.sp = no, lateral, power, k, t, sp
        self.flp = flp
        self.uchan = None
        self.b2g = None          # shared list-of-lists object
        self.g2b = None
        self.rx = self.ry = self.rz = self.c = 0.0


class _Cell:
    """one blist_t node (temperature_grid.h:63-80)"""
    __slots__ = ("idx", "occ", "lock", "hasRes", "hasCap", "rx", "ry", "rz", "cap")

    def __init__(self, idx, occ):
        self.idx, self.occ = idx, occ
        self.lock = self.hasRes = self.hasCap = 0
        self.rx = self.ry = self.rz = self.cap = 0.0


class _UChan:
    pass


class OracleModel:
    """Grid model set up from a workloads.Scenario, numerics in grid_oracle.c."""

    def __init__(self, sc):
        cfg = dict(DEFAULT_CONFIG)
        mats = read_materials(sc.materials)
        for k, v in sc.config.items():
            if k in cfg:
                cfg[k] = type(cfg[k])(v) if not isinstance(cfg[k], str) else v
        self.cfg = cfg
        self.mats = mats
        u = dict(DEFAULT_UCHAN)
        for k in DEFAULT_UCHAN:
            if k in sc.config:
                u[k] = float(sc.config[k])
        if "coolant_material" in sc.config:
            kk, cv, mu = mats[sc.config["coolant_material"]]
            u["coolant_res"], u["coolant_capac"], u["coolant_visc"] = 1.0 / kk, cv, mu
        self.ucfg = u
        self.nr, self.nc = int(cfg["grid_rows"]), int(cfg["grid_cols"])
        self.secondary = int(cfg["model_secondary"])
        self.d3 = bool(sc.detailed_3D)
        self.use_uc = bool(sc.use_microchannels)
        self.ambient = cfg["ambient"]
        self.init_temp = cfg["init_temp"]
        self.map_mode = cfg["grid_map_mode"].lower()
        self.has_lcf = cfg["grid_layer_file"] != "(null)"
        self._layers(sc)
        self.nl = len(self.layers)
        self.nx = EXTRA + (EXTRA_SEC if self.secondary else 0)
        self.spidx, self.hsidx = self.nl - 2, self.nl - 1
        self.n_blocks = sum(len(L.flp) for L in self.layers)
        self.layer_units = [len(L.flp) for L in self.layers]
        self.layer_power = [bool(L.power) for L in self.layers]
        self.n_cells = self.nl * self.nr * self.nc
        self._populate_R()
        self._populate_C()
        self._y = None

    # -- layers (temperature_grid.c:459-609, :612-892) ----------------------
    def _layers(self, sc):
        cfg = self.cfg
        if not self.has_lcf:
            flp = parse_flp_text(open(sc.flp).read())
            self.width, self.height = flp_width(flp), flp_height(flp)
            si = Layer(0, 1, 1, cfg["k_chip"], cfg["t_chip"], cfg["p_chip"], flp)
            tim = Layer(1, 1, 0, cfg["k_interface"], cfg["t_interface"], cfg["p_interface"], flp)
            si.b2g = [[None] * (self.nr * self.nc)]
            tim.b2g = si.b2g
            layers = [si, tim]
            self.own = [0]
        else:
            layers = []
            self.own = []
            toks = []
            for line in open(cfg["grid_layer_file"]):
                t = line.split()
                if t and not t[0].startswith("#"):
                    toks.append(t[0])
            i = 0
            while i < len(toks):
                no = int(toks[i])
                lat = toks[i + 1][0] in "Yy"
                pw = toks[i + 2][0] in "Yy"
                sp = _num(toks[i + 3])
                if sp is None:
                    k_, cv, _ = self.mats.get(toks[i + 3], (-1.0, -1.0, 0.0))
                    k, sp = k_, cv
                    i += 4
                else:
                    k = 1.0 / float(toks[i + 4])
                    i += 5
                thick = float(toks[i])
                fname = toks[i + 1]
                i += 2
                L = Layer(no, lat, pw, k, thick, sp, None)
                if fname.endswith(".csv") or ".csv" in fname:
                    L.uchan = fname
                else:
                    L.flp = parse_flp_text(open(fname).read())
                layers.append(L)
            first = next(L for L in layers if L.flp is not None)
            self.width, self.height = flp_width(first.flp), flp_height(first.flp)
            for idx, L in enumerate(layers):
                if L.uchan is not None:
                    L.flp = self._build_uchan(L)
                L.b2g = [[None] * (self.nr * self.nc)]
                self.own.append(idx)
        sp = Layer(len(layers), 1, 0, cfg["k_spreader"], cfg["t_spreader"], cfg["p_spreader"], layers[-1].flp)
        hs = Layer(len(layers) + 1, 1, 0, cfg["k_sink"], cfg["t_sink"], cfg["p_sink"], layers[-1].flp)
        sp.b2g = hs.b2g = layers[-1].b2g
        if self.d3:
            sp.b2g = [[None] * (self.nr * self.nc)]
            hs.b2g = sp.b2g
        self.layers = layers + [sp, hs]

    def _build_uchan(self, L):
        """microchannel.c:258-571: cell types, generated floorplan, pressures."""
        u = _UChan()
        for k, v in self.ucfg.items():
            setattr(u, k, v)
        u.cw, u.ch, u.thick = self.width / self.nc, self.height / self.nr, L.t
        rows = []
        for line in open(L.uchan):
            toks = [t for t in line.replace(",", " ").split()]
            rows.append([int(t) for t in toks])
        types = np.array(rows[: self.nr], dtype=np.int32)
        u.types = types
        fluid = np.isin(types, (FLUID, INLET, OUTLET))
        u.fluid = fluid
        lines = ["# Name\tw\th\tx\ty\tc_v\tp"]
        for i in range(self.nr):
            for j in range(self.nc):
                fl = fluid[i, j]
                lines.append("Cell_%d_%d\t%e\t%e\t%e\t%e\t%e\t%e" % (
                    i, j, u.cw, u.ch, j * u.cw, (self.nr - i - 1) * u.ch,
                    u.coolant_capac if fl else u.wall_capac, u.coolant_res if fl else u.wall_res))
        flp = parse_flp_text("\n".join(lines))
        # hydraulic conductance (microchannel.c:361-376)
        h, w, Lc, mu = u.thick, u.cw, u.ch, u.coolant_visc
        if h == w:
            hc = (0.42229 * math.pow(h, 4)) / (12 * mu * Lc)
        elif h > w:
            hc = ((1 - 0.63 * (w / h)) * (math.pow(w, 3)) * (h)) / (12 * mu * Lc)
        else:
            hc = ((1 - 0.63 * (h / w)) * (math.pow(h, 3)) * (w)) / (12 * mu * Lc)
        u.hc = hc
        u.pressure = self._pressures(u)
        L.uc = u
        return flp

    def _pressures(self, u):
        """pressure network (microchannel.c:378-565) solved directly (scipy)."""
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl
        nr, nc = self.nr, self.nc
        idx = -np.ones((nr, nc), dtype=np.int64)
        cells = np.argwhere(u.fluid)
        idx[u.fluid] = np.arange(len(cells))
        n = len(cells)
        ideal = u.pump_internal_res == 0
        npump = 0 if ideal else 1
        rows, cols, vals = [], [], []
        b = np.zeros(n + npump)
        for k, (i, j) in enumerate(cells):
            t = u.types[i, j]
            if t == FLUID or (t == INLET and not ideal):
                d = 0.0
                for di, dj in ((-1, 0), (1, 0), (0, -1), (0, 1)):
                    ii, jj = i + di, j + dj
                    if 0 <= ii < nr and 0 <= jj < nc and u.fluid[ii, jj]:
                        rows.append(k); cols.append(idx[ii, jj]); vals.append(-u.hc)
                        d += -u.hc
                rows.append(k); cols.append(k); vals.append(-d)
            if t == INLET:
                if not ideal:
                    rows.append(k); cols.append(n); vals.append(-1.0 / u.pump_internal_res)
                    rows.append(k); cols.append(k); vals.append(1.0 / u.pump_internal_res)
                else:
                    rows.append(k); cols.append(k); vals.append(1.0)
                    b[k] = u.pumping_pressure
            elif t == OUTLET:
                rows.append(k); cols.append(k); vals.append(1.0)
        if not ideal:
            rows.append(n); cols.append(n); vals.append(1.0)
            b[n] = u.pumping_pressure
        A = sp.csc_matrix((vals, (rows, cols)), shape=(n + npump, n + npump))
        x = spl.spsolve(A, b)
        p = np.full((nr, nc), np.nan)
        p[u.fluid] = x[:n]
        return p

    # -- occupancy maps (set_bgmap, temperature_grid.c:341-456) --------------
    def _bgmap(self, L, units):
        nr, nc = self.nr, self.nc
        cw, ch = self.width / nc, self.height / nr
        cells = [None] * (nr * nc)
        g2b = []
        d3 = self.d3
        for u, U in enumerate(units):
            lu, ru, bu, tu = U.x, U.x + U.w, U.y, U.y + U.h
            i1 = nr - tolerant_ceil(tu / ch)
            i2 = nr - tolerant_floor(bu / ch)
            j1 = tolerant_floor(lu / cw)
            j2 = tolerant_ceil(ru / cw)
            g2b.append((i1, i2, j1, j2))
            res = U.res if (U.has and d3) else 1 / L.k
            sh = U.cp if (U.has and d3) else L.sp
            for i in range(i1, i2):
                for j in range(j1, j2):
                    if i > i1 and i < i2 - 1 and j > j1 and j < j2 - 1:
                        occ, first = 1.0, 1
                    else:
                        lc, rc = j * cw, (j + 1) * cw
                        tc, bc = self.height - i * ch, self.height - (i + 1) * ch
                        oh = (min(tu, tc) - max(bu, bc))
                        ow = (min(ru, rc) - max(lu, lc))
                        if eq(oh / ch, 0):
                            oh = 0
                        elif eq(oh / ch, 1):
                            oh = ch
                        if eq(ow / cw, 0):
                            ow = 0
                        elif eq(ow / cw, 1):
                            ow = cw
                        occ, first = (oh * ow) / (ch * cw), 0
                    node = self._new_node(u, occ, res, sh, 1, d3, cw, ch, L.t)
                    lst = cells[i * nc + j]
                    if lst is None:
                        node.hasRes = 1
                        node.hasCap = int(U.has)
                        cells[i * nc + j] = [node]
                    else:
                        head = lst[0]
                        if d3 and head.lock != 1:      # blist_append :270-289
                            if occ >= 0.95:
                                head.lock = 1
                                head.rx = getr(1 / res, cw, ch * L.t)
                                head.ry = getr(1 / res, ch, cw * L.t)
                                head.rz = getr(1 / res, L.t, cw * ch)
                                head.cap = getcap(sh, L.t, cw * ch)
                            else:
                                head.rx = 1 / ((1 / head.rx) + ((1 / getr(1 / res, cw, ch * L.t)) * occ))
                                head.ry = 1 / ((1 / head.ry) + ((1 / getr(1 / res, ch, cw * L.t)) * occ))
                                head.rz = 1 / ((1 / head.rz) + ((1 / getr(1 / res, L.t, cw * ch)) * occ))
                                head.lock = 0
                        lst.append(self._new_node(u, occ, res, sh, first, d3, cw, ch, L.t))
        return cells, g2b

    @staticmethod
    def _new_node(idx, occ, res, sh, first, d3, cw, ch, t):   # new_blist :190-222
        n = _Cell(idx, occ)
        if first and d3:
            if occ >= 0.95:
                n.lock = 1
                n.rx = getr(1 / res, cw, ch * t)
                n.ry = getr(1 / res, ch, cw * t)
                n.rz = getr(1 / res, t, cw * ch)
            else:
                n.rx = 1 / ((1 / getr(1 / res, cw, ch * t)) * occ)
                n.ry = 1 / ((1 / getr(1 / res, ch, cw * t)) * occ)
                n.rz = 1 / ((1 / getr(1 / res, t, cw * ch)) * occ)
            n.cap = getcap(sh, t, cw * ch)
        return n

    # -- R and C (temperature_grid.c:950-1114, temperature.c:458-569) --------
    def _package(self):
        c, w, h = self.cfg, self.width, self.height
        s_sp, t_sp, s_s, t_s, r_cv = c["s_spreader"], c["t_spreader"], c["s_sink"], c["t_sink"], c["r_convec"]
        s_sub, t_sub, s_so, t_so = c["s_sub"], c["t_sub"], c["s_solder"], c["t_solder"]
        s_pcb, t_pcb, r_cs = c["s_pcb"], c["t_pcb"], c["r_convec_sec"]
        k_s, k_sp, c_cv, c_cs = c["k_sink"], c["k_spreader"], c["c_convec"], c["c_convec_sec"]
        p_s, p_sp = c["p_sink"], c["p_spreader"]
        P = {}
        P["r_sp1_x"] = getr(k_sp, (s_sp - w) / 4.0, (s_sp + 3 * h) / 4.0 * t_sp)
        P["r_sp1_y"] = getr(k_sp, (s_sp - h) / 4.0, (s_sp + 3 * w) / 4.0 * t_sp)
        P["r_hs1_x"] = getr(k_s, (s_sp - w) / 4.0, (s_sp + 3 * h) / 4.0 * t_s)
        P["r_hs1_y"] = getr(k_s, (s_sp - h) / 4.0, (s_sp + 3 * w) / 4.0 * t_s)
        P["r_hs2_x"] = getr(k_s, (s_sp - w) / 4.0, (3 * s_sp + h) / 4.0 * t_s)
        P["r_hs2_y"] = getr(k_s, (s_sp - h) / 4.0, (3 * s_sp + w) / 4.0 * t_s)
        P["r_hs"] = getr(k_s, (s_s - s_sp) / 4.0, (s_s + 3 * s_sp) / 4.0 * t_s)
        P["r_sp_per_x"] = getr(k_sp, t_sp, (s_sp + h) * (s_sp - w) / 4.0)
        P["r_sp_per_y"] = getr(k_sp, t_sp, (s_sp + w) * (s_sp - h) / 4.0)
        P["r_hs_c_per_x"] = getr(k_s, t_s, (s_sp + h) * (s_sp - w) / 4.0)
        P["r_hs_c_per_y"] = getr(k_s, t_s, (s_sp + w) * (s_sp - h) / 4.0)
        P["r_hs_per"] = getr(k_s, t_s, (s_s * s_s - s_sp * s_sp) / 4.0)
        P["r_amb_c_per_x"] = r_cv * (s_s * s_s) / ((s_sp + h) * (s_sp - w) / 4.0)
        P["r_amb_c_per_y"] = r_cv * (s_s * s_s) / ((s_sp + w) * (s_sp - h) / 4.0)
        P["r_amb_per"] = r_cv * (s_s * s_s) / ((s_s * s_s - s_sp * s_sp) / 4.0)
        P["r_sub1_x"] = getr(K_SUB, (s_sub - w) / 4.0, (s_sub + 3 * h) / 4.0 * t_sub)
        P["r_sub1_y"] = getr(K_SUB, (s_sub - h) / 4.0, (s_sub + 3 * w) / 4.0 * t_sub)
        P["r_solder1_x"] = getr(K_SOLDER, (s_so - w) / 4.0, (s_so + 3 * h) / 4.0 * t_so)
        P["r_solder1_y"] = getr(K_SOLDER, (s_so - h) / 4.0, (s_so + 3 * w) / 4.0 * t_so)
        P["r_pcb1_x"] = getr(K_PCB, (s_so - w) / 4.0, (s_so + 3 * h) / 4.0 * t_pcb)
        P["r_pcb1_y"] = getr(K_PCB, (s_so - h) / 4.0, (s_so + 3 * w) / 4.0 * t_pcb)
        P["r_pcb2_x"] = getr(K_PCB, (s_so - w) / 4.0, (3 * s_so + h) / 4.0 * t_pcb)
        P["r_pcb2_y"] = getr(K_PCB, (s_so - h) / 4.0, (3 * s_so + w) / 4.0 * t_pcb)
        P["r_pcb"] = getr(K_PCB, (s_pcb - s_so) / 4.0, (s_pcb + 3 * s_so) / 4.0 * t_pcb)
        P["r_sub_per_x"] = getr(K_SUB, t_sub, (s_sub + h) * (s_sub - w) / 4.0)
        P["r_sub_per_y"] = getr(K_SUB, t_sub, (s_sub + w) * (s_sub - h) / 4.0)
        P["r_solder_per_x"] = getr(K_SOLDER, t_so, (s_so + h) * (s_so - w) / 4.0)
        P["r_solder_per_y"] = getr(K_SOLDER, t_so, (s_so + w) * (s_so - h) / 4.0)
        P["r_pcb_c_per_x"] = getr(K_PCB, t_pcb, (s_so + h) * (s_so - w) / 4.0)
        P["r_pcb_c_per_y"] = getr(K_PCB, t_pcb, (s_so + w) * (s_so - h) / 4.0)
        P["r_pcb_per"] = getr(K_PCB, t_pcb, (s_pcb * s_pcb - s_so * s_so) / 4.0)
        P["r_amb_sec_c_per_x"] = r_cs * (s_pcb * s_pcb) / ((s_so + h) * (s_so - w) / 4.0)
        P["r_amb_sec_c_per_y"] = r_cs * (s_pcb * s_pcb) / ((s_so + w) * (s_so - h) / 4.0)
        P["r_amb_sec_per"] = r_cs * (s_pcb * s_pcb) / ((s_pcb * s_pcb - s_so * s_so) / 4.0)
        P["c_sp_per_x"] = getcap(p_sp, t_sp, (s_sp + h) * (s_sp - w) / 4.0)
        P["c_sp_per_y"] = getcap(p_sp, t_sp, (s_sp + w) * (s_sp - h) / 4.0)
        P["c_hs_c_per_x"] = getcap(p_s, t_s, (s_sp + h) * (s_sp - w) / 4.0)
        P["c_hs_c_per_y"] = getcap(p_s, t_s, (s_sp + w) * (s_sp - h) / 4.0)
        P["c_hs_per"] = getcap(p_s, t_s, (s_s * s_s - s_sp * s_sp) / 4.0)
        P["c_amb_c_per_x"] = C_FACTOR * c_cv / (s_s * s_s) * ((s_sp + h) * (s_sp - w) / 4.0)
        P["c_amb_c_per_y"] = C_FACTOR * c_cv / (s_s * s_s) * ((s_sp + w) * (s_sp - h) / 4.0)
        P["c_amb_per"] = C_FACTOR * c_cv / (s_s * s_s) * ((s_s * s_s - s_sp * s_sp) / 4.0)
        P["c_sub_per_x"] = getcap(SH_SUB, t_sub, (s_sub + h) * (s_sub - w) / 4.0)
        P["c_sub_per_y"] = getcap(SH_SUB, t_sub, (s_sub + w) * (s_sub - h) / 4.0)
        P["c_solder_per_x"] = getcap(SH_SOLDER, t_so, (s_so + h) * (s_so - w) / 4.0)
        P["c_solder_per_y"] = getcap(SH_SOLDER, t_so, (s_so + w) * (s_so - h) / 4.0)
        P["c_pcb_c_per_x"] = getcap(SH_PCB, t_pcb, (s_so + h) * (s_so - w) / 4.0)
        P["c_pcb_c_per_y"] = getcap(SH_PCB, t_pcb, (s_so + w) * (s_so - h) / 4.0)
        P["c_pcb_per"] = getcap(SH_PCB, t_pcb, (s_pcb * s_pcb - s_so * s_so) / 4.0)
        P["c_amb_sec_c_per_x"] = C_FACTOR * c_cs / (s_pcb * s_pcb) * ((s_so + h) * (s_so - w) / 4.0)
        P["c_amb_sec_c_per_y"] = C_FACTOR * c_cs / (s_pcb * s_pcb) * ((s_so + w) * (s_so - h) / 4.0)
        P["c_amb_sec_per"] = C_FACTOR * c_cs / (s_pcb * s_pcb) * ((s_pcb * s_pcb - s_so * s_so) / 4.0)
        return P

    def _populate_R(self):
        nr, nc = self.nr, self.nc
        done = {}
        for L in self.layers:
            key = id(L.b2g)
            if key in done:
                L.cells, L.g2b = done[key]
            else:
                cells, g2b = self._bgmap(L, L.flp)
                done[key] = (cells, g2b)
                L.cells, L.g2b = cells, g2b
        # the spreader/sink map of a detailed model carries no per-cell R/C
        if self.d3:
            for cell in self.layers[self.spidx].cells:
                if cell:
                    cell[0].hasRes = cell[0].hasCap = cell[0].lock = 0
        cw, ch = self.width / nc, self.height / nr
        self.P = self._package()
        for n, L in enumerate(self.layers):
            if L.lateral:
                L.rx = getr(L.k, cw, ch * L.t)
                L.ry = getr(L.k, ch, cw * L.t)
            else:
                L.rx = L.ry = LARGENUM
            L.rz = getr(L.k, L.t, cw * ch)
            if n == self.hsidx:
                L.rz += self.cfg["r_convec"] * (self.cfg["s_sink"] * self.cfg["s_sink"]) / (cw * ch)

    def _populate_C(self):
        cw, ch = self.width / self.nc, self.height / self.nr
        for L in self.layers:
            L.c = getcap(L.sp, L.t, cw * ch)
        self.layers[self.hsidx].c += C_FACTOR * self.cfg["c_convec"] * (cw * ch) / (self.cfg["s_sink"] * self.cfg["s_sink"])
        self._build_core()

    # -- find_res (temperature_grid.c:26-136) --------------------------------
    def _r3(self, n, i, j, choice):
        cell = self.layers[n].cells[i * self.nc + j]
        has = cell[0].hasRes if cell else 0
        L = self.layers[n]
        if choice == 1:
            return cell[0].rx if has else L.rx
        if choice == 2:
            return cell[0].ry if has else L.ry
        return cell[0].rz if has else L.rz

    def _fl(self, n, i, j):
        L = self.layers[n]
        return L.uchan is not None and bool(L.uc.fluid[i, j])

    def find_res(self, n1, i1, j1, n2, i2, j2):
        cw, ch = self.width / self.nc, self.height / self.nr
        htc = 0.0
        f1 = f2 = False
        if self.layers[n1].uchan is not None:
            htc = self.layers[n1].uc.htc
            f1 = self._fl(n1, i1, j1)
        if self.layers[n2].uchan is not None:
            htc = self.layers[n2].uc.htc
            f2 = self._fl(n2, i2, j2)
        if f1 != f2:
            if n1 == 0:
                return self._r3(n1, i1, j1, 3) + (1.0 / (htc * ch * cw)) + 0
            if n2 == 0:
                return self._r3(n2, i2, j2, 3) + (1.0 / (htc * ch * cw)) + 0
            if n1 != n2:
                return ((self._r3(n2, i2, j2, 3) if f1 else self._r3(n1, i1, j1, 3)) / 2.0) + (1.0 / (htc * ch * cw)) + 0
            if i1 != i2:
                th = self.layers[n1].t if f1 else self.layers[n2].t
                return ((self._r3(n2, i2, j2, 1) if f1 else self._r3(n1, i1, j1, 1)) / 2.0) + (1.0 / (htc * cw * th))
            th = self.layers[n1].t if f1 else self.layers[n2].t
            return ((self._r3(n2, i2, j2, 2) if f1 else self._r3(n1, i1, j1, 2)) / 2.0) + (1.0 / (htc * ch * th))
        if self.d3:
            if n1 == 0 and n2 != n1:
                return self._r3(n1, i1, j1, 3) + (self._r3(n2, i2, j2, 3) / 2.0)
            if n2 == 0 and n1 != n2:
                return self._r3(n2, i2, j2, 3) + (self._r3(n1, i1, j1, 3) / 2.0)
            if n1 != n2:
                return (self._r3(n1, i1, j1, 3) / 2.0) + (self._r3(n2, i2, j2, 3) / 2.0)
            if i1 != i2:
                return (self._r3(n1, i1, j1, 1) / 2.0) + (self._r3(n2, i2, j2, 1) / 2.0)
            return (self._r3(n1, i1, j1, 2) / 2.0) + (self._r3(n2, i2, j2, 2) / 2.0)
        L1, L2 = self.layers[n1], self.layers[n2]
        if n1 < n2:
            return L1.rz
        if n1 > n2:
            return L2.rz
        if i1 != i2:
            return (L1.rx / 2.0) + (L2.rx / 2.0)
        return (L1.ry / 2.0) + (L2.ry / 2.0)

    def _flow(self, u, i1, j1, i2, j2):      # microchannel.c:567-571
        return (u.pressure[i1, j1] - u.pressure[i2, j2]) * u.hc

    def _build_core(self):
        nl, nr, nc = self.nl, self.nr, self.nc
        N = self.n_cells
        self.field = self.d3 or any(L.uchan is not None for L in self.layers)
        self.arr = {}
        if self.field:
            a = np.zeros((7, N))
            c = 0
            for n in range(nl):
                for i in range(nr):
                    for j in range(nc):
                        if i > 0: a[0, c] = self.find_res(n, i - 1, j, n, i, j)
                        if i < nr - 1: a[1, c] = self.find_res(n, i + 1, j, n, i, j)
                        if j > 0: a[2, c] = self.find_res(n, i, j - 1, n, i, j)
                        if j < nc - 1: a[3, c] = self.find_res(n, i, j + 1, n, i, j)
                        if n > 0: a[4, c] = self.find_res(n - 1, i, j, n, i, j)
                        if n < nl - 1: a[5, c] = self.find_res(n + 1, i, j, n, i, j)
                        cell = self.layers[n].cells[i * nc + j]
                        a[6, c] = cell[0].cap if (cell and cell[0].lock == 1) else self.layers[n].c
                        c += 1
            self.arr["cells"] = a
        adv = None
        for n, L in enumerate(self.layers):
            if L.uchan is None:
                continue
            if adv is None:
                adv = np.zeros((6, N))
            u = L.uc
            fl = u.fluid
            Cv = u.coolant_capac
            for i in range(nr):
                for j in range(nc):
                    if not fl[i, j]:
                        continue
                    c = (n * nr + i) * nc + j
                    if i > 0 and fl[i - 1, j]: adv[0, c] = Cv * self._flow(u, i - 1, j, i, j)
                    if i < nr - 1 and fl[i + 1, j]: adv[1, c] = Cv * self._flow(u, i + 1, j, i, j)
                    if j > 0 and fl[i, j - 1]: adv[2, c] = Cv * self._flow(u, i, j - 1, i, j)
                    if j < nc - 1 and fl[i, j + 1]: adv[3, c] = Cv * self._flow(u, i, j + 1, i, j)
                    t = u.types[i, j]
                    if t in (INLET, OUTLET):
                        rate = 0
                        if i == 0: order = [(0, -1), (0, 1), (1, 0)]
                        elif i == nr - 1: order = [(0, -1), (0, 1), (-1, 0)]
                        elif j == 0: order = [(0, 1), (-1, 0), (1, 0)]
                        elif j == nc - 1: order = [(0, -1), (-1, 0), (1, 0)]
                        else: order = []
                        for di, dj in order:
                            ii, jj = i + di, j + dj
                            if 0 <= ii < nr and 0 <= jj < nc and fl[ii, jj]:
                                rate += self._flow(u, ii, jj, i, j)
                        rate *= -1
                        if t == INLET:
                            adv[5, c] = u.coolant_capac * rate * u.inlet_temperature
                        else:
                            adv[4, c] = u.coolant_capac * rate
        if adv is not None:
            self.arr["adv"] = adv
        self.rx = np.array([L.rx for L in self.layers])
        self.ry = np.array([L.ry for L in self.layers])
        self.rz = np.array([L.rz for L in self.layers])
        self.c = np.array([L.c for L in self.layers])
        self.pack = np.array([self.P[f] for f in PACK_FIELDS])
        self._cmodel = None

    # -- block <-> grid (xlate_vector_b2g / xlate_temp_g2b) -------------------
    def _b2g_ranks(self):
        """per list position r: (cells, global block, occupancy, block area),
        so sums run over each cell's list in the reference's order"""
        if getattr(self, "_ranks", None) is None:
            nr, nc = self.nr, self.nc
            ranks, base = [], 0
            for n, L in enumerate(self.layers):
                for k in range(nr * nc):
                    for r, node in enumerate(L.cells[k] or []):
                        while len(ranks) <= r:
                            ranks.append(([], [], [], []))
                        u = L.flp[node.idx]
                        ranks[r][0].append(n * nr * nc + k)
                        ranks[r][1].append(base + node.idx)
                        ranks[r][2].append(node.occ)
                        ranks[r][3].append(u.w * u.h)
                base += len(L.flp)
            self._ranks = [tuple(np.array(a) for a in rk) for rk in ranks]
        return self._ranks

    def b2g(self, b, power=True):
        """xlate_vector_b2g (temperature_grid.c:1888-1929)"""
        nr, nc = self.nr, self.nc
        area = (self.width * self.height) / (nc * nr)
        g = np.zeros(self.n_cells + self.nx)
        val = np.zeros(self.n_cells)
        for cells, blk, occ, wh in self._b2g_ranks():
            val[cells] += (occ * b[blk] / wh) if power else (occ * b[blk])
        g[:self.n_cells] = val * area if power else val
        g[self.n_cells:] = b[self.n_blocks:self.n_blocks + self.nx]
        return g

    def g2b(self, g):
        """xlate_temp_g2b (temperature_grid.c:1932-2015)"""
        nr, nc = self.nr, self.nc
        out = np.zeros(self.n_blocks + self.nx)
        base = 0
        for n, L in enumerate(self.layers):
            G = g[n * nr * nc:(n + 1) * nr * nc].reshape(nr, nc)
            for u, (i1, i2, j1, j2) in enumerate(L.g2b):
                if self.map_mode == "center":
                    ci1, cj1 = (i1 + i2) // 2, (j1 + j2) // 2
                    ci2 = ci1 - (0 if (i2 - i1) % 2 else 1)
                    cj2 = cj1 - (0 if (j2 - j1) % 2 else 1)
                    out[base + u] = (G[ci1, cj1] + G[ci2, cj1] + G[ci1, cj2] + G[ci2, cj2]) / 4
                    continue
                blk = G[i1:i2, j1:j2].ravel()
                if self.map_mode == "avg":
                    out[base + u] = np.cumsum(blk)[-1] / blk.size     # sequential row-major sum
                elif self.map_mode == "min":
                    out[base + u] = blk.min()
                else:
                    out[base + u] = blk.max()
            base += len(L.flp)
        out[self.n_blocks:] = g[self.n_cells:]
        return out

    # -- driver API (mirrors compute_temp / steady_state_temp) ---------------
    def vector(self, fill: float = 0.0):
        return np.full(self.n_blocks + self.nx, fill)

    def power_vector(self, row):
        p = self.vector()
        base = k = 0
        for l in range(self.nl):
            n = self.layer_units[l]
            if self.layer_power[l]:
                p[base:base + n] = row[k:k + n]
                k += n
            base += n
        return p

    def _core(self):
        if self._cmodel is None:
            self._cmodel = _CModel(self)
        return self._cmodel

    def compute_temp(self, power, temp, dt):
        power[self.n_blocks:] = 0.0
        p = self.b2g(power, True)
        if temp is not None:
            self._y = self.b2g(temp, False)
            self._last_temp = temp
        steps = self._core().compute_temp(self._y, p, dt)
        self._last_temp[:] = self.g2b(self._y)
        return steps

    def steady(self, power, temp, max_sweeps: int = 50_000_000):
        power[self.n_blocks:] = 0.0
        p = self.b2g(power, True)
        v = np.zeros(self.n_cells + self.nx)
        sweeps = self._core().steady(v, p, max_sweeps)
        self._steady = v
        temp[:] = self.g2b(v)
        return sweeps

    def grid(self, which="trans"):
        return (self._y if which == "trans" else self._steady).copy()

    def slope(self, y, p):
        return self._core().slope(y, p)

    # -- the steady system as a sparse matrix (temperature_grid.c:5196-6694) --
    def steady_system(self, power_grid):
        """G, P of G T = P: conduction, package, ambient and advection terms."""
        import scipy.sparse as sp
        nl, nr, nc, nx = self.nl, self.nr, self.nc, self.nx
        N = self.n_cells
        cw, ch = self.width / nc, self.height / nr
        Pk = self.P
        rows, cols, vals = [], [], []
        P = power_grid[:N + nx].copy()
        P[N:] = 0.0
        adv = self.arr.get("adv")
        cellsR = self.arr.get("cells")

        def add(r, c, v):
            rows.append(r); cols.append(c); vals.append(v)
        edge = {}
        for n in range(nl):
            L = self.layers[n]
            if n == self.spidx:
                edge[n] = ((L.ry / 2.0 + nc * Pk["r_sp1_y"]), (L.rx / 2.0 + nr * Pk["r_sp1_x"]),
                           (SP_N, SP_S, SP_E, SP_W))
            elif n == self.hsidx:
                edge[n] = ((L.ry / 2.0 + nc * Pk["r_hs1_y"]), (L.rx / 2.0 + nr * Pk["r_hs1_x"]),
                           (SINK_C_N, SINK_C_S, SINK_C_E, SINK_C_W))
        for n in range(nl):
            L = self.layers[n]
            for i in range(nr):
                for j in range(nc):
                    c = (n * nr + i) * nc + j
                    dia = 0.0
                    nb = []
                    if cellsR is not None:
                        R = cellsR[:, c]
                    else:
                        R = [self.find_res(n, i - 1, j, n, i, j) if i > 0 else 0,
                             self.find_res(n, i + 1, j, n, i, j) if i < nr - 1 else 0,
                             self.find_res(n, i, j - 1, n, i, j) if j > 0 else 0,
                             self.find_res(n, i, j + 1, n, i, j) if j < nc - 1 else 0,
                             self.find_res(n - 1, i, j, n, i, j) if n > 0 else 0,
                             self.find_res(n + 1, i, j, n, i, j) if n < nl - 1 else 0]
                    if i > 0: nb.append((c - nc, R[0], 0))
                    if i < nr - 1: nb.append((c + nc, R[1], 1))
                    if j > 0: nb.append((c - 1, R[2], 2))
                    if j < nc - 1: nb.append((c + 1, R[3], 3))
                    if n > 0: nb.append((c - nr * nc, R[4], -1))
                    if n < nl - 1: nb.append((c + nr * nc, R[5], -1))
                    for (k, r, d) in nb:
                        J = 0.0
                        if adv is not None and d >= 0:
                            J = -adv[d, c] / 2.0
                        add(c, k, -1.0 / r + J)
                        dia += 1.0 / r
                    if adv is not None:
                        dia += -(adv[0, c] + adv[1, c] + adv[2, c] + adv[3, c]) / 2.0
                        dia += -adv[4, c]
                        P[c] += adv[5, c]
                    if n in edge:
                        Rns, Rew, (eN, eS, eE, eW) = edge[n]
                        if i == 0: add(c, N + eN, -1.0 / Rns); dia += 1.0 / Rns
                        if i == nr - 1: add(c, N + eS, -1.0 / Rns); dia += 1.0 / Rns
                        if j == nc - 1: add(c, N + eE, -1.0 / Rew); dia += 1.0 / Rew
                        if j == 0: add(c, N + eW, -1.0 / Rew); dia += 1.0 / Rew
                    if n == self.hsidx:
                        dia += 1.0 / L.rz
                        P[c] += self.ambient / L.rz
                    add(c, c, dia)
        amb = self.ambient
        # package rows: the same couplings as slope_fn_pack, as conductances
        def link(a, b, r):
            add(N + a, N + b, -1.0 / r); add(N + a, N + a, 1.0 / r)
        def amb_link(a, r):
            add(N + a, N + a, 1.0 / r); P[N + a] += amb / r
        for (o, ci, rr) in ((SINK_N, SINK_C_N, "y"), (SINK_S, SINK_C_S, "y"), (SINK_W, SINK_C_W, "x"), (SINK_E, SINK_C_E, "x")):
            amb_link(o, Pk["r_hs_per"] + Pk["r_amb_per"])
            link(o, ci, Pk["r_hs2_" + rr] + Pk["r_hs"])
        for (ci, spn, o, rr, lay, which) in ((SINK_C_N, SP_N, SINK_N, "y", self.hsidx, "N"),
                                            (SINK_C_S, SP_S, SINK_S, "y", self.hsidx, "S"),
                                            (SINK_C_W, SP_W, SINK_W, "x", self.hsidx, "W"),
                                            (SINK_C_E, SP_E, SINK_E, "x", self.hsidx, "E")):
            self._edge_rows(add, N, ci, lay, which, edge)
            amb_link(ci, Pk["r_hs_c_per_" + rr] + Pk["r_amb_c_per_" + rr])
            link(ci, spn, Pk["r_sp_per_" + rr])
            link(ci, o, Pk["r_hs2_" + rr] + Pk["r_hs"])
        for (spn, ci, rr, which) in ((SP_N, SINK_C_N, "y", "N"), (SP_S, SINK_C_S, "y", "S"),
                                     (SP_W, SINK_C_W, "x", "W"), (SP_E, SINK_C_E, "x", "E")):
            self._edge_rows(add, N, spn, self.spidx, which, edge)
            link(spn, ci, Pk["r_sp_per_" + rr])
        G = sp.csr_matrix((vals, (rows, cols)), shape=(N + nx, N + nx))
        return G, P

    def _edge_rows(self, add, N, node, layer, which, edge):
        nr, nc = self.nr, self.nc
        Rns, Rew, _ = edge[layer]
        R = Rns if which in "NS" else Rew
        if which == "N": cells = [(layer * nr + 0) * nc + j for j in range(nc)]
        elif which == "S": cells = [(layer * nr + nr - 1) * nc + j for j in range(nc)]
        elif which == "W": cells = [(layer * nr + i) * nc + 0 for i in range(nr)]
        else: cells = [(layer * nr + i) * nc + nc - 1 for i in range(nr)]
        for c in cells:
            add(N + node, c, -1.0 / R)
            add(N + node, N + node, 1.0 / R)

    def steady_direct(self, power):
        """Converged FP64 steady state by sparse LU (SuperLU via scipy)."""
        import scipy.sparse.linalg as spl
        power = power.copy()
        power[self.n_blocks:] = 0.0
        G, P = self.steady_system(self.b2g(power, True))
        T = spl.splu(G.tocsc()).solve(P)
        return T, self.g2b(T)


# ---------------------------------------------------------------------------
# ctypes bridge to grid_oracle.c
# ---------------------------------------------------------------------------
class _OrcModel(C.Structure):
    _fields_ = [("nl", C.c_int), ("nr", C.c_int), ("nc", C.c_int), ("nx", C.c_int),
                ("spidx", C.c_int), ("hsidx", C.c_int), ("subidx", C.c_int), ("solderidx", C.c_int),
                ("pcbidx", C.c_int), ("field", C.c_int), ("adv", C.c_int),
                ("ambient", C.c_double), ("width", C.c_double), ("height", C.c_double),
                ("pcb_amb_num", C.c_double)] + \
               [(k, C.POINTER(C.c_double)) for k in ("rx", "ry", "rz", "c", "pack", "rN", "rS", "rW", "rE", "rA",
                                                     "rB", "cap", "aN", "aS", "aW", "aE", "aO", "qin")]


_olib = None
LIB_X87 = os.path.join(HERE, "_build", "libgrid_oracle_x87.so")


def olib():
    global _olib
    if _olib is None:
        _olib = _load(LIB_PATH, "restatement")
    return _olib


@contextlib.contextmanager
def x87_rounding():
    """Oracle calls made inside this block run the restatement compiled with
    x87 80-bit intermediates: the same algorithm with different roundings.
    The spread between the two builds is how far FP64 rounding alone moves a
    result, the floor for comparing two FP64 evaluation orders on
    ill-conditioned inputs (long intervals whose rejected attempts feed
    k1 = f(t1) into the retry, RCutil.c:557-571)."""
    global _olib
    keep = _olib
    _olib = _load(LIB_X87, "restatement-x87")
    try:
        yield
    finally:
        _olib = keep


def _load(path, target):
    if not os.path.exists(path):
        subprocess.run(["make", "-C", HERE, target], check=True, capture_output=True)
    L = C.CDLL(path)
    P = C.POINTER(_OrcModel)
    D = C.POINTER(C.c_double)
    L.orc_slope.argtypes = [P, D, D, D]
    L.orc_rk4.argtypes = [P, D, D, D]
    L.orc_rk4.restype = C.c_double
    L.orc_compute_temp.argtypes = [P, D, D, C.c_double]
    L.orc_compute_temp.restype = C.c_longlong
    L.orc_steady.argtypes = [P, D, D, C.c_longlong]
    L.orc_steady.restype = C.c_longlong
    L.orc_gs_sweep.argtypes = [P, D, D]
    L.orc_gs_sweep.restype = C.c_double
    return L


def _d(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class _CModel:
    def __init__(self, om: OracleModel):
        self.keep = []
        m = _OrcModel()
        m.nl, m.nr, m.nc, m.nx = om.nl, om.nr, om.nc, om.nx
        m.spidx, m.hsidx = om.spidx, om.hsidx
        m.subidx, m.solderidx, m.pcbidx = (2, 1, 0) if om.secondary else (-1, -1, -1)
        m.field = int(om.field)
        m.ambient, m.width, m.height = om.ambient, om.width, om.height
        m.pcb_amb_num = om.cfg["r_convec_sec"] * (om.cfg["s_pcb"] * om.cfg["s_pcb"])

        def keep(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            self.keep.append(a)
            return _d(a)
        m.rx, m.ry, m.rz, m.c, m.pack = keep(om.rx), keep(om.ry), keep(om.rz), keep(om.c), keep(om.pack)
        if om.field:
            a = om.arr["cells"]
            m.rN, m.rS, m.rW, m.rE, m.rA, m.rB, m.cap = [keep(a[k]) for k in range(7)]
        if "adv" in om.arr:
            a = om.arr["adv"]
            m.adv = 1
            m.aN, m.aS, m.aW, m.aE, m.aO, m.qin = [keep(a[k]) for k in range(6)]
        self.m = m

    def compute_temp(self, y, p, dt):
        return olib().orc_compute_temp(C.byref(self.m), _d(y), _d(p), dt)

    def steady(self, v, p, cap):
        r = olib().orc_steady(C.byref(self.m), _d(v), _d(p), cap)
        if r < 0:
            raise RuntimeError("oracle Gauss-Seidel hit its sweep cap")
        return r

    def slope(self, y, p):
        out = np.empty_like(y)
        olib().orc_slope(C.byref(self.m), _d(np.ascontiguousarray(y)), _d(np.ascontiguousarray(p)), _d(out))
        return out
