"""ctypes driver for the reference HotSpot build in ``oracle/_ref`` -- TEST INFRASTRUCTURE.

``oracle/_ref/libhsref.so`` is the reference's own C sources (compiled where
they lie by ``make -C oracle ref``) plus ``oracle/ref_harness.c``.  Only the
tests, ``__graft_entry__.smoke`` and ``bench.py``'s CPU-baseline leg load it,
and only as the oracle / the timed reference arm.  It does not exist unless
the reference sources were present when it was built; callers check
``available()`` first.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libhsref.so")
HOTSPOT_BIN = os.path.join(HERE, "_ref", "hotspot")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, dp, ip, d, i = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int), C.c_double, C.c_int
        L.ref_create.restype = vp
        L.ref_create.argtypes = [C.c_char_p, i, C.POINTER(C.c_char_p), C.POINTER(C.c_char_p), i, i, C.c_char_p]
        L.ref_populate.argtypes = [vp, i]
        L.ref_info.argtypes = [vp, ip]
        L.ref_layer_info.argtypes = [vp, i, ip, ip]
        L.ref_unit_name.argtypes = [vp, i, i]
        L.ref_unit_name.restype = C.c_char_p
        L.ref_layer_params.argtypes = [vp, dp]
        L.ref_package.argtypes = [vp, dp]
        L.ref_dims.argtypes = [vp, dp]
        L.ref_compute_temp.argtypes = [vp, dp, dp, d]
        L.ref_steady.argtypes = [vp, dp, dp]
        L.ref_get_grid.argtypes = [vp, i, dp]
        L.ref_set_grid.argtypes = [vp, i, dp]
        L.ref_power_grid.argtypes = [vp, dp, dp]
        L.ref_slope.argtypes = [vp, dp, dp, dp]
        L.ref_gs_converge.argtypes = [vp, dp, d, i]
        L.ref_gs_converge.restype = i
        L.ref_find_res.argtypes = [vp, i, i, i, i, i, i]
        L.ref_find_res.restype = d
        L.ref_find_cap.argtypes = [vp, i, i, i]
        L.ref_find_cap.restype = d
        L.ref_uchan.argtypes = [vp, i, ip, dp]
        L.ref_uchan.restype = d
        L.ref_flow_rate.argtypes = [vp, i, i, i, i, i]
        L.ref_flow_rate.restype = d
        L.ref_destroy.argtypes = [vp]
        _lib = L
    return _lib


def _dp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class RefModel:
    """The reference grid model built from a :class:`hotspot_b200.workloads.Scenario`."""

    def __init__(self, sc, populate_c: bool = True):
        L = lib()
        names = list(sc.config.keys())
        vals = [str(sc.config[k]) for k in names]
        arr_n = (C.c_char_p * len(names))(*[n.encode() for n in names])
        arr_v = (C.c_char_p * len(vals))(*[v.encode() for v in vals])
        self.h = L.ref_create((sc.flp or "").encode(), len(names), arr_n, arr_v,
                              int(sc.detailed_3D), int(sc.use_microchannels),
                              (sc.materials or "").encode())
        L.ref_populate(self.h, int(populate_c))
        info = (C.c_int * 6)()
        L.ref_info(self.h, info)
        self.nl, self.nr, self.nc, self.n_blocks, self.n_extra, self.has_lcf = list(info)
        self.n_cells = self.nl * self.nr * self.nc
        self.vlen = self.n_blocks + self.n_extra
        self.layer_units = []
        self.layer_power = []
        for l in range(self.nl):
            nu, hp = C.c_int(), C.c_int()
            L.ref_layer_info(self.h, l, C.byref(nu), C.byref(hp))
            self.layer_units.append(nu.value)
            self.layer_power.append(bool(hp.value))

    # -- block-vector helpers -------------------------------------------------
    def vector(self, fill: float = 0.0) -> np.ndarray:
        return np.full(self.vlen, fill, dtype=np.float64)

    def unit_names(self, l: int) -> list[str]:
        return [lib().ref_unit_name(self.h, l, u).decode() for u in range(self.layer_units[l])]

    def power_vector(self, row: np.ndarray) -> np.ndarray:
        """Scatter one trace row (power layers' blocks in floorplan order) into a block vector."""
        p = self.vector()
        base, k = 0, 0
        for l in range(self.nl):
            n = self.layer_units[l]
            if self.layer_power[l]:
                p[base:base + n] = row[k:k + n]
                k += n
            base += n
        return p

    # -- solver calls -----------------------------------------------------------
    def compute_temp(self, power: np.ndarray, temp: np.ndarray | None, dt: float):
        lib().ref_compute_temp(self.h, _dp(power), _dp(temp) if temp is not None else None, dt)

    def steady(self, power: np.ndarray, temp: np.ndarray):
        lib().ref_steady(self.h, _dp(power), _dp(temp))

    def grid(self, which: str = "trans") -> np.ndarray:
        out = np.empty(self.n_cells + self.n_extra)
        lib().ref_get_grid(self.h, 0 if which == "trans" else 1, _dp(out))
        return out

    def set_grid(self, which: str, v: np.ndarray):
        v = np.ascontiguousarray(v, dtype=np.float64)
        lib().ref_set_grid(self.h, 0 if which == "trans" else 1, _dp(v))

    def power_grid(self, power: np.ndarray) -> np.ndarray:
        out = np.empty(self.n_cells + self.n_extra)
        p = power.copy()
        lib().ref_power_grid(self.h, _dp(p), _dp(out))
        return out

    def slope(self, y: np.ndarray, pgrid: np.ndarray) -> np.ndarray:
        out = np.empty(self.n_cells + self.n_extra)
        lib().ref_slope(self.h, _dp(np.ascontiguousarray(y)), _dp(np.ascontiguousarray(pgrid)), _dp(out))
        return out

    def gs_converge(self, power: np.ndarray, tol: float = 1e-13, max_sweeps: int = 10_000_000) -> int:
        p = power.copy()
        return lib().ref_gs_converge(self.h, _dp(p), tol, max_sweeps)

    def layer_params(self) -> np.ndarray:
        out = np.empty((self.nl, 10))
        lib().ref_layer_params(self.h, _dp(out))
        return out

    def package(self) -> np.ndarray:
        out = np.empty(52)
        lib().ref_package(self.h, _dp(out))
        return out

    def dims(self) -> tuple[float, float]:
        out = np.empty(2)
        lib().ref_dims(self.h, _dp(out))
        return float(out[0]), float(out[1])

    def find_res(self, n1, i1, j1, n2, i2, j2) -> float:
        return lib().ref_find_res(self.h, n1, i1, j1, n2, i2, j2)

    def find_cap(self, n, i, j) -> float:
        return lib().ref_find_cap(self.h, n, i, j)

    def uchan(self, l: int):
        t = np.empty(self.nr * self.nc, dtype=np.int32)
        p = np.empty(self.nr * self.nc)
        hc = lib().ref_uchan(self.h, l, t.ctypes.data_as(C.POINTER(C.c_int)), _dp(p))
        return t.reshape(self.nr, self.nc), p.reshape(self.nr, self.nc), hc

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None
