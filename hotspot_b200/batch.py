"""Batches of grid models advanced together on one GPU (libhotspot_b200's
hsb_batch_* entry points): every model keeps its own adaptive RK4 step
sequence, and one persistent launch advances them all by K sampling
intervals."""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from ._abi import HotspotError, lib


def _check(rc: int):
    if rc != 0:
        raise HotspotError(lib().hsb_dev_last_error().decode(errors="replace").strip())


class Batch:
    """A batch over existing :class:`hotspot_b200.model.RCModel` objects."""

    def __init__(self, models):
        self.models = list(models)
        n = len(self.models)
        devs = (C.c_void_p * n)(*[lib().hsb_grid_device(m.ptr) for m in self.models])
        self.ptr = C.c_void_p()
        _check(lib().hsb_batch_create(C.byref(self.ptr), devs, n))
        self.n_cells = sum(m.n_cells for m in self.models)

    def transient(self, block_powers, dt: float) -> dict:
        """Advance every model by one interval of ``dt`` seconds; ``block_powers``
        is one block power vector per model (or None to keep the last powers)."""
        st = _abi.Stats()
        if block_powers is None:
            _check(lib().hsb_batch_transient(self.ptr, None, dt, C.byref(st)))
        else:
            flat = np.ascontiguousarray(np.concatenate(block_powers), dtype=np.float64)
            _check(lib().hsb_batch_transient(self.ptr, _abi.dptr(flat), dt, C.byref(st)))
        return st.as_dict()

    def trace(self, rows, dt: float) -> dict:
        """Advance every model by len(rows) intervals of ``dt`` seconds in one
        launch; ``rows[k]`` is interval k's list of block power vectors (one per model)."""
        flat = np.ascontiguousarray(np.stack([np.concatenate(r) for r in rows]), dtype=np.float64)
        st = _abi.Stats()
        _check(lib().hsb_batch_transient_trace(self.ptr, _abi.dptr(flat), int(flat.shape[0]), dt, C.byref(st)))
        return st.as_dict()

    def run_subset(self, chips, rows, dt: float) -> dict:
        """Advance only the models ``chips`` (indices) by len(rows) intervals in
        one launch; ``rows[k]`` is interval k's list of their block power
        vectors, in the order of ``chips``."""
        idx = np.ascontiguousarray(chips, dtype=np.int32)
        flat = np.ascontiguousarray(np.stack([np.concatenate(r) for r in rows]), dtype=np.float64)
        st = _abi.Stats()
        _check(lib().hsb_batch_run_subset(self.ptr, idx.ctypes.data_as(C.POINTER(C.c_int)), int(idx.size),
                                          _abi.dptr(flat), int(flat.shape[0]), dt, C.byref(st)))
        return st.as_dict()

    def set_ctas(self, ctas: int):
        """At most ``ctas`` CTAs per launch (0: every co-resident CTA)."""
        _check(lib().hsb_batch_set_ctas(self.ptr, int(ctas)))

    def set_schedule(self, policy: int, split: float = 1.0):
        """Tile policy (0, 1, 2; see hsb_batch_set_schedule) and CTA-group split."""
        _check(lib().hsb_batch_set_schedule(self.ptr, int(policy), float(split)))

    def info(self) -> dict:
        g, cells, pol, split = C.c_int(), C.c_longlong(), C.c_int(), C.c_double()
        _check(lib().hsb_batch_info(self.ptr, C.byref(g), C.byref(cells), C.byref(pol), C.byref(split)))
        return {"grid": g.value, "cells": cells.value, "policy": pol.value, "split": split.value}

    def tile(self, c: int) -> tuple[int, int]:
        r, cc = C.c_int(), C.c_int()
        _check(lib().hsb_batch_chip_tile(self.ptr, int(c), C.byref(r), C.byref(cc)))
        return r.value, cc.value

    def autotune(self, enable: bool = True):
        """Let the next calls try candidate schedules on the real work and keep the fastest."""
        _check(lib().hsb_batch_autotune(self.ptr, int(enable)))

    def tuning(self) -> list[dict]:
        buf = np.zeros(4 * 64)
        n = lib().hsb_batch_tuning(self.ptr, _abi.dptr(buf), 64)
        return [{"policy": int(buf[4 * k]), "split": float(buf[4 * k + 1]),
                 "ms_per_gcell_step": float(buf[4 * k + 3])} for k in range(n)]

    def chip_steps(self) -> np.ndarray:
        out = (C.c_longlong * len(self.models))()
        _check(lib().hsb_batch_chip_steps(self.ptr, out))
        return np.array(out[:], dtype=np.int64)

    def close(self):
        if self.ptr:
            lib().hsb_batch_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
