"""The grid dumps' row writer (hsb_format_grid_rows) against "%d\\t%.2f\\n".

dump_steady_temp_grid and dump_transient_temp_grid print one row per cell
(temperature_grid.c:1262-1319); the library writes them without a printf per
value.  Python's "%.2f" is correctly rounded, as glibc's printf is, so the
rows must match it byte for byte: on temperatures, on exact rounding ties
and values next to them, and on the values that take the snprintf path
(negative, large, inf, nan)."""
import ctypes as C

import numpy as np

from hotspot_b200 import _abi


def _rows(v):
    v = np.ascontiguousarray(v, dtype=np.float64)
    cap = 400 * len(v) + 1
    buf = C.create_string_buffer(cap)
    n = _abi.lib().hsb_format_grid_rows(v.ctypes.data_as(C.POINTER(C.c_double)), len(v), buf, cap)
    assert n >= 0
    return buf.raw[:n].decode()


def _expected(v):
    return "".join("%d\t%.2f\n" % (k, x) for k, x in enumerate(v))


def test_temperatures_match_printf():
    rng = np.random.default_rng(5)
    v = np.concatenate([rng.uniform(250.0, 450.0, 20000), rng.uniform(0.0, 10.0, 2000),
                        rng.uniform(1e5, 9.99e6, 2000)])
    assert _rows(v) == _expected(v)


def test_ties_and_neighbours_match_printf():
    base = np.array([333.125, 333.135, 300.005, 0.005, 0.015, 1.005, 2.675, 1234.565, 0.125, 99.995])
    v = np.concatenate([base, np.nextafter(base, 0), np.nextafter(base, 1e9),
                        np.round(np.random.default_rng(6).uniform(250, 450, 5000), 3)])
    assert _rows(v) == _expected(v)


def test_fallback_values_match_printf():
    v = np.array([-0.001, -1.234, -0.0, 0.0, 1e7, 123456789.125, 1e300, np.inf, -np.inf, np.nan, 5e-324])
    assert _rows(v) == _expected(v)


def test_short_buffer_is_refused():
    v = np.ones(10)
    buf = C.create_string_buffer(100)
    assert _abi.lib().hsb_format_grid_rows(v.ctypes.data_as(C.POINTER(C.c_double)), 10, buf, 100) < 0
