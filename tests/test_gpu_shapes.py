"""Grids that are not square, and planes narrower than one 32x8 tile.

HotSpot accepts any power-of-two row and column counts
(temperature_grid.c:901-905), not only square grids, so every form runs on
32 x 64 (wider than tall) and 64 x 16 (16 columns: every tile of the fast
kernels is a partial one) and is checked against the oracle:
- the parity form, transient and steady, to 1e-6 K;
- the fast transient, interval by interval and as one multi-interval call
  (bit-identical to each other), to 0.01 K of the FP64 replay;
- the fast steady solve (MG-PCG; the level hierarchy stops when a side gets
  below 8 columns) to 0.01 K of the sparse direct solution.
"""
import numpy as np
import pytest

from hotspot_b200 import FORM_FAST
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from oracle.restatement import OracleModel

pytestmark = pytest.mark.gpu
SHAPES = [(32, 64), (64, 16)]


def _scenario(workdir, rows, cols, seed):
    sc = W.scenario_chip2d(workdir, seed=seed, grid=rows, steps=6)
    sc.config["grid_cols"] = str(cols)
    return sc


@pytest.mark.parametrize("rows,cols", SHAPES)
def test_parity_form(workdir, rows, cols):
    sc = _scenario(workdir, rows, cols, 61)
    m, o = hm.from_scenario(sc), OracleModel(sc)
    assert m.n_cells % (rows * cols) == 0 and m.n_cells // (rows * cols) >= 1   # every layer has rows x cols cells
    t, to = m.vector(o.init_temp), o.vector(o.init_temp)
    for k in range(sc.steps):
        p = m.power_vector(sc.block_power[k])
        m.compute_temp(p.copy(), t if k == 0 else None, sc.dt)
        o.compute_temp(p.copy(), to if k == 0 else None, sc.dt)
    assert np.max(np.abs(t - to)) <= 1e-6
    assert np.max(np.abs(m.grid("trans") - o.grid("trans"))) <= 1e-6
    avg = m.power_vector(sc.block_power.mean(0))
    s, so = m.vector(), o.vector()
    m.steady(avg.copy(), s)
    o.steady(avg.copy(), so)
    assert np.max(np.abs(s - so)) <= 1e-6
    m.close()


@pytest.mark.parametrize("rows,cols", SHAPES)
def test_fast_forms(workdir, rows, cols):
    sc = _scenario(workdir, rows, cols, 62)
    a, b, o = hm.from_scenario(sc), hm.from_scenario(sc), OracleModel(sc)
    a.set_solver(FORM_FAST)
    t, to = a.vector(o.init_temp), o.vector(o.init_temp)
    powers = np.stack([a.power_vector(sc.block_power[k]) for k in range(sc.steps)])
    for k in range(sc.steps):
        a.compute_temp(powers[k].copy(), t if k == 0 else None, sc.dt)
        o.compute_temp(powers[k].copy(), to if k == 0 else None, sc.dt)
        assert np.max(np.abs(t - to)) <= 0.01
    assert np.max(np.abs(a.grid("trans") - o.grid("trans"))) <= 0.01
    out, _ = b.compute_trace(powers, b.vector(o.init_temp), sc.dt)
    assert np.array_equal(out, t)
    # steady: MG-PCG against the converged FP64 solution
    avg = a.power_vector(sc.block_power.mean(0))
    s = a.vector()
    a.steady(avg.copy(), s)
    T, Tb = o.steady_direct(avg)
    assert np.max(np.abs(s - Tb)) <= 0.01
    assert np.max(np.abs(a.grid("steady") - T)) <= 0.01
    a.close()
    b.close()
