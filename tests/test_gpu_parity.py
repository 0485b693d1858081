"""Parity of the CUDA exact-replay path (HSB_FORM_PARITY) with the oracle.

The oracle's restatement reproduces the reference's doubles exactly (pinned
in tests/test_cpu_oracle.py against the reference build and the golden
fixtures), so the device results are compared with it directly.  The bar is
max |dT| <= 1e-6 K (transient and steady, block and grid vectors); the
replay is designed to be bit-exact and the measured difference is reported.
"""
import numpy as np
import pytest

from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from oracle.restatement import OracleModel

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _run_pair(sc, steps):
    m = hm.from_scenario(sc)
    o = OracleModel(sc)
    t, to = m.vector(o.init_temp), o.vector(o.init_temp)
    for k in range(steps):
        p = m.power_vector(sc.block_power[k])
        m.compute_temp(p.copy(), t if k == 0 else None, sc.dt)
        o.compute_temp(p.copy(), to if k == 0 else None, sc.dt)
    return m, o, t, to


@pytest.mark.parametrize("grid,seed", [(16, 0), (32, 1), (64, 2)])
def test_transient_chip2d(workdir, grid, seed):
    sc = W.scenario_chip2d(workdir, seed=seed, grid=grid, steps=12)
    m, o, t, to = _run_pair(sc, sc.steps)
    assert np.max(np.abs(t - to)) <= TOL
    assert np.max(np.abs(m.grid("trans") - o.grid("trans"))) <= TOL
    st = m.stats()
    assert st["rk4_steps"] >= 1 and st["slope_evals"] == 1 * st["rk4_steps"] + 10 * st["rk4_attempts"]
    m.close()


@pytest.mark.parametrize("grid,seed", [(16, 3), (32, 4), (64, 5)])
def test_steady_chip2d(workdir, grid, seed):
    sc = W.scenario_chip2d(workdir, seed=seed, grid=grid, steps=4)
    m = hm.from_scenario(sc)
    o = OracleModel(sc)
    avg = m.power_vector(sc.block_power.mean(0))
    s, so = m.vector(), o.vector()
    m.steady(avg.copy(), s)
    o.steady(avg.copy(), so)
    assert np.max(np.abs(s - so)) <= TOL
    assert np.max(np.abs(m.grid("steady") - o.grid("steady"))) <= TOL
    m.close()


def test_stack3d_lcf(workdir):
    sc = W.scenario_stack3d(workdir, seed=7, grid=32, steps=6, n_blocks=12)
    m, o, t, to = _run_pair(sc, sc.steps)
    assert np.max(np.abs(t - to)) <= TOL
    avg = m.power_vector(sc.block_power.mean(0))
    s, so = m.vector(), o.vector()
    m.steady(avg.copy(), s)
    o.steady(avg.copy(), so)
    assert np.max(np.abs(s - so)) <= TOL
    m.close()


def test_detailed3d_and_map_modes(workdir):
    sc = W.scenario_stack3d(workdir, seed=8, grid=32, steps=4, n_blocks=10)
    sc.detailed_3D = True
    for mode in ("avg", "min", "max", "center"):
        sc.config["grid_map_mode"] = mode
        m, o, t, to = _run_pair(sc, sc.steps)
        assert np.max(np.abs(t - to)) <= TOL, mode
        m.close()
    avg = o.power_vector(sc.block_power.mean(0))
    m = hm.from_scenario(sc)
    s, so = m.vector(), o.vector()
    m.steady(avg.copy(), s)
    o.steady(avg.copy(), so)
    assert np.max(np.abs(s - so)) <= TOL
    m.close()


def test_microchannel_transient(workdir):
    sc = W.scenario_microchannel(workdir, seed=1, grid=32, die=2e-3, channel_w=125e-6,
                                 channel_h=125e-6, pitch=250e-6, blocks=8)
    sc.block_power = np.repeat(sc.block_power, 3, axis=0)
    sc.dt = 1e-5
    m, o, t, to = _run_pair(sc, 3)
    assert np.max(np.abs(t - to)) <= TOL
    assert np.max(np.abs(m.grid("trans") - o.grid("trans"))) <= TOL
    m.close()


def _golden(workdir, name):
    import importlib.util
    import os
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(here, "make_golden.py"))
    mg = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mg)
    sc, n = mg.cases(workdir)[name]
    return sc, n, np.load(os.path.join(here, name + ".npz"))


def test_secondary_path_against_reference_golden(workdir):
    """The secondary heat path (substrate, solder and PCB layers, 28 package
    nodes), against the reference's own results (golden vectors made by the
    reference build): the FP64 replay to 1e-6 K, the fast forms to 0.01 K."""
    from hotspot_b200 import FORM_FAST
    sc, n, g = _golden(workdir, "secondary_16")
    for form, tol in ((None, TOL), (FORM_FAST, 0.01)):
        m = hm.from_scenario(sc)
        if form is not None:
            m.set_solver(form)
        t = m.vector(333.15)
        assert t.size == g["temps"].shape[1]
        for k in range(n):
            p = g["block_power"][k].copy()
            m.compute_temp(p, t if k == 0 else None, sc.dt)
            assert np.max(np.abs(t - g["temps"][k])) <= tol, (form, k)
        assert np.max(np.abs(m.grid("trans") - g["grid_trans"])) <= tol
        if form is None:   # the FP64 replay of the reference's steady solver
            s = m.vector()
            m.steady(g["steady_power"].copy(), s)
            assert np.max(np.abs(s - g["steady"])) <= TOL
            assert np.max(np.abs(m.grid("steady") - g["grid_steady"])) <= TOL
        m.close()
