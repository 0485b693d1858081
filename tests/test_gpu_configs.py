"""Parity at the benchmark workloads' own sizes.

The other GPU test files pin every form on grids of at most 64x64.  Here the
same checks run on the workloads the benchmark measures:

* the 2-D chip (64x64, default package, 15 blocks): the full 1000-row power
  trace at 3.333 us plus the steady solve of its average power, FP64 replay
  against the reference's own C code (``oracle/_ref``, else the oracle's C
  restatement, which reproduces it bit for bit), bar 1e-6 K;
* the 3-D stack (4 chip layers + spreader/sink, 256x256 over 20x20 mm):
  the FP64 replay over 5 rows against the reference and its steady solve
  against the oracle, bar 1e-6 K; the fast form over 1000 rows against the
  FP64 replay, bar 0.01 K, with the accepted-step counts compared;
* the microchannel stack at 256x256: FP32 BiCGStab with FP64 refinement
  against FP64 sparse LU of the same system, bar 0.01 K.
"""
import numpy as np
import pytest

from hotspot_b200 import FORM_FAST, FORM_PARITY
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from oracle import ref as R
from oracle.restatement import OracleModel

pytestmark = pytest.mark.gpu
TOL_FP64 = 1e-6
TOL_FAST = 0.01


def _reference(sc):
    """The reference's own code when it was built here, else the oracle."""
    return R.RefModel(sc) if R.available() else OracleModel(sc)


def test_chip2d_full_trace_and_steady(workdir):
    sc = W.scenario_chip2d(workdir, seed=0, grid=64, steps=1000)
    m, o = hm.from_scenario(sc), _reference(sc)
    m.set_solver(FORM_PARITY)
    t, to = m.vector(m.config.init_temp), o.vector(333.15)
    worst = 0.0
    steps = 0
    for k in range(sc.steps):
        p = m.power_vector(sc.block_power[k])
        m.compute_temp(p.copy(), t if k == 0 else None, sc.dt)
        o.compute_temp(p.copy(), to if k == 0 else None, sc.dt)
        steps += m.stats()["rk4_steps"]
        worst = max(worst, float(np.max(np.abs(t - to))))
    assert worst <= TOL_FP64, worst
    assert np.max(np.abs(m.grid("trans") - o.grid("trans"))) <= TOL_FP64
    assert steps >= sc.steps
    avg = m.power_vector(sc.block_power.mean(0))
    s, so = m.vector(), o.vector()
    m.steady(avg.copy(), s)
    o.steady(avg.copy(), so)
    assert np.max(np.abs(s - so)) <= TOL_FP64
    assert np.max(np.abs(m.grid("steady") - o.grid("steady"))) <= TOL_FP64
    m.close()
    if hasattr(o, "close"):
        o.close()


def test_stack256_fp64_replay(workdir):
    sc = W.scenario_stack3d(workdir, seed=100, grid=256, steps=6)
    m, ref = hm.from_scenario(sc), _reference(sc)
    m.set_solver(FORM_PARITY)
    t, tr = m.vector(m.config.init_temp), ref.vector(333.15)
    for k in range(5):
        p = m.power_vector(sc.block_power[k])
        m.compute_temp(p.copy(), t if k == 0 else None, sc.dt)
        ref.compute_temp(p.copy(), tr if k == 0 else None, sc.dt)
        assert np.max(np.abs(t - tr)) <= TOL_FP64, k
    assert np.max(np.abs(m.grid("trans") - ref.grid("trans"))) <= TOL_FP64
    if hasattr(ref, "close"):
        ref.close()
    # steady: the oracle's C restatement of the reference's solver (the
    # reference itself needs ~90 s here; the restatement is bit-exact with it)
    o = OracleModel(sc)
    avg = m.power_vector(sc.block_power.mean(0))
    s, so = m.vector(), o.vector()
    m.steady(avg.copy(), s)
    o.steady(avg.copy(), so)
    assert np.max(np.abs(s - so)) <= TOL_FP64
    assert np.max(np.abs(m.grid("steady") - o.grid("steady"))) <= TOL_FP64
    m.close()


def test_stack256_fast_form_1000_rows(workdir):
    """The fast form against the FP64 replay (pinned to the reference above)
    over 1000 rows of the 256x256 stack: every row's block temperatures
    within 0.01 K and the same adaptive step sequence (accepted steps per
    row)."""
    rows = 1000
    sc = W.scenario_stack3d(workdir, seed=100, grid=256, steps=rows)
    runs = []
    for form in (FORM_PARITY, FORM_FAST):
        m = hm.from_scenario(sc)
        m.set_solver(form)
        t = m.vector(m.config.init_temp)
        temps, steps = np.empty((rows, t.size)), np.empty(rows, dtype=np.int64)
        for k in range(rows):
            m.compute_temp(m.power_vector(sc.block_power[k]), t if k == 0 else None, sc.dt)
            temps[k] = t
            steps[k] = m.stats()["rk4_steps"]
        runs.append((temps, steps, m.grid("trans")))
        m.close()
    (tp, sp, gp), (tf, sf, gf) = runs
    assert np.max(np.abs(tp - tf)) <= TOL_FAST
    assert np.max(np.abs(gp - gf)) <= TOL_FAST
    # the error norm is computed from FP32 vectors, so a step size can differ
    # in its last bits; the accepted-step sequence is the reference's
    assert np.array_equal(sp, sf), (int(sp.sum()), int(sf.sum()), int(np.sum(sp != sf)))


def test_microchannel256_bicgstab(workdir):
    from hotspot_b200 import STEADY_BICGSTAB
    sc = W.scenario_microchannel(workdir, seed=3, grid=256, die=256 * 20e-6, blocks=16)
    m = hm.from_scenario(sc)
    m.set_solver(FORM_FAST, STEADY_BICGSTAB)
    o = OracleModel(sc)
    p = m.power_vector(sc.block_power[0])
    s = m.vector()
    m.steady(p.copy(), s)
    st = m.stats()
    T, Tb = o.steady_direct(p)
    err_b = float(np.max(np.abs(s - Tb)))
    err_g = float(np.max(np.abs(m.grid("steady") - T)))
    m.close()
    assert err_b <= TOL_FAST and err_g <= TOL_FAST, (err_b, err_g, st)
    assert st["residual"] < 1e-6
