"""The fast forms (HSB_FORM_FAST) against the FP64 oracle.

Transient: FP32 stencil stages with FP64 state, error norm and step control
on the device; compared with the oracle's exact FP64 replay of the
reference (same adaptive algorithm), bar max |dT| <= 0.01 K.
Steady: FP32 multigrid-preconditioned CG inside FP64 iterative refinement;
compared with the converged FP64 solution of the same system by sparse
direct LU, bar max |dT| <= 0.01 K (the solver converges far below it).
"""
import numpy as np
import pytest

from hotspot_b200 import FORM_FAST
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from oracle.restatement import OracleModel

pytestmark = pytest.mark.gpu
TOL = 0.01


def _transient(sc, steps):
    m = hm.from_scenario(sc)
    m.set_solver(FORM_FAST)
    o = OracleModel(sc)
    t, to = m.vector(o.init_temp), o.vector(o.init_temp)
    worst = 0.0
    for k in range(steps):
        p = m.power_vector(sc.block_power[k])
        m.compute_temp(p.copy(), t if k == 0 else None, sc.dt)
        o.compute_temp(p.copy(), to if k == 0 else None, sc.dt)
        worst = max(worst, float(np.max(np.abs(t - to))))
    grid_err = float(np.max(np.abs(m.grid("trans") - o.grid("trans"))))
    m.close()
    return worst, grid_err


@pytest.mark.parametrize("grid", [32, 64])
def test_fast_transient_chip2d(workdir, grid):
    sc = W.scenario_chip2d(workdir, seed=11, grid=grid, steps=40)
    worst, grid_err = _transient(sc, sc.steps)
    assert worst <= TOL and grid_err <= TOL


def test_fast_transient_stack(workdir):
    sc = W.scenario_stack3d(workdir, seed=12, grid=64, steps=20, n_blocks=16)
    worst, grid_err = _transient(sc, sc.steps)
    assert worst <= TOL and grid_err <= TOL


def test_fast_transient_detailed(workdir):
    sc = W.scenario_stack3d(workdir, seed=13, grid=32, steps=10, n_blocks=10)
    sc.detailed_3D = True
    worst, grid_err = _transient(sc, sc.steps)
    assert worst <= TOL and grid_err <= TOL


def test_fast_transient_microchannel(workdir):
    sc = W.scenario_microchannel(workdir, seed=2, grid=32, die=2e-3, channel_w=125e-6,
                                 channel_h=125e-6, pitch=250e-6, blocks=8)
    sc.block_power = np.repeat(sc.block_power, 3, axis=0)
    sc.dt = 1e-5
    worst, grid_err = _transient(sc, 3)
    assert worst <= TOL and grid_err <= TOL


@pytest.mark.parametrize("builder,grid", [("chip2d", 64), ("stack3d", 64), ("detailed", 32)])
def test_mg_steady_converged(workdir, builder, grid):
    if builder == "chip2d":
        sc = W.scenario_chip2d(workdir, seed=21, grid=grid, steps=2)
    else:
        sc = W.scenario_stack3d(workdir, seed=22, grid=grid, steps=2, n_blocks=14)
        sc.detailed_3D = builder == "detailed"
    m = hm.from_scenario(sc)
    m.set_solver(FORM_FAST)
    o = OracleModel(sc)
    avg = m.power_vector(sc.block_power.mean(0))
    s = m.vector()
    m.steady(avg.copy(), s)
    T, Tb = o.steady_direct(avg)
    assert np.max(np.abs(s - Tb)) <= TOL
    assert np.max(np.abs(m.grid("steady") - T)) <= TOL
    st = m.stats()
    assert st["refinements"] >= 1
    m.close()


@pytest.mark.parametrize("builder", ["chip2d", "stack3d", "detailed"])
def test_krylov_form_matches_stage_form(workdir, builder):
    """The default fast transient (step-doubling RK4 evaluated through Krylov
    vectors of the affine slope operator) against the same fast arithmetic
    evaluated stage by stage: same accepted steps, temperatures within 1e-3 K."""
    from hotspot_b200 import FORM_FAST_STAGES
    if builder == "chip2d":
        sc = W.scenario_chip2d(workdir, seed=31, grid=64, steps=25)
    else:
        sc = W.scenario_stack3d(workdir, seed=32, grid=64, steps=25, n_blocks=12)
        sc.detailed_3D = builder == "detailed"
    runs = []
    for form in (FORM_FAST, FORM_FAST_STAGES):
        m = hm.from_scenario(sc)
        m.set_solver(form)
        t = m.vector(m.config.init_temp)
        out = []
        tot = {"rk4_steps": 0, "rk4_attempts": 0, "fallbacks": 0}
        for k in range(sc.steps):
            m.compute_temp(m.power_vector(sc.block_power[k]), t if k == 0 else None, sc.dt)
            out.append(t.copy())
            st = m.stats()
            for key in tot:
                tot[key] += st[key]
        runs.append((np.array(out), m.grid("trans"), tot))
        m.close()
    (a, ga, sa), (b, gb, sb) = runs
    assert sa["rk4_steps"] == sb["rk4_steps"] and sa["rk4_attempts"] == sb["rk4_attempts"]
    assert sa["fallbacks"] == 0
    assert np.max(np.abs(a - b)) <= 1e-3 and np.max(np.abs(ga - gb)) <= 1e-3


@pytest.mark.parametrize("grid,seed", [(32, 41), (64, 42)])
def test_bicgstab_microchannel_steady(workdir, grid, seed):
    """The non-symmetric steady system of a microchannel model (advection
    terms +-Cv*flow/2, which the reference can only hand to SuperLU) by FP32
    BiCGStab with FP64 refinement, against FP64 sparse LU of the same
    system: bar max |dT| <= 0.01 K."""
    from hotspot_b200 import STEADY_BICGSTAB
    sc = W.scenario_microchannel(workdir, seed=seed, grid=grid, die=grid * 20e-6, blocks=8)
    m = hm.from_scenario(sc)
    m.set_solver(FORM_FAST, STEADY_BICGSTAB)
    o = OracleModel(sc)
    p = m.power_vector(sc.block_power[0])
    s = m.vector()
    m.steady(p.copy(), s)
    T, Tb = o.steady_direct(p)
    st = m.stats()
    err_b = float(np.max(np.abs(s - Tb)))
    err_g = float(np.max(np.abs(m.grid("steady") - T)))
    m.close()
    assert err_b <= TOL and err_g <= TOL, (err_b, err_g, st)
    assert st["refinements"] >= 1 and st["residual"] < 1e-6


def test_bicgstab_symmetric_model(workdir):
    """The same solver on a model without advection agrees with the direct solve."""
    from hotspot_b200 import STEADY_BICGSTAB
    sc = W.scenario_stack3d(workdir, seed=43, grid=64, steps=2, n_blocks=10)
    sc.detailed_3D = True
    m = hm.from_scenario(sc)
    m.set_solver(FORM_FAST, STEADY_BICGSTAB)
    o = OracleModel(sc)
    avg = m.power_vector(sc.block_power.mean(0))
    s = m.vector()
    m.steady(avg.copy(), s)
    T, Tb = o.steady_direct(avg)
    err = float(np.max(np.abs(m.grid("steady") - T)))
    m.close()
    assert np.max(np.abs(s - Tb)) <= TOL and err <= TOL, err


@pytest.mark.parametrize("builder", ["chip2d", "stack3d", "detailed"])
def test_trace_equals_single_intervals(workdir, builder):
    """K intervals in one persistent launch (hsb_dev_transient_trace) give the
    results of K single-interval calls of the fast form, bit for bit."""
    if builder == "chip2d":
        sc = W.scenario_chip2d(workdir, seed=51, grid=64, steps=12)
    else:
        sc = W.scenario_stack3d(workdir, seed=52, grid=64, steps=12, n_blocks=12)
        sc.detailed_3D = builder == "detailed"
    a, b = hm.from_scenario(sc), hm.from_scenario(sc)
    a.set_solver(FORM_FAST)
    t = a.vector(a.config.init_temp)
    powers = np.stack([a.power_vector(sc.block_power[k]) for k in range(sc.steps)])
    steps_a = 0
    for k in range(sc.steps):
        a.compute_temp(powers[k].copy(), t if k == 0 else None, sc.dt)
        steps_a += a.stats()["rk4_steps"]
    out, st = b.compute_trace(powers, b.vector(b.config.init_temp), sc.dt)
    assert st["rk4_steps"] == steps_a
    assert np.array_equal(out, t)
    assert np.array_equal(a.grid("trans"), b.grid("trans"))
    a.close()
    b.close()


def test_forms_alternate_on_one_model(workdir):
    """Switching one model between the parity and the fast forms from call to
    call: each form keeps its own state buffers and swaps them as steps are
    accepted, so the fast form's replayed interval graphs must follow the
    buffers' current roles.  The trajectory stays within 0.01 K of the FP64
    replay."""
    from hotspot_b200 import FORM_PARITY
    sc = W.scenario_chip2d(workdir, seed=71, grid=32, steps=12)
    m, o = hm.from_scenario(sc), OracleModel(sc)
    t, to = m.vector(o.init_temp), o.vector(o.init_temp)
    forms = [FORM_FAST, FORM_FAST, FORM_PARITY, FORM_FAST, FORM_FAST, FORM_PARITY, FORM_PARITY, FORM_FAST,
             FORM_FAST, FORM_FAST, FORM_PARITY, FORM_FAST]
    for k, form in enumerate(forms):
        m.set_solver(form)
        p = m.power_vector(sc.block_power[k])
        m.compute_temp(p.copy(), t if k == 0 else None, sc.dt)
        o.compute_temp(p.copy(), to if k == 0 else None, sc.dt)
        assert np.max(np.abs(t - to)) <= TOL, k
    assert np.max(np.abs(m.grid("trans") - o.grid("trans"))) <= TOL
    m.close()


def test_mg_steady_secondary_path(workdir):
    """The MG-PCG steady solve on the secondary heat path (substrate, solder
    and PCB layers, 28 package nodes; the steady package equations of
    temperature_grid.c:2228-2379) against the reference's own steady result
    (golden vectors of the reference build, which stops within 1e-3 K of the
    fixed point) and, on a 64x64 chip, against the FP64 replay of the
    reference's Gauss-Seidel: 0.01 K, with a converged FP64 residual."""
    from test_gpu_parity import _golden
    sc, n, g = _golden(workdir, "secondary_16")
    m = hm.from_scenario(sc)
    m.set_solver(FORM_FAST)
    s = m.vector()
    m.steady(g["steady_power"].copy(), s)
    assert np.max(np.abs(s - g["steady"])) <= TOL
    assert np.max(np.abs(m.grid("steady") - g["grid_steady"])) <= TOL
    assert m.stats()["refinements"] >= 1
    m.close()
    sc = W.scenario_chip2d(workdir, seed=23, grid=64, steps=2)
    sc.config["model_secondary"] = "1"
    out = []
    for form in (FORM_FAST, None):
        m = hm.from_scenario(sc)
        if form is not None:
            m.set_solver(form)
        p = m.power_vector(sc.block_power.mean(0))
        s = m.vector()
        m.steady(p.copy(), s)
        out.append((s, m.grid("steady"), m.stats()))
        m.close()
    (sf, gf, stf), (sr, gr, _) = out
    assert np.max(np.abs(sf - sr)) <= TOL and np.max(np.abs(gf - gr)) <= TOL
    assert stf["residual"] < 1e-6
