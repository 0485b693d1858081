"""The temporally blocked fast transient (HSB_FORM_FAST_BLOCKED; the kernel of
HSB_FORM_FAST for models of 2^21 cells and more) against

* the same arithmetic run one grid-wide pass per Krylov vector
  (HSB_FORM_FAST_PASSES): the same accepted steps and attempts, block and
  grid temperatures within 1e-4 K (both are FP32-vector forms; they differ
  only in the order of the FP64 sums of increment, error and edge sums);
* the oracle's FP64 replay of the reference: 0.01 K.

The same kernel with every stencil pass in FP64 (HSB_FORM_FP64_BLOCKED)
must take the same accepted steps as the FP64 replay of the reference's RK4
and stay within 1e-6 K of it (on long intervals with rejected attempts,
within four times the spread FP64 rounding alone gives the reference
algorithm there).

Cases cover tiles that are all boundary ("ring") tiles (16x16), grids with
interior tiles (256x256), rectangular grids, the secondary heat path (28
package nodes, 20 edges), 3-D stacks, and long sampling intervals whose
adaptive steps are rejected (the retry recomputes its vectors with a larger
halo in sub-tiles).
"""
import contextlib

import numpy as np
import pytest

from hotspot_b200 import FORM_FAST_BLOCKED, FORM_FAST_PASSES, FORM_FP64_BLOCKED, FORM_PARITY
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from oracle.restatement import OracleModel, x87_rounding

pytestmark = pytest.mark.gpu
TOL_FORMS = 1e-4
TOL_FP64 = 0.01


def _scenario(workdir, case):
    if case == "chip2d16":
        return W.scenario_chip2d(workdir, seed=81, grid=16, steps=8)
    if case == "chip2d64":
        return W.scenario_chip2d(workdir, seed=82, grid=64, steps=8)
    if case == "rect32x64":
        sc = W.scenario_chip2d(workdir, seed=83, grid=32, steps=8)
        sc.config["grid_cols"] = "64"
        return sc
    if case == "rect128x32":
        sc = W.scenario_chip2d(workdir, seed=84, grid=128, steps=6)
        sc.config["grid_cols"] = "32"
        return sc
    if case == "secondary":
        sc = W.scenario_chip2d(workdir, seed=85, grid=32, steps=6)
        sc.config["model_secondary"] = "1"
        return sc
    if case == "stack64":
        return W.scenario_stack3d(workdir, seed=86, grid=64, steps=6, n_blocks=12)
    if case == "stack256":
        return W.scenario_stack3d(workdir, seed=87, grid=256, steps=4)
    if case == "long_chip2d":        # 1 ms rows: steps are rejected and retried
        sc = W.scenario_chip2d(workdir, seed=88, grid=32, steps=4)
        sc.dt = 1e-3
        return sc
    if case == "long_stack":
        sc = W.scenario_stack3d(workdir, seed=89, grid=64, steps=3, n_blocks=10)
        sc.dt = 1e-3
        return sc
    raise ValueError(case)


def _run(sc, form, rows):
    m = hm.from_scenario(sc)
    m.set_solver(form)
    t = m.vector(m.config.init_temp)
    temps, steps, attempts, fallbacks = [], 0, 0, 0
    for k in range(rows):
        m.compute_temp(m.power_vector(sc.block_power[k]), t if k == 0 else None, sc.dt)
        s = m.stats()
        steps += s["rk4_steps"]
        attempts += s["rk4_attempts"]
        fallbacks += s["fallbacks"]
        temps.append(t.copy())
    g = m.grid("trans")
    m.close()
    return np.array(temps), g, steps, attempts, fallbacks


CASES = ["chip2d16", "chip2d64", "rect32x64", "rect128x32", "secondary", "stack64", "stack256", "long_chip2d",
         "long_stack"]


@pytest.mark.parametrize("case", CASES)
def test_blocked_matches_pass_by_pass(workdir, case):
    sc = _scenario(workdir, case)
    rows = min(sc.steps, sc.block_power.shape[0])
    ta, ga, sa, aa, fa = _run(sc, FORM_FAST_BLOCKED, rows)
    tb, gb, sb, ab, fb = _run(sc, FORM_FAST_PASSES, rows)
    assert fa == 0 and fb == 0, "a retry outgrew the kernel"
    if case.startswith("long"):
        # rows of 1 ms: many steps sit at the accept/reject threshold, where
        # the two forms' FP32 rounding can take different decisions; both
        # follow the reference's step rule, and both stay within the fast
        # form's bar of the FP64 replay
        assert aa > sa and ab > sb, "the long rows were meant to reject some steps"
        assert abs(sa - sb) <= 0.1 * sb
        tr, gr, *_ = _run(sc, FORM_PARITY, rows)
        assert np.max(np.abs(ta - tr)) <= TOL_FP64 and np.max(np.abs(tb - tr)) <= TOL_FP64
        return
    assert (sa, aa) == (sb, ab), (sa, aa, sb, ab)
    assert np.max(np.abs(ta - tb)) <= TOL_FORMS
    assert np.max(np.abs(ga - gb)) <= TOL_FORMS


@pytest.mark.parametrize("case", ["chip2d64", "secondary", "stack64", "long_chip2d"])
def test_blocked_against_fp64_replay(workdir, case):
    """Against the FP64 replay on the GPU, which reproduces the reference's
    own doubles (pinned by the parity tests and, for the secondary heat
    path, by the reference's golden vectors)."""
    sc = _scenario(workdir, case)
    rows = min(sc.steps, sc.block_power.shape[0], 4)
    ta, ga, *_ = _run(sc, FORM_FAST_BLOCKED, rows)
    tr, gr, *_ = _run(sc, FORM_PARITY, rows)
    assert np.max(np.abs(ta - tr)) <= TOL_FP64
    assert np.max(np.abs(ga - gr)) <= TOL_FP64


def test_blocked_against_fp64_oracle(workdir):
    """The same against the oracle's restatement on the CPU (primary path)."""
    sc = _scenario(workdir, "stack64")
    rows = 4
    ta, ga, *_ = _run(sc, FORM_FAST_BLOCKED, rows)
    o = OracleModel(sc)
    to = o.vector(o.init_temp)
    for k in range(rows):
        o.compute_temp(o.power_vector(sc.block_power[k]), to if k == 0 else None, sc.dt)
        assert np.max(np.abs(ta[k] - to)) <= TOL_FP64, k
    assert np.max(np.abs(ga - o.grid("trans"))) <= TOL_FP64


TOL_REPLAY = 1e-6


def _rounding_spread(sc, rows):
    """How far FP64 rounding alone moves the reference algorithm's result on
    this input: the oracle against the same oracle compiled with x87 80-bit
    intermediates, blocks and grid."""
    out = []
    for ctx in (contextlib.nullcontext(), x87_rounding()):
        with ctx:
            o = OracleModel(sc)
            to = o.vector(o.init_temp)
            for k in range(rows):
                o.compute_temp(o.power_vector(sc.block_power[k]), to if k == 0 else None, sc.dt)
            out.append((to.copy(), o.grid("trans")))
    return max(np.max(np.abs(out[0][0] - out[1][0])), np.max(np.abs(out[0][1] - out[1][1])))


@pytest.mark.parametrize("case", ["chip2d16", "chip2d64", "secondary", "stack64", "stack256", "rect128x32",
                                  "long_chip2d", "long_stack"])
def test_fp64_blocked_matches_replay(workdir, case):
    """1e-6 K, or on long intervals with rejected attempts four times the
    spread that FP64 rounding alone gives the reference algorithm there: a
    retry takes k1 = f(t1) of the rejected, unstable attempt (RCutil.c:
    557-571), whose large stiff components cancel in the accepted step, so any
    two FP64 evaluation orders (the replay's stage by stage, this kernel's
    polynomial in L) differ by more than 1e-6 K (long_stack: 2.1e-6 K between
    the oracle's SSE and x87 builds)."""
    sc = _scenario(workdir, case)
    rows = min(sc.steps, sc.block_power.shape[0])
    ta, ga, sa, aa, fa = _run(sc, FORM_FP64_BLOCKED, rows)
    tb, gb, sb, ab, fb = _run(sc, FORM_PARITY, rows)
    assert fa == 0, "a retry outgrew the kernel"
    assert sa == sb and aa == ab, (sa, aa, sb, ab)
    tol = TOL_REPLAY
    if case.startswith("long_"):
        tol = max(tol, 4.0 * _rounding_spread(sc, rows))
    assert np.max(np.abs(ta - tb)) <= tol, tol
    assert np.max(np.abs(ga - gb)) <= tol, tol


def test_fast_form_picks_kernel_by_size(workdir):
    """HSB_FORM_FAST runs the pass-by-pass kernel below 2^21 cells and the
    blocked kernel from there up; there its result is the explicit blocked
    form's, bit for bit."""
    from hotspot_b200 import FORM_FAST
    small = W.scenario_chip2d(workdir, seed=97, grid=64, steps=2)
    m = hm.from_scenario(small)
    m.set_solver(FORM_FAST)
    m.compute_temp(m.power_vector(small.block_power[0]), m.vector(m.config.init_temp), small.dt)
    assert m.transient_kernel() == "passes"
    m.close()
    big = W.scenario_random_chip(workdir, np.random.default_rng(98), "big", side=512, chip_layers=6, steps=2)
    grids = []
    for form in (FORM_FAST, FORM_FAST_BLOCKED):
        m = hm.from_scenario(big)
        assert m.n_cells >= 1 << 21
        m.set_solver(form)
        m.compute_temp(m.power_vector(big.block_power[0]), m.vector(m.config.init_temp), big.dt)
        assert m.transient_kernel() == "blocked"
        grids.append(m.grid("trans"))
        m.close()
    assert np.array_equal(grids[0], grids[1])
