"""The allocation-free transient entry point, hsb_dev_transient_noalloc.

Callers that may not allocate device memory while they run (a simulator
that reserves its GPU memory at start-up, a real-time loop that cannot take
cudaMalloc's implicit synchronisation) get one more C entry point that runs
the fast transient form with its temporaries in a static device array.
This test calls it through the C-ABI on a state and power vectors held in
device memory, twice in a row, and checks each result
  * against the regular entry point (compute_temp with the stage-by-stage
    fast form, the arithmetic the allocation-free entry point runs), within
    the parity tolerance used by the GPU tests, and
  * against the reference's own FP64 code (the live build; else the
    oracle's restatement), within the fast form's 0.01 K bar,
on models that exercise the static scratch's sizing: a 2-D chip, the
secondary heat path (28 package nodes), a 6-layer stack, and a rectangular
grid of exactly HSB_NOALLOC_MAX_CELLS cells.  It also checks the defining
property: the model it ran on never allocated a fast-transient workspace.
It lives in its own file so a run that stops at the first failure has run
every other test first; it passes alone in a fresh process and after the
other tests.
"""
import ctypes as C

import numpy as np
import pytest

from hotspot_b200 import FORM_FAST_STAGES, _abi
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from oracle import ref as R
from oracle.restatement import OracleModel

pytestmark = pytest.mark.gpu
TOL = 1e-6
TOL_FP64 = 0.01
MAX_CELLS = 65536


def _scenario(workdir, case):
    if case == "chip2d":
        return W.scenario_chip2d(workdir, seed=31, grid=64, steps=3)
    if case == "secondary":
        sc = W.scenario_chip2d(workdir, seed=33, grid=32, steps=3)
        sc.config["model_secondary"] = "1"
        return sc
    if case == "stack":
        return W.scenario_stack3d(workdir, seed=34, grid=64, steps=3, n_blocks=12)
    # rectangular: 4 layers x 64 x 256 = the scratch's maximum cell count
    sc = W.scenario_chip2d(workdir, seed=35, grid=64, steps=3)
    sc.config["grid_cols"] = "256"
    return sc


@pytest.mark.parametrize("case", ["chip2d", "secondary", "stack", "max_cells"])
def test_noalloc_matches_regular_entry(workdir, case):
    import torch

    sc = _scenario(workdir, case)
    L = _abi.lib()

    # regular entry point: the stage-by-stage fast form through compute_temp
    a = hm.from_scenario(sc)
    if case == "max_cells":
        assert a.n_cells == MAX_CELLS
    a.set_solver(FORM_FAST_STAGES)
    temp = a.vector(a.config.init_temp)
    p0 = a.power_vector(sc.block_power[0])
    a.compute_temp(p0.copy(), temp, 0.0)          # zero-length interval: state = b2g(temp)
    y0 = a.grid("trans")
    expected = []
    for k in (1, 2):
        a.compute_temp(a.power_vector(sc.block_power[k]).copy(), None, sc.dt)
        expected.append(a.grid("trans"))

    # the reference's own FP64 code from the same state (the live build;
    # else the oracle's restatement, which covers the primary heat path)
    live = R.available()
    if not live and case == "secondary":
        pytest.skip("the secondary heat path needs the live reference build")
    o = R.RefModel(sc) if live else OracleModel(sc)
    to = o.vector(333.15)
    o.compute_temp(o.power_vector(sc.block_power[0]), to, 0.0)
    assert np.max(np.abs(o.grid("trans") - y0)) <= TOL
    exact = []
    for k in (1, 2):
        o.compute_temp(o.power_vector(sc.block_power[k]), None, sc.dt)
        exact.append(o.grid("trans"))

    # the same intervals through the allocation-free entry point
    b = hm.from_scenario(sc)
    assert b.n_cells <= MAX_CELLS
    dev = L.hsb_grid_device(b.ptr)
    y = torch.tensor(y0, dtype=torch.float64, device="cuda")
    for k, exp, ex64 in zip((1, 2), expected, exact):
        p = b.power_vector(sc.block_power[k])
        pgrid = o.power_grid(p.copy()) if live else o.b2g(p.copy(), True)
        pg = torch.tensor(pgrid, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()        # y and pg are complete before the call reads them
        st = _abi.Stats()
        rc = L.hsb_dev_transient_noalloc(dev, C.c_void_p(y.data_ptr()), C.c_void_p(pg.data_ptr()),
                                         sc.dt, C.byref(st))
        assert rc == 0, L.hsb_dev_last_error().decode()
        assert st.rk4_steps >= 1
        got = y.cpu().numpy()
        assert np.max(np.abs(got - exp)) <= TOL
        assert np.max(np.abs(got - ex64)) <= TOL_FP64
    mask = C.c_int(-1)
    assert L.hsb_dev_workspaces(dev, C.byref(mask)) == 0
    assert mask.value & 1 == 0, "the allocation-free entry point allocated a fast-transient workspace"
    a.close()
    b.close()
    if live:
        o.close()


def test_noalloc_rejects_oversized_models(workdir):
    import torch

    sc = W.scenario_chip2d(workdir, seed=32, grid=256, steps=1)    # 262,144 cells
    L = _abi.lib()
    m = hm.from_scenario(sc)
    y = torch.zeros(m.n_cells + m.n_extra, dtype=torch.float64, device="cuda")
    rc = L.hsb_dev_transient_noalloc(L.hsb_grid_device(m.ptr), C.c_void_p(y.data_ptr()),
                                     C.c_void_p(y.data_ptr()), 1e-6, None)
    assert rc != 0
    assert "HSB_NOALLOC_MAX_CELLS" in L.hsb_dev_last_error().decode()
    m.close()
