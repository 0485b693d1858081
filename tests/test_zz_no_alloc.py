"""The allocation-free transient entry point, hsb_dev_transient_noalloc.

Callers that may not allocate device memory while they run (a simulator
that reserves its GPU memory at start-up, a real-time loop that cannot take
cudaMalloc's implicit synchronisation) get one more C entry point that runs
the fast transient form with its temporaries in a static device array.
This test calls it through the C-ABI on a state and power vectors held in
device memory, twice in a row, and checks each result against the regular
entry point (compute_temp with the stage-by-stage fast form, the arithmetic
the allocation-free entry point runs) within the parity tolerance used by the
GPU tests.  It lives in its own file so a
run that stops at the first failure has run every other test first; it
passes alone in a fresh process and after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from hotspot_b200 import FORM_FAST_STAGES, _abi
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from oracle.restatement import OracleModel

pytestmark = pytest.mark.gpu
TOL = 1e-6


def test_noalloc_matches_regular_entry(workdir):
    import torch

    sc = W.scenario_chip2d(workdir, seed=31, grid=64, steps=3)
    L = _abi.lib()

    # regular entry point: the stage-by-stage fast form through compute_temp
    a = hm.from_scenario(sc)
    a.set_solver(FORM_FAST_STAGES)
    temp = a.vector(a.config.init_temp)
    p0 = a.power_vector(sc.block_power[0])
    a.compute_temp(p0.copy(), temp, 0.0)          # zero-length interval: state = b2g(temp)
    y0 = a.grid("trans")
    expected = []
    for k in (1, 2):
        a.compute_temp(a.power_vector(sc.block_power[k]).copy(), None, sc.dt)
        expected.append(a.grid("trans"))

    # the same intervals through the allocation-free entry point
    b = hm.from_scenario(sc)
    assert b.n_cells <= 65536
    o = OracleModel(sc)                            # grid power vectors (bit-exact b2g)
    dev = L.hsb_grid_device(b.ptr)
    y = torch.tensor(y0, dtype=torch.float64, device="cuda")
    for k, exp in zip((1, 2), expected):
        pg = torch.tensor(o.b2g(b.power_vector(sc.block_power[k]).copy(), True), dtype=torch.float64,
                          device="cuda")
        torch.cuda.synchronize()
        st = _abi.Stats()
        rc = L.hsb_dev_transient_noalloc(dev, C.c_void_p(y.data_ptr()), C.c_void_p(pg.data_ptr()),
                                         sc.dt, C.byref(st))
        assert rc == 0, L.hsb_dev_last_error().decode()
        assert st.rk4_steps >= 1
        got = y.cpu().numpy()
        assert np.max(np.abs(got - exp)) <= TOL
    a.close()
    b.close()


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
