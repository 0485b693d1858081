"""The temperature-leakage fixed point on the device (hsb_grid_steady_leakage)
against the reference's loop (temperature.c:706-746, calc_leakage at
temperature.c:910-927) restated here on the host over the same steady
solver: the same number of steady solves and block temperatures within
1e-9 K in the parity form (the device and host exp may differ in the last
bit); the fast form within 0.01 K of the parity form."""
import numpy as np
import pytest

from hotspot_b200 import FORM_FAST
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _host_loop(m, power, temp):
    """temperature.c:706-746 with steady_state_temp_grid = m.steady."""
    h, w = m.block_dims()
    pw = h > 0
    temp = temp.copy()
    for it in range(101):
        new = np.zeros_like(power)
        new[:h.size][pw] = power[:h.size][pw] + 1.5e4 * h[pw] * w[pw] * np.exp(0.036 * (temp[:h.size][pw] - 383.15))
        old = temp[:h.size][pw].copy()
        m.steady(new, temp)
        dmax = max(0.0, float(np.max(temp[:h.size][pw] - old)))
        if dmax < 0.01:
            return temp, it + 1
    raise RuntimeError("no convergence")


@pytest.mark.parametrize("case", ["chip2d", "stack3d"])
def test_leakage_loop_on_device(workdir, case):
    if case == "chip2d":
        sc = W.scenario_chip2d(workdir, seed=71, grid=32, steps=2)
    else:
        sc = W.scenario_stack3d(workdir, seed=72, grid=32, steps=2, n_blocks=8)
    out = {}
    for form in (None, FORM_FAST):
        m = hm.from_scenario(sc)
        if form is not None:
            m.set_solver(form)
        # a start at ambient, so the first solve is a rise and the loop takes several
        p = m.power_vector(0.5 * sc.block_power.mean(0))
        t0 = m.vector(m.config.ambient)
        t_dev = t0.copy()
        n_dev = m.steady_leakage(p.copy(), t_dev)
        t_host, n_host = _host_loop(m, p.copy(), t0)
        assert n_dev == n_host and n_dev >= 2, (n_dev, n_host)
        assert np.max(np.abs(t_dev - t_host)) <= (1e-9 if form is None else 1e-6)
        out[form] = t_dev
        m.close()
    assert np.max(np.abs(out[None] - out[FORM_FAST])) <= 0.01
