"""Grid-state checkpoints and the grid text dumps.

A checkpoint (hsb_grid_save_state) holds both grid vectors; a second model
of the same grid that loads it continues the transient bit for bit as the
first one does, and a model of another grid refuses it.  The dumps
(dump_transient_temp_grid, dump_steady_temp_grid) print the device state in
the reference's text format, "t = %lf", "Layer %d:" and "%d\\t%.2f" rows
(temperature_grid.c:1262-1319), byte for byte."""
import os

import numpy as np
import pytest

from hotspot_b200 import FORM_FAST, _abi
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W

pytestmark = pytest.mark.gpu


def test_checkpoint_resumes_bit_for_bit(workdir):
    sc = W.scenario_chip2d(workdir, seed=81, grid=32, steps=8)
    a, b = hm.from_scenario(sc), hm.from_scenario(sc)
    a.set_solver(FORM_FAST)
    b.set_solver(FORM_FAST)
    powers = np.stack([a.power_vector(sc.block_power[k]) for k in range(sc.steps)])
    a.compute_trace(powers[:4], a.vector(a.config.init_temp), sc.dt)
    a.steady(powers.mean(0).copy(), a.vector())
    path = os.path.join(workdir, "state.bin")
    a.save_state(path)
    b.load_state(path)
    assert np.array_equal(b.grid("trans"), a.grid("trans"))
    assert np.array_equal(b.grid("steady"), a.grid("steady"))
    out_a, _ = a.compute_trace(powers[4:], None, sc.dt)
    out_b, _ = b.compute_trace(powers[4:], None, sc.dt)
    assert np.array_equal(out_a, out_b)
    assert np.array_equal(a.grid("trans"), b.grid("trans"))
    other = hm.from_scenario(W.scenario_chip2d(workdir, seed=82, grid=16, steps=2))
    with pytest.raises(_abi.HotspotError, match="checkpoint"):
        other.load_state(path)
    for m in (a, b, other):
        m.close()


def _layers_text(m, g):
    plane = m.n_cells // m.n_layers
    out = []
    for l in range(m.n_layers):
        out.append("Layer %d:\n" % l)
        out.extend("%d\t%.2f\n" % (k, x) for k, x in enumerate(g[l * plane:(l + 1) * plane]))
    return "".join(out)


def test_dumps_match_the_reference_format(workdir):
    sc = W.scenario_stack3d(workdir, seed=83, grid=64, steps=3, n_blocks=12)
    m = hm.from_scenario(sc)
    m.set_solver(FORM_FAST)
    t = m.vector(m.config.init_temp)
    for k in range(2):
        m.compute_temp(m.power_vector(sc.block_power[k]).copy(), t if k == 0 else None, sc.dt)
    path = os.path.join(workdir, "grid.ttrace")
    m.dump_transient(1, sc.dt, path)
    m.dump_transient(2, sc.dt, path)   # appends
    frame = _layers_text(m, m.grid("trans"))
    want = "t = %f\n" % (1 * sc.dt) + frame + "t = %f\n" % (2 * sc.dt) + frame
    assert open(path).read() == want
    m.steady(m.power_vector(sc.block_power.mean(0)).copy(), m.vector())
    spath = os.path.join(workdir, "grid.steady")
    _abi.lib().dump_steady_temp_grid(m.ptr, spath.encode())
    assert open(spath).read() == _layers_text(m, m.grid("steady"))
    m.close()
