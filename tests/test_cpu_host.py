"""Host-side logic without a GPU: the reference's fatal() error behaviour of
the C entry points (checked in a child process, since fatal exits), the
loud failure when no GPU is visible, and the seeded input generators."""
import os
import subprocess
import sys
import textwrap

import numpy as np
import pytest

from hotspot_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _child(code: str):
    r = subprocess.run([sys.executable, "-c", textwrap.dedent(code)], cwd=ROOT, capture_output=True,
                       text=True, env={**os.environ, "CUDA_VISIBLE_DEVICES": ""})
    return r.returncode, r.stdout + r.stderr


PRELUDE = """
import sys, ctypes as C
sys.path.insert(0, '.')
from hotspot_b200 import _abi, model as hm, workloads as W
L = _abi.lib()
"""


def test_non_power_of_two_grid_is_fatal(workdir):
    rc, out = _child(PRELUDE + f"""
sc = W.scenario_chip2d({workdir!r}, seed=0, grid=16, steps=1)
cfg = hm.default_thermal_config()
hm.thermal_config_add_from_strs(cfg, None, dict(sc.config, grid_rows='48'))
flp = hm.read_flp(sc.flp)
L.alloc_grid_model(C.byref(cfg), flp, None, None, 0, 0)
print('not reached')
""")
    assert rc == 1 and "error: grid rows and columns should both be powers of two" in out


def test_unknown_map_mode_is_fatal(workdir):
    rc, out = _child(PRELUDE + f"""
sc = W.scenario_chip2d({workdir!r}, seed=0, grid=16, steps=1)
cfg = hm.default_thermal_config()
hm.thermal_config_add_from_strs(cfg, None, dict(sc.config, grid_map_mode='median'))
L.alloc_grid_model(C.byref(cfg), hm.read_flp(sc.flp), None, None, 0, 0)
""")
    assert rc == 1 and "error: unknown mapping mode" in out


def test_bad_layer_file_is_fatal(workdir):
    lcf = os.path.join(workdir, "bad.lcf")
    open(lcf, "w").write("0\nY\nQ\n1.75e6\n0.01\n1e-4\nx.flp\n")
    rc, out = _child(PRELUDE + f"""
cfg = hm.default_thermal_config()
hm.thermal_config_add_from_strs(cfg, None, dict(model_type='grid', grid_layer_file={lcf!r}))
L.alloc_grid_model(C.byref(cfg), None, None, None, 0, 0)
""")
    assert rc == 1 and "error: invalid layer power dissipation indicator" in out


def test_missing_floorplan_in_lcf_is_fatal(workdir):
    lcf = os.path.join(workdir, "m.lcf")
    open(lcf, "w").write("0\nY\nY\n1.75e6\n0.01\n1e-4\n/nonexistent/x.flp\n")
    rc, out = _child(PRELUDE + f"""
cfg = hm.default_thermal_config()
hm.thermal_config_add_from_strs(cfg, None, dict(model_type='grid', grid_layer_file={lcf!r}))
L.alloc_grid_model(C.byref(cfg), None, None, None, 0, 0)
""")
    assert rc == 1 and "error opening file /nonexistent/x.flp" in out


def test_no_gpu_fails_loudly(workdir):
    rc, out = _child(PRELUDE + f"""
sc = W.scenario_chip2d({workdir!r}, seed=0, grid=16, steps=1)
try:
    hm.from_scenario(sc)
except _abi.HotspotError as e:
    print('raised:', e); sys.exit(3)
""")
    assert rc == 3 and "no CUDA device" in out


DROPIN_BIN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "..", "oracle", "_ref", "hotspot_b200drv")


@pytest.mark.skipif(not os.path.exists(DROPIN_BIN), reason="drop-in CLI not built (make -C oracle dropin)")
def test_dropin_cli_fails_loudly_without_gpu(workdir):
    """HotSpot's own CLI linked against this library stops with the library's
    fatal() message when no GPU is visible: there is no CPU path."""
    from conftest import has_gpu
    if has_gpu():
        pytest.skip("a GPU is visible")
    sc = W.scenario_chip2d(workdir, seed=0, grid=16, steps=2)
    ptrace = W.write_ptrace(os.path.join(workdir, "p.ptrace"), sc.power_layers[0], sc.block_power)
    r = subprocess.run([DROPIN_BIN, "-f", sc.flp, "-p", ptrace, "-model_type", "grid", "-grid_rows", "16",
                        "-grid_cols", "16"], cwd=workdir, capture_output=True, text=True, timeout=120)
    assert r.returncode == 1 and "no CUDA device" in r.stdout + r.stderr


def test_status_api_reports_instead_of_exiting(workdir):
    rc, out = _child(PRELUDE + f"""
sc = W.scenario_chip2d({workdir!r}, seed=0, grid=16, steps=1)
cfg = hm.default_thermal_config()
hm.thermal_config_add_from_strs(cfg, None, dict(sc.config, grid_cols='12'))
g = C.POINTER(_abi.GridModel)()
r = L.hsb_grid_alloc(C.byref(g), C.byref(cfg), hm.read_flp(sc.flp), None, None, 0, 0)
print('rc', r, L.hsb_last_error().decode().strip())
""")
    assert rc == 0 and "rc -1 grid rows and columns should both be powers of two" in out


@pytest.mark.parametrize("n", [10, 15, 40, 100])
def test_guillotine_floorplan_tiles_the_die(n):
    rng = np.random.default_rng(n)
    units = W.guillotine_floorplan(rng, 16e-3, 12e-3, n)
    assert len(units) == n
    assert abs(sum(u.width * u.height for u in units) - 16e-3 * 12e-3) < 1e-15
    for u in units:
        assert 0.33 - 1e-9 <= u.width / u.height <= 3.0 + 1e-9
        assert u.leftx >= -1e-15 and u.bottomy >= -1e-15
        assert u.leftx + u.width <= 16e-3 + 1e-15 and u.bottomy + u.height <= 12e-3 + 1e-15


def test_ar1_power_is_seeded_and_nonnegative():
    a = W.ar1_power(np.random.default_rng(3), np.array([0.5, 5.0, 20.0]), 500)
    b = W.ar1_power(np.random.default_rng(3), np.array([0.5, 5.0, 20.0]), 500)
    assert np.array_equal(a, b) and a.min() >= 0.0
    assert abs(a[:, 2].mean() - 20.0) < 1.0


def test_straight_channels_layout(workdir):
    path, lanes = W.straight_channels_csv(os.path.join(workdir, "c.csv"), 32, 32, 62.5e-6, 125e-6, 250e-6)
    t = np.loadtxt(path, delimiter=",", dtype=int)
    assert lanes == 8 and set(np.unique(t)) <= {0, 1, 2, 3}
    assert (t[0][t[0] > 0] == 2).all() and (t[-1][t[-1] > 0] == 3).all()
