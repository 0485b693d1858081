"""The drop-in at the level of HotSpot's own command-line driver.

`make -C oracle dropin` links the reference's hotspot.c, with every reference
object but temperature_grid.o, against libhotspot_b200 -- what a HotSpot user
does to put the GPU under the grid model (oracle/_ref/hotspot_b200drv).  The
reference's own build of the same sources is oracle/_ref/hotspot.  Both run
the same floorplan and power trace (also with the secondary heat path,
-model_secondary 1); in the default (parity) form every output
file -- the block transient trace, the steady block temperatures and the grid
dumps of the steady and of every transient interval -- must be identical,
byte for byte."""
import os
import subprocess

import numpy as np

import pytest

from hotspot_b200 import workloads as W

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
REF_BIN = os.path.join(HERE, "..", "oracle", "_ref", "hotspot")
DROPIN_BIN = os.path.join(HERE, "..", "oracle", "_ref", "hotspot_b200drv")


@pytest.mark.skipif(not (os.path.exists(REF_BIN) and os.path.exists(DROPIN_BIN)),
                    reason="reference build not present (make -C oracle ref dropin)")
@pytest.mark.parametrize("grid,seed,extra", [(32, 91, []), (64, 92, []), (32, 94, ["-model_secondary", "1"])])
def test_cli_outputs_identical(workdir, grid, seed, extra):
    sc = W.scenario_chip2d(workdir, seed=seed, grid=grid, steps=20)
    ptrace = W.write_ptrace(os.path.join(workdir, "p.ptrace"), sc.power_layers[0], sc.block_power)
    outs = ("ttrace", "steady", "grid.steady", "grid.ttrace")
    env = {k: v for k, v in os.environ.items() if k != "HOTSPOT_B200_FORM"}
    for tag, exe in (("ref", REF_BIN), ("gpu", DROPIN_BIN)):
        args = [exe, "-f", sc.flp, "-p", ptrace, "-o", f"{tag}.ttrace", "-model_type", "grid",
                "-grid_rows", str(grid), "-grid_cols", str(grid), "-sampling_intvl", "3.333e-06",
                "-steady_file", f"{tag}.steady", "-grid_steady_file", f"{tag}.grid.steady",
                "-grid_transient_file", f"{tag}.grid.ttrace"] + extra
        r = subprocess.run(args, cwd=workdir, capture_output=True, text=True, timeout=600, env=env)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
    for o in outs:
        a = open(os.path.join(workdir, f"ref.{o}"), "rb").read()
        b = open(os.path.join(workdir, f"gpu.{o}"), "rb").read()
        assert len(a) > 0 and a == b, o


@pytest.mark.skipif(not (os.path.exists(REF_BIN) and os.path.exists(DROPIN_BIN)),
                    reason="reference build not present (make -C oracle ref dropin)")
@pytest.mark.parametrize("detailed", ["off", "on"])
def test_cli_layer_stack_identical(workdir, detailed):
    """The 4-layer stack from a layer configuration file, with uniform and
    with detailed (per-cell) R/C assignment."""
    sc = W.scenario_stack3d(workdir, seed=93, grid=32, steps=10, n_blocks=10)
    ptrace = W.write_ptrace(os.path.join(workdir, "p.ptrace"), sc.power_layers[0] + sc.power_layers[2],
                            sc.block_power)
    flp0 = sc.lcf.replace(".lcf", "_si0.flp")
    env = {k: v for k, v in os.environ.items() if k != "HOTSPOT_B200_FORM"}
    for tag, exe in (("ref", REF_BIN), ("gpu", DROPIN_BIN)):
        args = [exe, "-f", flp0, "-p", ptrace, "-o", f"{tag}.ttrace", "-model_type", "grid", "-grid_rows", "32",
                "-grid_cols", "32", "-sampling_intvl", "1e-05", "-grid_layer_file", sc.lcf, "-detailed_3D", detailed,
                "-steady_file", f"{tag}.steady", "-grid_steady_file", f"{tag}.grid.steady"]
        r = subprocess.run(args, cwd=workdir, capture_output=True, text=True, timeout=600, env=env)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
    for o in ("ttrace", "steady", "grid.steady"):
        a = open(os.path.join(workdir, f"ref.{o}"), "rb").read()
        b = open(os.path.join(workdir, f"gpu.{o}"), "rb").read()
        assert len(a) > 0 and a == b, o


@pytest.mark.skipif(not (os.path.exists(REF_BIN) and os.path.exists(DROPIN_BIN)),
                    reason="reference build not present (make -C oracle ref dropin)")
def test_cli_leakage_loop_identical(workdir):
    """The reference's temperature-leakage fixed point (temperature.c:708-746),
    a host loop of steady solves, over this library's steady solver."""
    sc = W.scenario_chip2d(workdir, seed=95, grid=32, steps=4)
    ptrace = W.write_ptrace(os.path.join(workdir, "p.ptrace"), sc.power_layers[0], sc.block_power)
    env = {k: v for k, v in os.environ.items() if k != "HOTSPOT_B200_FORM"}
    for tag, exe in (("ref", REF_BIN), ("gpu", DROPIN_BIN)):
        args = [exe, "-f", sc.flp, "-p", ptrace, "-model_type", "grid", "-grid_rows", "32", "-grid_cols", "32",
                "-leakage_used", "1", "-steady_file", f"{tag}.steady", "-grid_steady_file", f"{tag}.grid.steady"]
        r = subprocess.run(args, cwd=workdir, capture_output=True, text=True, timeout=600, env=env)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
    for o in ("steady", "grid.steady"):
        a = open(os.path.join(workdir, f"ref.{o}"), "rb").read()
        b = open(os.path.join(workdir, f"gpu.{o}"), "rb").read()
        assert len(a) > 0 and a == b, o


@pytest.mark.skipif(not (os.path.exists(REF_BIN) and os.path.exists(DROPIN_BIN)),
                    reason="reference build not present (make -C oracle ref dropin)")
def test_cli_microchannel_transient_identical(workdir):
    """A microchannel-cooled stack (-use_microchannels 1 -detailed_3D on,
    hotspot.c:496-497) through the CLI: the block and grid transient traces
    are identical byte for byte.  The driver then computes the steady state,
    which for microchannel models the reference only has with SuperLU: its
    build stops there with exit status 1 after writing the traces, while this
    library solves it (BiCGStab with FP64 refinement) and the run completes."""
    sc = W.scenario_microchannel(workdir, seed=6, grid=32, die=2e-3, channel_w=125e-6, channel_h=125e-6,
                                 pitch=250e-6, blocks=8)
    rows = sc.block_power.repeat(4, axis=0) * (1.0 + 0.1 * np.arange(4))[:, None]
    ptrace = W.write_ptrace(os.path.join(workdir, "p.ptrace"), sc.power_layers[0], rows)
    flp0 = sc.lcf.replace(".lcf", "_si.flp")
    env = {k: v for k, v in os.environ.items() if k != "HOTSPOT_B200_FORM"}
    for tag, exe in (("ref", REF_BIN), ("gpu", DROPIN_BIN)):
        args = [exe, "-f", flp0, "-p", ptrace, "-o", f"{tag}.ttrace", "-model_type", "grid", "-grid_rows", "32",
                "-grid_cols", "32", "-sampling_intvl", "1e-05", "-grid_layer_file", sc.lcf, "-detailed_3D", "on",
                "-use_microchannels", "1", "-materials_file", sc.materials,
                "-pumping_pressure", sc.config["pumping_pressure"], "-inlet_temperature", "300",
                "-coolant_material", "water", "-grid_map_mode", "avg",
                "-grid_transient_file", f"{tag}.grid.ttrace"]
        r = subprocess.run(args, cwd=workdir, capture_output=True, text=True, timeout=600, env=env)
        if tag == "ref":
            assert r.returncode == 1, (tag, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
            assert "Steady-state computations with microfluidic cooling" in r.stderr, (tag, r.stderr[-2000:])
        else:
            assert r.returncode == 0, (tag, r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    for o in ("ttrace", "grid.ttrace"):
        a = open(os.path.join(workdir, f"ref.{o}"), "rb").read()
        b = open(os.path.join(workdir, f"gpu.{o}"), "rb").read()
        assert len(a) > 0 and a == b, o


PACKAGE_NATURAL = """\
# natural convection heat sink (fin-channel), package model of HotSpot's CLI
-natural_convec 1
-flow_type 0
-sink_type 0
-fin_height 0.03
-fin_width 0.001
-channel_width 0.002
-pin_height 0.02
-pin_diam 0.002
-pin_dist 0.005
-fan_radius 0.03
-motor_radius 0.01
-rpm 1000
"""


@pytest.mark.skipif(not (os.path.exists(REF_BIN) and os.path.exists(DROPIN_BIN)),
                    reason="reference build not present (make -C oracle ref dropin)")
def test_cli_natural_convection_identical(workdir):
    """The natural-convection loop of hotspot.c:668-682: steady solve, sink
    temperature, new convection resistance from the package model,
    populate_R_model again (this library re-uploads the conductances), until
    the resistance settles -- the steady outputs identical byte for byte."""
    sc = W.scenario_chip2d(workdir, seed=96, grid=32, steps=6)
    ptrace = W.write_ptrace(os.path.join(workdir, "p.ptrace"), sc.power_layers[0], sc.block_power * 0.05)
    pkg = os.path.join(workdir, "natural.config")
    with open(pkg, "w") as f:
        f.write(PACKAGE_NATURAL)
    env = {k: v for k, v in os.environ.items() if k != "HOTSPOT_B200_FORM"}
    for tag, exe in (("ref", REF_BIN), ("gpu", DROPIN_BIN)):
        args = [exe, "-f", sc.flp, "-p", ptrace, "-o", f"{tag}.ttrace", "-model_type", "grid", "-grid_rows", "32",
                "-grid_cols", "32", "-package_model_used", "1", "-package_config_file", pkg,
                "-steady_file", f"{tag}.steady", "-grid_steady_file", f"{tag}.grid.steady"]
        r = subprocess.run(args, cwd=workdir, capture_output=True, text=True, timeout=900, env=env)
        assert r.returncode == 0, (tag, r.stdout[-2000:], r.stderr[-2000:])
    for o in ("ttrace", "steady", "grid.steady"):
        a = open(os.path.join(workdir, f"ref.{o}"), "rb").read()
        b = open(os.path.join(workdir, f"gpu.{o}"), "rb").read()
        assert len(a) > 0 and a == b, o
