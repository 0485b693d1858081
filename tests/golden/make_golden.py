"""Generate the golden vectors in tests/golden/ from the reference itself.

Runs the reference HotSpot C code (oracle/_ref/libhsref.so, built from the
HotSpot sources by `make -C oracle ref`) on small seeded scenarios and saves
its in-memory FP64 results: block temperatures after every sampling interval,
the final transient grid vector, the steady block and grid vectors.  The
scenario inputs are regenerated from their seeds by hotspot_b200.workloads;
the power rows used are stored too, so a change of the generator is caught.

    python tests/golden/make_golden.py [case ...]
"""
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from hotspot_b200 import workloads as W  # noqa: E402
from oracle.ref import RefModel  # noqa: E402


def cases(d):
    """name -> (scenario, intervals)"""
    out = {}
    out["chip2d_16"] = (W.scenario_chip2d(d, seed=0, grid=16, steps=6), 6)
    sc = W.scenario_chip2d(d, seed=1, grid=32, steps=5)
    sc.config["grid_map_mode"] = "avg"
    out["chip2d_32_avg"] = (sc, 5)
    out["stack3d_32"] = (W.scenario_stack3d(d, seed=2, grid=32, steps=4, n_blocks=10), 4)
    sc = W.scenario_stack3d(d, seed=3, grid=16, steps=3, n_blocks=6)
    sc.detailed_3D = True
    sc.config["grid_map_mode"] = "max"
    out["detailed_16_max"] = (sc, 3)
    sc = W.scenario_microchannel(d, seed=4, grid=32, die=2e-3, channel_w=125e-6, channel_h=125e-6,
                                 pitch=250e-6, blocks=8)
    sc.block_power = np.repeat(sc.block_power, 2, axis=0)
    sc.dt = 1e-5
    out["microchannel_32"] = (sc, 2)
    # the secondary heat path: five more chip-side layers (substrate, solder,
    # PCB ...) and 16 more package nodes (temperature_grid.c:2228-2379)
    sc = W.scenario_chip2d(d, seed=9, grid=16, steps=4)
    sc.config["model_secondary"] = "1"
    out["secondary_16"] = (sc, 4)
    return out


def run(sc, intervals, steady=True):
    m = RefModel(sc)
    t = m.vector(333.15)
    temps, powers = [], []
    for k in range(intervals):
        p = m.power_vector(sc.block_power[k])
        powers.append(p.copy())
        m.compute_temp(p, t if k == 0 else None, sc.dt)
        temps.append(t.copy())
    res = {"block_power": np.array(powers), "temps": np.array(temps), "grid_trans": m.grid("trans")}
    if steady:
        avg = m.power_vector(sc.block_power[:intervals].mean(0))
        s = m.vector()
        m.steady(avg.copy(), s)
        res["steady_power"] = avg
        res["steady"] = s
        res["grid_steady"] = m.grid("steady")
    m.close()
    return res


def main(names=None):
    with tempfile.TemporaryDirectory() as d:
        for name, (sc, n) in cases(d).items():
            if names and name not in names:
                continue
            res = run(sc, n, steady=not sc.use_microchannels)
            np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **res)
            print(name, {k: v.shape for k, v in res.items()})


if __name__ == "__main__":
    main(sys.argv[1:])
