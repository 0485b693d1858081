"""The JSON contract of bench.py's reference arm (runs on the host cores).

`bench.py --impl reference` times the reference's own C implementation of
the grid model (oracle/_ref, compiled from the HotSpot sources) on the
headline workload and prints one JSON line with the same metric, unit and
config object as the GPU arm.  Under torchrun only rank 0 prints.
"""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _run(env_extra):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "1"], capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)


def test_reference_arm_line():
    import bench
    from oracle import ref as R
    r = _run({"RANK": "0", "WORLD_SIZE": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads([l for l in r.stdout.splitlines() if l.startswith("{")][-1])
    assert line["impl"] == "reference"
    assert line["metric"] == bench.METRIC and line["unit"] == "cell-steps/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 1
    assert line["config"] == bench.headline_config(256, 6 * 256 * 256, 1)
    cb = line["cpu_baseline"]
    assert cb["value"] == line["value"] and cb["cores"] >= 1
    assert cb["kind"] == ("reference" if R.available() else "port")
    assert line["e2e"] == {"value": line["value"], "unit": "cell-steps/s", "h2d_bytes_per_step": 0,
                           "d2h_bytes_per_step": 0}


def test_reference_arm_other_ranks_are_silent():
    r = _run({"RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert not [l for l in r.stdout.splitlines() if l.startswith("{")]
