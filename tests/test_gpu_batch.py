"""Batched fast transient (hsb_batch_transient / _trace): many models of
uneven size in one persistent launch of the temporally blocked kernel.  Each
model's arithmetic is that of the single-model fast form, so the batch must
reproduce the single-model results on the same tiles -- the same accepted
steps, temperatures within 1e-9 K -- for every chip, whether it runs on a CTA
group (with chip-local barriers) or shares a CTA with others, and whether its
intervals run one per call or K per launch."""
import numpy as np
import pytest

from hotspot_b200 import FORM_FAST_BLOCKED
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from hotspot_b200.batch import Batch

pytestmark = pytest.mark.gpu
TOL = 1e-9


def _chips(workdir, specs):
    out = []
    for k, (kind, grid) in enumerate(specs):
        if kind == "chip2d":
            sc = W.scenario_chip2d(workdir, seed=60 + k, grid=grid, steps=8)
        elif kind == "secondary":
            sc = W.scenario_chip2d(workdir, seed=60 + k, grid=grid, steps=8)
            sc.config["model_secondary"] = "1"
        elif kind == "random":
            sc = W.scenario_random_chip(workdir, np.random.default_rng(60 + k), f"r{k}", side=grid, steps=8)
        else:
            sc = W.scenario_stack3d(workdir, seed=60 + k, grid=grid, steps=8, n_blocks=10)
        sc.dt = 3.333e-6            # one sampling interval for the whole batch
        out.append(sc)
    return out


def _models(scs):
    single, batched = [], []
    for sc in scs:
        for lst in (single, batched):
            m = hm.from_scenario(sc)
            m.set_solver(FORM_FAST_BLOCKED)
            t = m.vector(m.config.init_temp)
            m.compute_temp(m.power_vector(sc.block_power[0]), t, 0.0)
            lst.append(m)
    return single, batched


def _run(scs, intervals, schedule=None, per_launch=1):
    single, batched = _models(scs)
    bt = Batch(batched)
    if schedule:
        bt.set_schedule(*schedule)
    for c, a in enumerate(single):     # the single models on the batch's tiles: the same sums
        a.set_tile(*bt.tile(c))
    steps_single = np.zeros(len(scs), dtype=np.int64)
    steps_batch = np.zeros(len(scs), dtype=np.int64)
    for k in range(1, intervals + 1):
        for i, (sc, a) in enumerate(zip(scs, single)):
            a.compute_temp(a.power_vector(sc.block_power[k]), None, sc.dt)
            steps_single[i] += a.stats()["rk4_steps"]
    k = 1
    while k <= intervals:
        kk = min(per_launch, intervals + 1 - k)
        rows = [[b.power_vector(sc.block_power[k + j]) for sc, b in zip(scs, batched)] for j in range(kk)]
        if kk == 1:
            bt.transient(rows[0], scs[0].dt)
        else:
            bt.trace(rows, scs[0].dt)
        steps_batch += bt.chip_steps()
        k += kk
    errs = [float(np.max(np.abs(a.grid("trans") - b.grid("trans")))) for a, b in zip(single, batched)]
    info = bt.info()
    bt.close()
    for m in single + batched:
        m.close()
    return errs, steps_single, steps_batch, info


def test_batch_matches_single_models(workdir):
    scs = _chips(workdir, [("chip2d", 32), ("stack3d", 64), ("chip2d", 64), ("stack3d", 32), ("chip2d", 128),
                           ("secondary", 32), ("random", 64)])
    errs, s1, s2, info = _run(scs, 5)
    assert np.array_equal(s1, s2), (s1, s2)
    assert max(errs) <= TOL, errs


@pytest.mark.parametrize("schedule", [(0, 1.0), (2, 4.0), (1, 0.25)])
def test_batch_schedules(workdir, schedule):
    """Chips split over CTA groups (chip-local barriers) and packed chips,
    under every tile policy."""
    scs = _chips(workdir, [("stack3d", 256), ("chip2d", 32), ("chip2d", 64), ("stack3d", 64)] * 2)
    errs, s1, s2, info = _run(scs, 3, schedule)
    assert np.array_equal(s1, s2) and max(errs) <= TOL, (errs, info)


def test_batch_trace_matches_single_intervals(workdir):
    """K intervals per launch (block powers mapped in the kernel) against
    single-model calls interval by interval."""
    scs = _chips(workdir, [("stack3d", 128), ("chip2d", 32), ("random", 64), ("chip2d", 64)])
    errs, s1, s2, info = _run(scs, 7, per_launch=4)
    assert np.array_equal(s1, s2), (s1, s2)
    assert max(errs) <= TOL, errs


def test_batch_autotuner(workdir):
    """The autotuner runs each candidate schedule on a real interval; results
    stay within 1e-9 K of the single-model form and a measured candidate wins."""
    scs = _chips(workdir, [("stack3d", 64), ("chip2d", 32), ("chip2d", 64)] * 2)
    for sc in scs:
        sc.block_power = np.repeat(sc.block_power, 2, axis=0)
    single, batched = _models(scs)
    bt = Batch(batched)
    bt.autotune(True)
    for k in range(1, 12):
        for sc, a in zip(scs, single):
            a.compute_temp(a.power_vector(sc.block_power[k]), None, sc.dt)
        bt.transient([b.power_vector(sc.block_power[k]) for sc, b in zip(scs, batched)], scs[0].dt)
    tun = bt.tuning()
    info = bt.info()
    errs = [float(np.max(np.abs(a.grid("trans") - b.grid("trans")))) for a, b in zip(single, batched)]
    bt.close()
    for m in single + batched:
        m.close()
    assert len(tun) == 9 and all(t["ms_per_gcell_step"] > 0 for t in tun)
    best = min(tun, key=lambda t: t["ms_per_gcell_step"])
    assert info["policy"] == best["policy"] and info["split"] == best["split"]
    assert max(errs) <= TOL, errs


def test_batch_subset_launches(workdir):
    """Launches over a subset of the models, a few intervals each (the ticks of
    the serving batch engine): the listed chips match the single-model form
    on the same tiles (same steps, 1e-9 K) and the others keep their state
    bit for bit."""
    scs = _chips(workdir, [("stack3d", 128), ("chip2d", 32), ("random", 64), ("chip2d", 64), ("secondary", 32)])
    single, batched = _models(scs)
    bt = Batch(batched)
    bt.set_ctas(40)                    # fewer CTAs than the device holds: groups shrink
    for c, a in enumerate(single):
        a.set_tile(*bt.tile(c))
    done = [0] * len(scs)
    for chips, K in [([2, 0], 3), ([1, 3, 4], 2), ([4, 0, 2, 1, 3], 1), ([3], 2)]:
        before = {c: batched[c].grid("trans") for c in range(len(scs)) if c not in chips}
        rows = [[batched[c].power_vector(scs[c].block_power[1 + done[c] + j]) for c in chips] for j in range(K)]
        st = bt.run_subset(chips, rows, scs[0].dt)
        assert st["launches"] == 1
        steps = bt.chip_steps()
        for c in chips:
            s1 = 0
            for j in range(K):
                single[c].compute_temp(single[c].power_vector(scs[c].block_power[1 + done[c] + j]), None, scs[c].dt)
                s1 += single[c].stats()["rk4_steps"]
            assert steps[c] == s1, (c, steps[c], s1)
            done[c] += K
        for c, g in before.items():
            assert np.array_equal(batched[c].grid("trans"), g), c
    errs = [float(np.max(np.abs(a.grid("trans") - b.grid("trans")))) for a, b in zip(single, batched)]
    bt.close()
    for m in single + batched:
        m.close()
    assert max(errs) <= TOL, errs
