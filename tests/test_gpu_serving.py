"""Serving loop (hsb_server_run): requests over resident models, admitted
continuously, several in flight on their models' streams.  Every result must
be the same alone and in the mix (bit for bit: the kernels are
deterministic and models share no device state), and the steady results
must meet the 0.01 K bar against the converged FP64 solution."""
import numpy as np
import pytest

from hotspot_b200 import _abi
from hotspot_b200 import model as hm
from hotspot_b200 import workloads as W
from hotspot_b200.serving import Request, Server, latency_report
from oracle.restatement import OracleModel

pytestmark = pytest.mark.gpu


def _requests(server, scs, models, rng, n, rate):
    reqs, t = [], 0.0
    for k in range(n):
        t += rng.exponential(1.0 / rate)
        mi = int(rng.integers(0, len(models)))
        m, sc = models[mi], scs[mi]
        nblk = sum(m.layer_units[l] for l in range(m.n_layers) if m.layer_power[l])
        if mi < 2:
            reqs.append(Request(mi, _abi.REQ_STEADY, m.power_vector(rng.uniform(0.5, 20.0, nblk)), t,
                                tag=f"steady{mi}"))
        else:
            # 70 intervals: more than one launch chunk of a background transient
            trace = W.ar1_power(rng, rng.uniform(0.5, 20.0, nblk), 70)
            p = np.stack([m.power_vector(trace[s]) for s in range(70)])
            reqs.append(Request(mi, _abi.REQ_TRANSIENT, p, t, temp_in=m.vector(m.config.init_temp), steps=70,
                                dt=3.333e-6, tag="transient"))
    return reqs


def test_alone_equals_mixed(workdir):
    rng = np.random.default_rng(90)
    scs = [W.scenario_random_chip(workdir, rng, "a", side=64, chip_layers=2, steps=0),
           # 256x256x8 = 2^19 cells: a background steady solve this large runs
           # its passes iteration by iteration in the mixed run
           W.scenario_random_chip(workdir, rng, "b", side=256, chip_layers=6, steps=0),
           W.scenario_random_chip(workdir, rng, "c", side=64, chip_layers=4, steps=0)]
    models = [hm.from_scenario(sc) for sc in scs]
    srv = Server(workers=4)
    for m in models:
        srv.add_model(m, _abi.FORM_FAST, 1e-6)
    # a high-priority class: its own stream priority and workers, dispatched
    # first; in the mixed run the other requests pause between chunks while it
    # runs, alone (no high-priority request in the run) they run unchunked
    srv.set_priority(0, True)
    mixed = _requests(srv, scs, models, np.random.default_rng(91), 24, 4000.0)
    # alone: the same requests one at a time
    alone = [Request(r.model, r.kind, r.power, 0.0, r.temp_in, r.steps, r.dt, r.tag) for r in mixed]
    for r in alone:
        srv.run([r])
    srv.run(mixed)
    for a, b in zip(alone, mixed):
        assert a.status == 0 and b.status == 0
        assert np.array_equal(a.out, b.out), (a.tag, np.max(np.abs(a.out - b.out)))
    # overlap: some requests were in flight together
    spans = sorted((r.start, r.finish) for r in mixed)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))
    # the steady answers against the converged FP64 solution
    for r in mixed[:6]:
        if r.kind == _abi.REQ_STEADY and models[r.model].n_cells <= 1 << 17:   # sparse LU stays quick
            T, Tb = OracleModel(scs[r.model]).steady_direct(r.power)
            assert np.max(np.abs(r.out - Tb)) <= 0.01
    rep = latency_report(mixed)
    assert rep["n"] == len(mixed) and rep["p99_ms"] >= rep["p50_ms"] > 0
    srv.close()
    for m in models:
        m.close()


def test_admission_refuses_what_does_not_fit(workdir):
    rng = np.random.default_rng(92)
    sc = W.scenario_random_chip(workdir, rng, "d", side=64, chip_layers=2, steps=0)
    m = hm.from_scenario(sc)
    srv = Server(workers=2, reserve_bytes=1 << 62)      # no request can be admitted
    srv.add_model(m, _abi.FORM_FAST, 1e-6)
    nblk = sum(m.layer_units[l] for l in range(m.n_layers) if m.layer_power[l])
    r = Request(0, _abi.REQ_STEADY, m.power_vector(np.ones(nblk)), 0.0)
    with pytest.raises(Exception):
        srv.run([r])
    assert r.status == -3                               # HSB_E_NOMEM
    srv.close()
    m.close()


def test_pool_members_serve_one_class(workdir):
    """A pool of resident models of one class: requests naming the pool run on
    whichever member is idle, concurrently; each result equals the result of
    the same request alone on the pool's first model, bit for bit (members
    are built from the same scenario and every request carries its inputs)."""
    rng = np.random.default_rng(93)
    sc = W.scenario_random_chip(workdir, rng, "p", side=128, chip_layers=3, steps=0)
    members = [hm.from_scenario(sc) for _ in range(3)]
    srv = Server(workers=4)
    pool = srv.add_model(members[0], _abi.FORM_FAST, 1e-6)
    for m in members[1:]:
        srv.add_replica(pool, m)
    m = members[0]
    nblk = sum(m.layer_units[l] for l in range(m.n_layers) if m.layer_power[l])
    reqs, t = [], 0.0
    r2 = np.random.default_rng(94)
    for k in range(12):
        t += r2.exponential(1.0 / 5000.0)
        if k % 2:
            reqs.append(Request(pool, _abi.REQ_STEADY, m.power_vector(r2.uniform(0.5, 20.0, nblk)), t, tag="s"))
        else:
            trace = W.ar1_power(r2, r2.uniform(0.5, 20.0, nblk), 20)
            p = np.stack([m.power_vector(trace[s]) for s in range(20)])
            reqs.append(Request(pool, _abi.REQ_TRANSIENT, p, t, temp_in=m.vector(m.config.init_temp), steps=20,
                                dt=3.333e-6, tag="t"))
    alone = [Request(r.model, r.kind, r.power, 0.0, r.temp_in, r.steps, r.dt, r.tag) for r in reqs]
    for r in alone:
        srv.run([r])
    srv.run(reqs)
    for a, b in zip(alone, reqs):
        assert a.status == 0 and b.status == 0
        assert np.array_equal(a.out, b.out), (a.tag, np.max(np.abs(a.out - b.out)))
    spans = sorted((r.start, r.finish) for r in reqs)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1)), "no two requests of the pool overlapped"
    srv.close()
    for mm in members:
        mm.close()


def test_batched_transients_join_and_leave(workdir):
    """Continuous batching: transients of several classes and pool members,
    two interval lengths, arriving over time, advanced by the batch engine a
    tick at a time while steady requests run on the workers.  Each result
    equals the same request served alone (through the engine, bit for bit:
    a chip's result does not depend on its batch mates, its CTAs or its
    launch boundaries); requests shared ticks; a transient's result stays
    within 0.01 K of the oracle's FP64 replay."""
    rng = np.random.default_rng(95)
    scs = [W.scenario_random_chip(workdir, rng, "ta", side=64, chip_layers=2, steps=0),
           W.scenario_random_chip(workdir, rng, "tb", side=128, chip_layers=3, steps=0),
           W.scenario_random_chip(workdir, rng, "tc", side=32, chip_layers=5, steps=0),
           W.scenario_random_chip(workdir, rng, "sd", side=128, chip_layers=2, steps=0)]
    models = [hm.from_scenario(sc) for sc in scs]
    srv = Server(workers=3)
    idx = [srv.add_model(m, _abi.FORM_FAST, 1e-6) for m in models]
    reps = [hm.from_scenario(scs[0]) for _ in range(2)]
    for r in reps:
        srv.add_replica(idx[0], r)
    srv.set_batching(True)
    r2 = np.random.default_rng(96)
    reqs, t = [], 0.0
    for k in range(18):
        t += r2.exponential(1.0 / 3000.0)
        mi = 2 if k == 0 else int(r2.integers(0, 4))
        m = models[mi]
        nblk = sum(m.layer_units[l] for l in range(m.n_layers) if m.layer_power[l])
        if mi == 3:
            reqs.append(Request(mi, _abi.REQ_STEADY, m.power_vector(r2.uniform(0.5, 20.0, nblk)), t, tag="s"))
            continue
        steps = int(r2.integers(5, 60))
        dt = 3.333e-6 if k % 3 else 1e-5
        trace = W.ar1_power(r2, r2.uniform(0.5, 20.0, nblk), steps)
        p = np.stack([m.power_vector(trace[s]) for s in range(steps)])
        reqs.append(Request(mi, _abi.REQ_TRANSIENT, p, t, temp_in=m.vector(m.config.init_temp), steps=steps, dt=dt,
                            tag=f"t{mi}"))
    alone = [Request(r.model, r.kind, r.power, 0.0, r.temp_in, r.steps, r.dt, r.tag) for r in reqs]
    for r in alone:
        srv.run([r])
    st0 = srv.batch_stats()
    srv.run(reqs)
    st1 = srv.batch_stats()
    for a, b in zip(alone, reqs):
        assert a.status == 0 and b.status == 0
        assert np.array_equal(a.out, b.out), (a.tag, np.max(np.abs(a.out - b.out)))
        assert (b.worker == -1) == (b.kind == _abi.REQ_TRANSIENT), (b.tag, b.worker)
    ticks = st1["ticks"] - st0["ticks"]
    shared = (st1["requests_per_tick"] * st1["ticks"] - st0["requests_per_tick"] * st0["ticks"]) / ticks
    assert shared > 1.0, shared            # mean requests advanced per tick in the mixed run
    # one transient against the oracle's FP64 replay of the reference
    r = next(r for r in reqs if r.kind == _abi.REQ_TRANSIENT and r.model == 2)
    o = OracleModel(scs[2])
    to = np.array(r.temp_in, dtype=np.float64)
    for k in range(r.steps):
        o.compute_temp(r.power[k].copy(), to if k == 0 else None, r.dt)
    assert np.max(np.abs(r.out - to)) <= 0.01
    srv.close()
    for m in models + reps:
        m.close()
