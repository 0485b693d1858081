"""Serving: steady and transient requests over resident models
(libhotspot_b200's hsb_server_* entry points), and the seeded request mix
of the serving benchmark.

The loop itself is native (hotspot_b200/csrc/serve.cu): worker threads keep
several requests in flight, each on its own model's CUDA stream, admitting a
request as soon as it has arrived, its model is idle and -- on a model's
first use -- free device memory covers its solver workspace.  This module
holds the Python-side objects: a Server, the Request records, and the mix
generator (Poisson arrivals; 70% steady solves of 64..1024-cell-side chips
with 1..8 chip layers, 30% 500-interval transients of 64..256-cell-side chips).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _abi
from . import workloads as W
from ._abi import FORM_FAST, HotspotError, lib

# device memory a model's first solve allocates, per cell (fast-form
# transient work arrays and Krylov vectors, or multigrid / BiCGStab levels)
WORKSPACE_BYTES_PER_CELL = 200


def _check(rc: int):
    if rc != 0:
        raise HotspotError(lib().hsb_dev_last_error().decode(errors="replace").strip())


@dataclass
class Request:
    model: int
    kind: int                         # _abi.REQ_STEADY or _abi.REQ_TRANSIENT
    power: np.ndarray                 # (nb,) steady or (steps, nb) transient
    arrival: float
    temp_in: np.ndarray | None = None
    steps: int = 1
    dt: float = 0.0
    tag: str = ""
    out: np.ndarray | None = None
    start: float = 0.0
    finish: float = 0.0
    status: int = 0
    worker: int = 0                   # written by the server; -1: the batch engine

    @property
    def latency(self) -> float:
        return self.finish - self.arrival


class Server:
    """A set of resident models served by `workers` concurrent requests."""

    def __init__(self, workers: int = 8, reserve_bytes: int = 1 << 30):
        self.ptr = C.c_void_p()
        _check(lib().hsb_server_create(C.byref(self.ptr), int(workers), int(reserve_bytes)))
        self.models = []

    def add_model(self, model, form: int = FORM_FAST, steady_tol: float = 0.0) -> int:
        dev = lib().hsb_grid_device(model.ptr)
        idx = lib().hsb_server_add_model(self.ptr, dev, int(form), float(steady_tol),
                                         int(model.n_cells * WORKSPACE_BYTES_PER_CELL))
        if idx < 0:
            _check(idx)
        self.models.append(model)
        return idx

    def add_replica(self, model: int, replica) -> int:
        """Register ``replica`` (same grid and floorplans) as another member of
        ``model``'s pool: requests naming the pool run on whichever member is idle."""
        idx = lib().hsb_server_add_replica(self.ptr, int(model), lib().hsb_grid_device(replica.ptr))
        if idx < 0:
            _check(idx)
        self.models.append(replica)
        return idx

    def set_priority(self, model: int, high: bool = True):
        """Dispatch this model's requests first and run them on a high-priority stream."""
        _check(lib().hsb_server_set_priority(self.ptr, int(model), int(bool(high))))

    def set_batching(self, on: bool = True):
        """Serve the transients of fast-form models through the continuous batch
        engine: one launch per tick advances every admitted transient of one
        interval length; requests join and leave between ticks."""
        _check(lib().hsb_server_set_batching(self.ptr, int(bool(on))))

    def batch_stats(self) -> dict:
        """Engine counters: ticks (launches), mean requests advanced per tick,
        request-intervals advanced."""
        t, rt, ri = C.c_longlong(), C.c_longlong(), C.c_longlong()
        _check(lib().hsb_server_batch_stats(self.ptr, C.byref(t), C.byref(rt), C.byref(ri)))
        return {"ticks": t.value, "requests_per_tick": rt.value / t.value if t.value else 0.0,
                "request_intervals": ri.value}

    def run(self, requests: list[Request]):
        n = len(requests)
        arr = (_abi.Request * n)()
        keep = []
        for k, r in enumerate(requests):
            m = self.models[r.model]
            nb = m.total_n_blocks + m.n_extra
            p = np.ascontiguousarray(r.power, dtype=np.float64)
            assert p.size == nb * (r.steps if r.kind == _abi.REQ_TRANSIENT else 1)
            r.out = np.zeros(nb)
            ti = None if r.temp_in is None else np.ascontiguousarray(r.temp_in, dtype=np.float64)
            keep += [p, ti]
            a = arr[k]
            a.model, a.kind, a.steps, a.dt = r.model, r.kind, int(r.steps), float(r.dt)
            a.power = p.ctypes.data
            a.temp_in = ti.ctypes.data if ti is not None else None
            a.out = r.out.ctypes.data
            a.arrival = float(r.arrival)
        rc = lib().hsb_server_run(self.ptr, arr, n)
        for k, r in enumerate(requests):
            r.start, r.finish, r.status = arr[k].start, arr[k].finish, arr[k].status
            r.worker = arr[k].worker       # -1: served by the batch engine
        _check(rc)
        return requests

    def close(self):
        if self.ptr:
            lib().hsb_server_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# the serving mix
# ---------------------------------------------------------------------------
@dataclass
class Mix:
    requests: list
    classes: dict = field(default_factory=dict)   # (kind, side, layers) -> model (pool) index
    models: list = field(default_factory=list)
    members: dict = field(default_factory=dict)   # pool index -> number of resident models in it


def serving_mix(workdir: str, server: Server, seed: int = 0, rate: float = 2000.0, duration: float = 1.0,
                steady_frac: float = 0.7, transient_steps: int = 500, dt: float = 3.333e-6,
                steady_sides=(64, 128, 256, 512, 1024), transient_sides=(64, 128, 256),
                max_layers: int = 8, model_factory=None, high_priority_cells: int = 0,
                high_priority_classes=(), reuse: Mix | None = None, replicas: int = 1,
                replica_max_side: int = 256, probe_rate: float = 0.0, probe_class=(256, 4)) -> Mix:
    """Seeded Poisson arrivals at `rate` req/s for `duration` s.  Steady
    requests: side drawn log-uniformly from `steady_sides`, 1..max_layers
    chip layers; transients: `transient_steps` intervals of `dt` on
    `transient_sides`.  One resident model per (kind, side, layers) class,
    registered on `server`; every request carries its own power map
    (U(0.5, 20) W per block, AR(1) over a transient) and transients their
    initial block temperatures, so results do not depend on history.
    Steady classes of at most `high_priority_cells` cells, and the steady
    classes named in `high_priority_classes` as (side, chip layers), get the
    high priority class.  `reuse`: the resident models of an earlier mix on
    the same server serve the classes they cover.  `replicas`: resident
    models per class of side at most `replica_max_side` (a pool; requests of
    one class then run concurrently on its idle members).  `probe_rate`: an
    extra seeded Poisson stream of steady requests of `probe_class` (side,
    chip layers) at that rate over the same window, tagged like the class's
    own requests, so a latency percentile of that class rests on enough
    samples."""
    from . import model as hm
    rng = np.random.default_rng(seed)
    mix = Mix(requests=[])
    if reuse is not None:
        mix.classes, mix.models, mix.members = reuse.classes, reuse.models, reuse.members
    model_factory = model_factory or hm.from_scenario
    scen = {}
    # arrivals: the mix, then the probe stream, merged in time order
    arrivals = []
    t = 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        steady = rng.random() < steady_frac
        sides = steady_sides if steady else transient_sides
        side = int(sides[rng.integers(0, len(sides))])
        layers = int(rng.integers(1, max_layers + 1))
        arrivals.append((t, steady, side, layers))
    if probe_rate > 0:
        prng = np.random.default_rng([seed, 7919])
        t = 0.0
        while True:
            t += prng.exponential(1.0 / probe_rate)
            if t >= duration:
                break
            arrivals.append((t, True, int(probe_class[0]), int(probe_class[1])))
        arrivals.sort(key=lambda a: a[0])
    for t, steady, side, layers in arrivals:
        key = ("steady" if steady else "transient", side, layers)
        if key not in mix.classes:
            crng = np.random.default_rng([seed, side, layers, int(steady)])
            sc = W.scenario_random_chip(workdir, crng, f"srv_{key[0]}_{side}_{layers}", side=side,
                                        chip_layers=layers, steps=0)
            m = model_factory(sc)
            mix.models.append(m)
            scen[key] = sc
            mix.classes[key] = server.add_model(m, FORM_FAST, 1e-5)
            if steady and (m.n_cells <= high_priority_cells or (side, layers) in set(high_priority_classes)):
                server.set_priority(mix.classes[key], True)
            mix.members[mix.classes[key]] = 1
            for _ in range(replicas - 1 if side <= replica_max_side else 0):
                rep = model_factory(sc)
                mix.models.append(rep)
                server.add_replica(mix.classes[key], rep)
                mix.members[mix.classes[key]] += 1
        mi = mix.classes[key]
        m = server.models[mi]
        nblk = sum(m.layer_units[l] for l in range(m.n_layers) if m.layer_power[l])
        if steady:
            row = rng.uniform(0.5, 20.0, nblk)
            req = Request(mi, _abi.REQ_STEADY, m.power_vector(row), t, tag=f"steady_{side}_{layers}")
        else:
            means = rng.uniform(0.5, 20.0, nblk)
            trace = W.ar1_power(rng, means, transient_steps)
            p = np.stack([m.power_vector(trace[k]) for k in range(transient_steps)])
            req = Request(mi, _abi.REQ_TRANSIENT, p, t, temp_in=m.vector(m.config.init_temp),
                          steps=transient_steps, dt=dt, tag=f"transient_{side}_{layers}")
        mix.requests.append(req)
    return mix


def latency_report(requests, tag: str | None = None) -> dict:
    rs = [r for r in requests if (tag is None or r.tag == tag) and r.status == 0]
    if not rs:
        return {"n": 0}
    lat = np.array([r.latency for r in rs]) * 1e3
    return {"n": len(rs), "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()), "max_ms": float(lat.max())}
