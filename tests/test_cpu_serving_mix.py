"""The serving benchmark's request mix (hotspot_b200.serving.serving_mix),
host logic only: seeded Poisson arrivals, the 70/30 steady/transient split,
side and layer draws, one resident model per class, and the priority class.
Models and the server are stand-ins here; the GPU tests run the real ones."""
import numpy as np

from hotspot_b200 import _abi
from hotspot_b200.serving import serving_mix


class FakeModel:
    def __init__(self, sc):
        side = int(sc.config["grid_rows"])
        chip = len(sc.power_layers)
        self.n_layers = chip + 2
        self.n_cells = side * side * self.n_layers
        self.layer_power = [bool(p) for p in sc.power_layers] + [False, False]
        self.layer_units = [max(len(p), 1) for p in sc.power_layers] + [1, 1]
        self.config = type("Cfg", (), {"init_temp": 333.15})()
        self.side, self.chip_layers = side, chip

    def power_vector(self, row):
        return np.asarray(row, dtype=np.float64)

    def vector(self, fill=0.0):
        return np.full(1, fill)


class FakeServer:
    def __init__(self):
        self.models, self.high = [], set()

    def add_model(self, m, form, tol):
        self.models.append(m)
        return len(self.models) - 1

    def set_priority(self, idx, high=True):
        self.high.add(idx)


def _mix(workdir, seed, **kw):
    srv = FakeServer()
    mix = serving_mix(workdir, srv, seed=seed, rate=2000.0, duration=0.25, transient_steps=20,
                      model_factory=FakeModel, **kw)
    return srv, mix


def test_seeded_and_poisson(workdir):
    srv, mix = _mix(workdir, 4)
    _, again = _mix(workdir, 4)
    t = np.array([r.arrival for r in mix.requests])
    assert [(r.arrival, r.kind, r.tag) for r in mix.requests] == [(r.arrival, r.kind, r.tag) for r in again.requests]
    assert np.all(np.diff(t) > 0) and t[-1] < 0.25
    assert 0.8 * 500 < len(t) < 1.2 * 500            # 2000 req/s over 0.25 s
    steady = np.mean([r.kind == _abi.REQ_STEADY for r in mix.requests])
    assert abs(steady - 0.7) < 0.07


def test_classes_and_requests(workdir):
    srv, mix = _mix(workdir, 5)
    for (kind, side, layers), idx in mix.classes.items():
        m = srv.models[idx]
        assert m.side == side and m.chip_layers == layers and 1 <= layers <= 8
        assert side in ((64, 128, 256, 512, 1024) if kind == "steady" else (64, 128, 256))
    assert len(srv.models) == len(mix.classes)        # one resident model per class
    for r in mix.requests:
        m = srv.models[r.model]
        nblk = sum(m.layer_units[l] for l in range(m.n_layers) if m.layer_power[l])
        if r.kind == _abi.REQ_STEADY:
            assert r.power.shape == (nblk,) and np.all((r.power >= 0.5) & (r.power <= 20.0))
        else:
            assert r.steps == 20 and r.power.shape == (20, nblk) and np.all(r.power >= 0.0)
            assert r.temp_in is not None and r.dt > 0


def test_priority_class(workdir):
    srv, mix = _mix(workdir, 6, high_priority_classes=[(256, 4)])
    want = {idx for (kind, side, layers), idx in mix.classes.items() if (kind, side, layers) == ("steady", 256, 4)}
    assert want and srv.high == want
    srv, mix = _mix(workdir, 6, high_priority_cells=128 * 128 * 10)
    for (kind, side, layers), idx in mix.classes.items():
        assert (idx in srv.high) == (kind == "steady" and side * side * (layers + 2) <= 128 * 128 * 10)
