"""Seeded synthetic inputs in HotSpot's own file formats.

The reference ships no benchmark inputs with outputs, so every workload here is
generated from a seed and written in the reference's formats, so that the
reference CLI/library and this package read byte-identical inputs:

* ``.flp``  floorplan: ``name width height leftx bottomy [cv rho]`` per line
  (reader: flp.c:1059-1120, 5 or 7 fields).
* ``.lcf``  layer configuration: 7 lines per layer, ``no lateral power sp rho
  thickness floorplan`` (reader: temperature_grid.c:612-752).
* ``.ptrace`` power trace: header of unit names, then one row of watts per
  sampling interval, tab separated (reader: hotspot.c:182-247).
* ``.csv``  microchannel network: one row per grid row of cell types
  (-1 TSV, 0 solid, 1 fluid, 2 inlet, 3 outlet; microchannel.c:258-315).

Generators (floorplan slicing, AR(1) power, Gaussian hot-spot maps) follow the
synthetic-input recipe of the benchmark configurations; they are not taken
from any external suite.
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Unit:
    name: str
    width: float
    height: float
    leftx: float
    bottomy: float
    cv: float | None = None      # volumetric specific heat (7-field lines)
    rho: float | None = None     # thermal resistivity (7-field lines)


def guillotine_floorplan(rng: np.random.Generator, width: float, height: float,
                         n_blocks: int, prefix: str = "b",
                         aspect: tuple[float, float] = (0.33, 3.0),
                         frac: tuple[float, float] = (0.3, 0.7)) -> list[Unit]:
    """Seeded guillotine slicing of a ``width`` x ``height`` die.

    Repeatedly takes the largest-area leaf and cuts it across its longer side
    at a uniform fraction in ``frac``; fractions that would make a child's
    aspect ratio leave ``aspect`` are redrawn.  Returns ``n_blocks`` units that
    tile the die exactly (no overlap, no dead space).
    """
    leaves = [(0.0, 0.0, float(width), float(height))]
    lo, hi = aspect
    while len(leaves) < n_blocks:
        k = max(range(len(leaves)), key=lambda t: leaves[t][2] * leaves[t][3])
        x, y, w, h = leaves.pop(k)
        vertical = w >= h
        for _ in range(1000):
            f = rng.uniform(*frac)
            if vertical:
                a, b = (x, y, w * f, h), (x + w * f, y, w * (1 - f), h)
            else:
                a, b = (x, y, w, h * f), (x, y + h * f, w, h * (1 - f))
            if all(lo <= c[2] / c[3] <= hi for c in (a, b)):
                break
        else:  # pragma: no cover - aspect window always admits f = 0.5
            f = 0.5
            if vertical:
                a, b = (x, y, w * f, h), (x + w * f, y, w * (1 - f), h)
            else:
                a, b = (x, y, w, h * f), (x, y + h * f, w, h * (1 - f))
        leaves.extend([a, b])
    leaves.sort(key=lambda c: (-(c[1] + c[3]), c[0]))
    return [Unit(f"{prefix}{i}", c[2], c[3], c[0], c[1]) for i, c in enumerate(leaves)]


def uniform_tiling(width: float, height: float, nx: int, ny: int,
                   prefix: str = "t") -> list[Unit]:
    """``nx`` x ``ny`` equal rectangles covering the die (row-major from the top)."""
    w, h = width / nx, height / ny
    units = []
    for r in range(ny):
        for c in range(nx):
            units.append(Unit(f"{prefix}_{r}_{c}", w, h, c * w, height - (r + 1) * h))
    return units


def write_flp(path: str, units: list[Unit]) -> str:
    with open(path, "w") as f:
        f.write("# name\twidth\theight\tleftx\tbottomy\n")
        for u in units:
            if u.cv is None:
                f.write(f"{u.name}\t{u.width!r}\t{u.height!r}\t{u.leftx!r}\t{u.bottomy!r}\n")
            else:
                f.write(f"{u.name}\t{u.width!r}\t{u.height!r}\t{u.leftx!r}\t{u.bottomy!r}"
                        f"\t{u.cv!r}\t{u.rho!r}\n")
    return path


@dataclass
class Layer:
    lateral: bool
    power: bool
    sp: float | str          # specific heat, or a material name
    rho: float | None        # resistivity (None when sp is a material name)
    thickness: float
    flp: str


def write_lcf(path: str, layers: list[Layer]) -> str:
    with open(path, "w") as f:
        for i, L in enumerate(layers):
            f.write(f"# layer {i}\n{i}\n{'Y' if L.lateral else 'N'}\n{'Y' if L.power else 'N'}\n")
            if isinstance(L.sp, str):
                f.write(f"{L.sp}\n")
            else:
                f.write(f"{L.sp!r}\n{L.rho!r}\n")
            f.write(f"{L.thickness!r}\n{L.flp}\n\n")
    return path


def ar1_power(rng: np.random.Generator, means: np.ndarray, steps: int,
              rho: float = 0.9, rel_sigma: float = 0.1) -> np.ndarray:
    """``steps`` x ``len(means)`` power rows: mean + AR(1) fluctuation, clamped >= 0.

    x_t = rho x_{t-1} + e_t with e_t ~ N(0, (rel_sigma*mean)^2 (1 - rho^2)),
    so the stationary standard deviation is rel_sigma*mean.
    """
    means = np.asarray(means, dtype=np.float64)
    sig = rel_sigma * means * math.sqrt(1.0 - rho * rho)
    out = np.empty((steps, means.size))
    x = rng.normal(0.0, rel_sigma * means)
    for t in range(steps):
        x = rho * x + rng.normal(0.0, sig)
        out[t] = np.maximum(means + x, 0.0)
    return out


def write_ptrace(path: str, names: list[str], rows: np.ndarray) -> str:
    with open(path, "w") as f:
        f.write("\t".join(names) + "\n")
        for r in rows:
            f.write("\t".join(f"{v:.10g}" for v in r) + "\n")
    return path


def straight_channels_csv(path: str, nr: int, nc: int, cell_w: float,
                          channel_w: float, pitch: float) -> tuple[str, int]:
    """North-to-south straight channels: inlet row 0, outlet row nr-1.

    A column is fluid when its centre lies inside a channel of width
    ``channel_w`` repeated every ``pitch`` (all in metres).  Returns the path
    and the number of channel lanes.
    """
    types = np.zeros((nr, nc), dtype=np.int32)
    cols = []
    for j in range(nc):
        xc = (j + 0.5) * cell_w
        off = math.fmod(xc, pitch)
        if off < channel_w:
            cols.append(j)
    cols = np.array(cols, dtype=np.int64)
    types[:, cols] = 1
    types[0, cols] = 2
    types[nr - 1, cols] = 3
    lanes = int(np.sum(np.diff(cols) != 1) + 1) if cols.size else 0
    with open(path, "w") as f:
        for i in range(nr):
            f.write(",".join(str(int(v)) for v in types[i]) + "\n")
    return path, lanes


def gaussian_hotspot_map(rng: np.random.Generator, units: list[Unit], width: float,
                         height: float, n_blobs: int = 6, peak=(1.0, 5.0),
                         background: float = 0.2, sigma=(0.3e-3, 1.0e-3),
                         sub: int = 4) -> np.ndarray:
    """Block powers (W) integrating a W/mm^2 density of Gaussian blobs over a background."""
    cx = rng.uniform(0, width, n_blobs)
    cy = rng.uniform(0, height, n_blobs)
    pk = rng.uniform(*peak, n_blobs)
    sg = rng.uniform(*sigma, n_blobs)
    out = np.empty(len(units))
    for k, u in enumerate(units):
        xs = u.leftx + (np.arange(sub) + 0.5) * u.width / sub
        ys = u.bottomy + (np.arange(sub) + 0.5) * u.height / sub
        X, Y = np.meshgrid(xs, ys)
        dens = np.full_like(X, background)
        for b in range(n_blobs):
            dens += pk[b] * np.exp(-((X - cx[b]) ** 2 + (Y - cy[b]) ** 2) / (2 * sg[b] ** 2))
        out[k] = dens.mean() * (u.width * u.height * 1e6)
    return out


# ---------------------------------------------------------------------------
# The benchmark configurations (sizes and distributions as specified for the
# grid-model benchmark; inputs are synthetic and seeded).
# ---------------------------------------------------------------------------

@dataclass
class Scenario:
    """Everything needed to build one model and drive it."""
    name: str
    config: dict = field(default_factory=dict)   # thermal_config name -> value string
    flp: str | None = None                         # default-layer floorplan
    lcf: str | None = None
    detailed_3D: bool = False
    use_microchannels: bool = False
    materials: str | None = None
    power_layers: list = field(default_factory=list)  # per layer: list of unit names (power layers)
    block_power: np.ndarray | None = None          # (steps, n_power_blocks) in trace order
    steps: int = 0
    dt: float = 0.0


def scenario_chip2d(workdir: str, seed: int = 0, grid: int = 64, steps: int = 1000,
                    n_blocks: int = 15, die: float = 16e-3) -> Scenario:
    """Single-layer 2-D chip on the default package (16x16 mm, 0.15 mm Si, 64x64)."""
    rng = np.random.default_rng(seed)
    units = guillotine_floorplan(rng, die, die, n_blocks)
    flp = write_flp(os.path.join(workdir, f"chip2d_s{seed}.flp"), units)
    means = rng.uniform(0.5, 20.0, len(units))
    trace = ar1_power(rng, means, steps)
    cfg = {"model_type": "grid", "grid_rows": str(grid), "grid_cols": str(grid),
           "sampling_intvl": "3.333e-06"}
    return Scenario("chip2d", cfg, flp=flp, power_layers=[[u.name for u in units]],
                    block_power=trace, steps=steps, dt=3.333e-6)


def scenario_stack3d(workdir: str, seed: int = 0, grid: int = 256, steps: int = 10000,
                     n_blocks: int = 40, die: float = 20e-3) -> Scenario:
    """4-layer 3-D stack: Si 0.1 mm / TIM 20 um / Si 0.1 mm / TIM 20 um over 20x20 mm."""
    rng = np.random.default_rng(seed)
    si_a = guillotine_floorplan(rng, die, die, n_blocks, prefix="a")
    si_b = guillotine_floorplan(rng, die, die, n_blocks, prefix="c")
    tim = [Unit("tim", die, die, 0.0, 0.0)]
    fa = write_flp(os.path.join(workdir, f"stack_s{seed}_si0.flp"), si_a)
    fb = write_flp(os.path.join(workdir, f"stack_s{seed}_si1.flp"), si_b)
    ft = write_flp(os.path.join(workdir, f"stack_s{seed}_tim.flp"), tim)
    layers = [Layer(True, True, 1.75e6, 0.01, 1e-4, fa),
              Layer(True, False, 4e6, 0.25, 2e-5, ft),
              Layer(True, True, 1.75e6, 0.01, 1e-4, fb),
              Layer(True, False, 4e6, 0.25, 2e-5, ft)]
    lcf = write_lcf(os.path.join(workdir, f"stack_s{seed}.lcf"), layers)
    means = []
    for us in (si_a, si_b):
        dens = rng.uniform(0.1, 2.0, len(us))            # W/mm^2
        means.append(dens * np.array([u.width * u.height * 1e6 for u in us]))
    means = np.concatenate(means)
    trace = ar1_power(rng, means, steps)
    cfg = {"model_type": "grid", "grid_rows": str(grid), "grid_cols": str(grid),
           "grid_layer_file": lcf, "sampling_intvl": "1e-05"}
    return Scenario("stack3d", cfg, lcf=lcf,
                    power_layers=[[u.name for u in si_a], [], [u.name for u in si_b], []],
                    block_power=trace, steps=steps, dt=1e-5)


def scenario_random_chip(workdir: str, rng: np.random.Generator, tag: str,
                         side: int | None = None, chip_layers: int | None = None,
                         steps: int = 2000, die: float = 16e-3) -> Scenario:
    """One chip of the batched mix: side 2^k (k in 5..9), 1..8 chip layers
    alternating Si/TIM (top is Si, power on Si layers), 10..100 blocks."""
    if side is None:
        side = int(2 ** rng.integers(5, 10))
    if chip_layers is None:
        chip_layers = int(rng.integers(1, 9))
    nb = int(rng.integers(10, 101))
    layers, power_layers, means = [], [], []
    tim = write_flp(os.path.join(workdir, f"{tag}_tim.flp"), [Unit("tim", die, die, 0.0, 0.0)])
    for l in range(chip_layers):
        if l % 2 == 0:
            us = guillotine_floorplan(rng, die, die, nb, prefix=f"l{l}_")
            f = write_flp(os.path.join(workdir, f"{tag}_l{l}.flp"), us)
            layers.append(Layer(True, True, 1.75e6, 0.01, 1e-4, f))
            power_layers.append([u.name for u in us])
            means.append(rng.uniform(0.5, 20.0, len(us)))
        else:
            layers.append(Layer(True, False, 4e6, 0.25, 2e-5, tim))
            power_layers.append([])
    lcf = write_lcf(os.path.join(workdir, f"{tag}.lcf"), layers)
    trace = ar1_power(rng, np.concatenate(means), steps) if steps else None
    cfg = {"model_type": "grid", "grid_rows": str(side), "grid_cols": str(side),
           "grid_layer_file": lcf, "sampling_intvl": "3.333e-06"}
    return Scenario(f"chip_{tag}", cfg, lcf=lcf, power_layers=power_layers,
                    block_power=trace, steps=steps, dt=3.333e-6)


WATER_MATERIALS = """\
# name type k volumetric_heat_capacity viscosity
water
fluid
0.6069
4172638
0.000889

silicon
solid
130
1635660
"""


def write_materials(path: str) -> str:
    with open(path, "w") as f:
        f.write(WATER_MATERIALS)
    return path


def scenario_microchannel(workdir: str, seed: int = 0, grid: int = 512,
                          die: float = 10.24e-3, channel_w: float = 100e-6,
                          channel_h: float = 200e-6, pitch: float = 200e-6,
                          blocks: int = 64) -> Scenario:
    """Si (0.1 mm, power) over a 0.2 mm straight-channel water layer.

    The default die is 10.24 mm, i.e. 20 um cells at 512x512: the channel
    layer's floorplan is generated from the CSV with printf("%e") positions
    (7 significant digits, microchannel.c), so cell sizes whose multiples
    need more digits (10 mm / 512 = 19.53125 um) make the generated units
    overrun the grid and the reference's own set_bgmap rejects them.
    """
    rng = np.random.default_rng(seed)
    cw = die / grid
    csv, lanes = straight_channels_csv(os.path.join(workdir, f"uchan_s{seed}.csv"),
                                       grid, grid, cw, channel_w, pitch)
    units = uniform_tiling(die, die, blocks, blocks, prefix="p")
    fsi = write_flp(os.path.join(workdir, f"uchan_s{seed}_si.flp"), units)
    mats = write_materials(os.path.join(workdir, "uchan.materials"))
    layers = [Layer(True, True, 1.75e6, 0.01, 1e-4, fsi),
              Layer(True, False, 1.75e6, 0.01, channel_h, csv)]
    lcf = write_lcf(os.path.join(workdir, f"uchan_s{seed}.lcf"), layers)
    # flow rate per channel (mL/min) -> ideal pump pressure across rows-1 links
    q_ml_min = rng.uniform(1.0, 10.0)
    q = q_ml_min * 1e-6 / 60.0                      # m^3/s per channel
    width_cells = max(1, int(round(channel_w / cw)))
    h, w, L = channel_h, cw, cw
    mu = 0.000889
    if h == w:
        hc = 0.42229 * h ** 4 / (12 * mu * L)
    elif h > w:
        hc = (1 - 0.63 * (w / h)) * w ** 3 * h / (12 * mu * L)
    else:
        hc = (1 - 0.63 * (h / w)) * h ** 3 * w / (12 * mu * L)
    dp = q * (grid - 1) / (width_cells * hc)
    power = gaussian_hotspot_map(rng, units, die, die)
    cfg = {"model_type": "grid", "grid_rows": str(grid), "grid_cols": str(grid),
           "grid_layer_file": lcf, "pumping_pressure": repr(dp),
           "inlet_temperature": "300", "coolant_material": "water",
           "grid_map_mode": "avg"}
    sc = Scenario("microchannel", cfg, lcf=lcf, detailed_3D=True, use_microchannels=True,
                  materials=mats, power_layers=[[u.name for u in units], []],
                  block_power=power[None, :], steps=1, dt=0.0)
    sc.lanes = lanes
    sc.flow_ml_min = q_ml_min
    return sc
