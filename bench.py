#!/usr/bin/env python
"""Benchmark of the grid thermal model on B200.

Workload: the 3-D stacked IC -- Si 0.1 mm / TIM 20 um / Si 0.1 mm / TIM 20 um
plus spreader and sink, 256x256 cells over 20x20 mm (393,216 cells), a
seeded 40-block floorplan per silicon layer with 0.1-2 W/mm^2, power rows at
10 us.  One bench step = one sampling interval of the transient trace
(compute_temp with the next power row: every adaptive RK4 step it takes).

  value      cell-steps/s of the fast form (FP32 stencil, FP64 state), whole
             job over all ranks, state resident in HBM, device time (CUDA
             events on the library's stream), L2 flushed between steps
  e2e        the same metric through the C-ABI call compute_temp_grid with
             host power/temperature buffers (copies inside), wall clock
  steady     steady solves/s: fast form (FP32 MG-PCG + FP64 refinement) and
             the plain FP64 form (exact replay of the reference's solver)
  accuracy   max |dT| of the fast form against the plain FP64 form

Further legs on one GPU (skipped under torchrun and with --headline-only):
  batched       512 synthetic chips of uneven size (sides 32..512, 1..8 chip
                layers) advanced together, one persistent launch per interval
                (autotuned schedule), cell-steps/s and its HBM roofline
  microchannel  512x512 Si + water-channel stack, non-symmetric steady system
                by FP32 BiCGStab + FP64 refinement, solves/s and residual
  serving       the seeded request mix (Poisson arrivals at 2000 req/s, 70%
                steady 64..1024 sides, 30% 500-interval transients), latency
                percentiles and throughput of the serving loop

Multi-GPU: independent replicas (one chip per rank, weak scaling); the
timed region is bracketed by barriers and the max over ranks is reported.

--impl reference times the reference's own C implementation (oracle/_ref,
compiled from the HotSpot sources) on the same workload on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "cell-steps/s"
ALG_BYTES_FP32 = 108   # per cell-step: 22 FP32 stage fields + FP64 state r/w + FP32 power
ALG_BYTES_FP64 = 200   # per cell-step, all FP64


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=256)
    ap.add_argument("--no-plain", action="store_true", help="skip the plain FP64 comparison legs")
    ap.add_argument("--profile", action="store_true",
                    help="transient intervals of the fast form only (the case profiled with ncu)")
    ap.add_argument("--headline-only", action="store_true", help="skip the batched / microchannel / serving legs")
    ap.add_argument("--legs", default="chip2d,batched,microchannel,serving",
                    help="comma-separated legs to run after the headline")
    ap.add_argument("--serving-batching", type=int, default=1,
                    help="serve transients through the continuous batch engine (1) or the workers (0)")
    ap.add_argument("--profile-case", choices=["batch", "microchannel", "steady"], default=None,
                    help="small cases of the other kernels, for ncu captures (a few GB at most)")
    ap.add_argument("--chip2d-rows", type=int, default=1000, help="rows of the 2-D chip leg's trace")
    ap.add_argument("--batch-chips", type=int, default=512)
    ap.add_argument("--batch-intervals", type=int, default=200)
    ap.add_argument("--serving-seconds", type=float, default=1.0,
                    help="length of the request arrival window of the serving leg at 2000 req/s")
    ap.add_argument("--serving-probe-rate", type=float, default=220.0,
                    help="rate of the SLO-class probe stream added to the 2000 req/s mix")
    ap.add_argument("--serving-replicas", type=int, default=3,
                    help="resident models per serving class of side <= 256")
    ap.add_argument("--serving-calm-rate", type=float, default=30.0,
                    help="offered rate of the serving leg's second, sustainable run")
    ap.add_argument("--serving-calm-seconds", type=float, default=4.0)
    return ap.parse_args()


def dist():
    from hotspot_b200 import replicas
    return replicas.world()


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [l.split(",") for l in open(self.f.name).read().strip().splitlines() if l.strip()]
        os.unlink(self.f.name)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if "Active" in r[5 + k] and "Not" not in r[5 + k]:
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic(name: str, key: str = "dram_bytes_per_launch"):
    """A figure (DRAM bytes per launch, or per cell-step) from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.strip().startswith(key + ":"):
                return float(line.split(":")[1].split()[0])
    except OSError:
        pass
    return None


def cpu_reference_sample(grid: int, intervals: int, seed: int):
    """Reference C code (oracle/_ref) on `intervals` rows of the workload:
    returns (cell-steps, seconds, kind)."""
    from hotspot_b200 import workloads as W
    from oracle import ref as R
    with tempfile.TemporaryDirectory() as d:
        sc = W.scenario_stack3d(d, seed=seed, grid=grid, steps=intervals + 1)
        if R.available():
            m, kind = R.RefModel(sc), "reference"
        else:
            from oracle.restatement import OracleModel
            m, kind = OracleModel(sc), "port"
        t = m.vector(333.15)
        p = m.power_vector(sc.block_power[0])
        m.compute_temp(p, t, sc.dt)
        cells = m.nl * m.nr * m.nc if hasattr(m, "nr") else m.n_cells
        t0 = time.perf_counter()
        steps = 0
        for k in range(1, intervals + 1):
            p = m.power_vector(sc.block_power[k])
            r = m.compute_temp(p, None, sc.dt)
            steps += r if isinstance(r, (int, np.integer)) else 0
        el = time.perf_counter() - t0
        if kind == "reference":
            # the reference reports no step count: replay its step rule on the port
            from oracle.restatement import OracleModel
            o = OracleModel(sc)
            to = o.vector(333.15)
            o.compute_temp(o.power_vector(sc.block_power[0]), to, sc.dt)
            steps = sum(int(o.compute_temp(o.power_vector(sc.block_power[k]), None, sc.dt))
                        for k in range(1, intervals + 1))
            m.close()
        return cells * steps, el, kind


def _cpu_worker(args):
    grid, intervals, seed = args
    cs, el, kind = cpu_reference_sample(grid, intervals, seed)
    return cs, el, kind


def cpu_throughput(grid: int, intervals: int, procs: int):
    """Independent single-threaded reference replicas on `procs` host cores."""
    import multiprocessing as mp
    if procs <= 1:
        cs, el, kind = cpu_reference_sample(grid, intervals, 0)
        return cs / el, 1, kind, cs, el
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        res = pool.map(_cpu_worker, [(grid, intervals, s) for s in range(procs)])
    rate = sum(cs / el for cs, el, _ in res)
    return rate, procs, res[0][2], sum(r[0] for r in res), max(r[1] for r in res)


def headline_config(grid, cells, ws):
    """The headline workload, named the same way by both arms."""
    return {"workload": f"3-D stack 4 chip layers + spreader/sink, {grid}x{grid} over 20x20 mm, "
                        "40 blocks per Si layer, 10 us rows",
            "cells_per_rank": cells, "l2": "256 MB buffer rewritten between timed steps (GPU arm)",
            "parallelism": f"replicas x{ws}"}


def run_reference(args):
    ws, rank, _ = dist()
    if rank != 0:
        return
    procs = max(1, min(os.cpu_count() or 1, 16))
    # one bench step = one sampling interval; a bounded sample per step
    intervals = max(1, min(args.steps, 3))
    rate, cores, kind, cs, el = cpu_throughput(args.grid, intervals, procs)
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "cell-steps/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": headline_config(args.grid, 6 * args.grid * args.grid, ws),
            "cpu_baseline": {"value": rate, "unit": "cell-steps/s", "cores": cores, "kind": kind,
                             "sample": f"{intervals} rows x {cores} independent single-threaded replicas"},
            "e2e": {"value": rate, "unit": "cell-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# further legs (one GPU)
# ---------------------------------------------------------------------------
def cpu_batch_sample(scs, idx, dt):
    """The reference's C code (oracle/_ref, else the oracle's restatement) on
    one interval of each sampled chip, single-threaded: {chip: cell-steps/s}."""
    from oracle import ref as R
    from oracle.restatement import OracleModel
    rates, kind = {}, "reference" if R.available() else "port"
    for c in idx:
        sc = scs[c]
        o = R.RefModel(sc) if R.available() else OracleModel(sc)
        to = o.vector(333.15)
        o.compute_temp(o.power_vector(sc.block_power[0]), to, 0.0)
        t0 = time.perf_counter()
        o.compute_temp(o.power_vector(sc.block_power[1]), None, dt)
        el = time.perf_counter() - t0
        # the step count: the oracle replays the reference's step rule exactly
        q = OracleModel(sc)
        tq = q.vector(333.15)
        q.compute_temp(q.power_vector(sc.block_power[0]), tq, 0.0)
        steps = int(q.compute_temp(q.power_vector(sc.block_power[1]), None, dt))
        rates[c] = q.n_cells * steps / el
        if hasattr(o, "close"):
            o.close()
    return rates, kind


def leg_batched(args, flush):
    """512 synthetic chips advanced together: K intervals per persistent launch
    of the temporally blocked kernel (hsb_batch_transient_trace)."""
    import torch
    from hotspot_b200 import FORM_FAST
    from hotspot_b200 import model as hm
    from hotspot_b200 import workloads as W
    from hotspot_b200.batch import Batch
    K = args.batch_intervals
    rng = np.random.default_rng(2024)
    d = tempfile.mkdtemp(prefix="hsb_batch_")
    t0 = time.perf_counter()
    tune_rows = 9
    scs = [W.scenario_random_chip(d, rng, f"c{i}", steps=K + tune_rows + 2) for i in range(args.batch_chips)]
    models = []
    for sc in scs:
        m = hm.from_scenario(sc)
        m.set_solver(FORM_FAST)
        t = m.vector(m.config.init_temp)
        m.compute_temp(m.power_vector(sc.block_power[0]), t, 0.0)
        models.append(m)
    cells = np.array([m.n_cells for m in models], dtype=np.float64)
    bt = Batch(models)
    setup_s = time.perf_counter() - t0
    dt = scs[0].dt

    def pw(k):
        return [m.power_vector(sc.block_power[k]) for sc, m in zip(scs, models)]
    bt.autotune(True)
    k = 1
    for _ in range(len(bt.tuning())):      # the autotuner tries one candidate schedule per call
        bt.transient(pw(k), dt)
        k += 1
    tuned = dict(bt.info(), candidates=bt.tuning())
    rows = [pw(k + j) for j in range(K)]
    flush.fill_(2.0)
    torch.cuda.synchronize()
    st = bt.trace(rows, dt)
    chip_steps = bt.chip_steps()
    kms = st["kernel_ms"]
    cs = float(np.sum(chip_steps * cells))
    rate = cs / (kms / 1e3)
    peak, peak_kind = measured_peak()
    achieved = ALG_BYTES_FP32 * rate / 1e9
    tiles = {}
    for c, m in enumerate(models):
        tiles.setdefault(f"{m.rows}x{m.cols}", bt.tile(c))
    bt.close()
    # CPU baseline: 8 chips stratified by grid side, one interval each on the
    # reference's code, extrapolated to the batch by the drawn size mix
    sides = [m.rows for m in models]
    sample = []
    for side in (512, 256, 128, 64, 32, 512, 256, 128):
        cand = [c for c, s_ in enumerate(sides) if s_ == side and c not in sample]
        if cand:
            sample.append(cand[0])
    rates, kind = cpu_batch_sample(scs, sample, dt)
    by_side = {}
    for c, r in rates.items():
        by_side.setdefault(sides[c], []).append(r)
    side_rate = {s_: float(np.mean(v)) for s_, v in by_side.items()}
    cpu_time = sum(cells[c] * chip_steps[c] / side_rate.get(sides[c], min(side_rate.values()))
                   for c in range(len(models)))
    cpu_rate = cs / cpu_time
    # each chip's steady solve: all 512 at once through the serving loop, 32 in flight
    from hotspot_b200.serving import Request, Server
    from hotspot_b200 import _abi
    srv = Server(workers=32)
    for mm in models:
        srv.add_model(mm, FORM_FAST, 1e-5)
    sreq = [Request(i, _abi.REQ_STEADY, mm.power_vector(sc.block_power[:k].mean(0)), 0.0, tag="steady")
            for i, (sc, mm) in enumerate(zip(scs, models))]
    srv.run([Request(r.model, r.kind, r.power, 0.0) for r in sreq])   # workspaces, graphs
    srv.run(sreq)
    steady_span = max(r.finish for r in sreq)
    srv.close()
    for m in models:
        m.close()
    return {"workload": f"{args.batch_chips} chips, sides 2^5..2^9, 1..8 chip layers + spreader/sink, "
                        "10..100 blocks, 3.333 us intervals", "cells": int(cells.sum()),
            "cell_steps_per_s": rate, "intervals": K, "launches_timed": st["launches"],
            "ms_per_interval": kms / K, "rk4_steps": int(chip_steps.sum()),
            "steady_solves_per_s": len(sreq) / steady_span,
            "steady_note": "every chip's steady solve (MG-PCG, FP64 refinement to 1e-5 K), all submitted at once to "
                           "the serving loop, 32 in flight on their own streams",
            "schedule": tuned, "tiles_by_grid": tiles, "setup_s": setup_s,
            "cpu_baseline": {"kind": kind, "cores": 1, "cell_steps_per_s": cpu_rate,
                             "sample": f"{len(sample)} chips stratified by side, one interval each, "
                                       "extrapolated to the batch's size mix and step counts",
                             "rates_by_side": side_rate},
            "roofline": {"bound": "hbm", "kernel": "rk4_tb_kernel", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": (lambda b: b * cs if b else None)(
                             profiled_traffic("rk4_tb_kernel_batch.md", "dram_bytes_per_cell_step")),
                         "note": "108 B per cell-step algorithmic (FP32 stages, FP64 state); the temporally "
                                 "blocked kernel moves far fewer bytes (traffic: DRAM bytes per cell-step of the "
                                 "profiled 16-chip batch x this launch's cell-steps)"},
            "l2": f"one launch of {K} intervals; the {int(cells.sum())}-cell state (FP64) is far larger than L2"}


def leg_chip2d(args, flush):
    """The 2-D chip (64x64, default package, 15 blocks): its 1000-row trace at
    3.333 us plus the steady solve of the average power, in the plain FP64
    form and the fast form, with the reference's own C code timed on the
    host on the same rows (single-threaded, as the reference runs)."""
    import torch
    from hotspot_b200 import FORM_FAST, FORM_PARITY
    from hotspot_b200 import model as hm
    from hotspot_b200 import workloads as W
    rows = args.chip2d_rows
    d = tempfile.mkdtemp(prefix="hsb_c0_")
    sc = W.scenario_chip2d(d, seed=0, grid=64, steps=rows)
    out = {"workload": "2-D chip 64x64 (Si 0.15 mm + TIM + spreader/sink), 16x16 mm, 15 blocks, "
                       f"{rows} rows at 3.333 us, then the steady solve of the average power"}
    temps = {}
    for name, form in (("plain_fp64", FORM_PARITY), ("fast", FORM_FAST)):
        m = hm.from_scenario(sc)
        m.set_solver(form)
        t = m.vector(m.config.init_temp)
        m.compute_temp(m.power_vector(sc.block_power[0]), t, 0.0)     # state and workspaces set up
        flush.fill_(1.0)
        torch.cuda.synchronize()
        dev_ms = ker_ms = 0.0
        steps = launches = 0
        tr = np.empty((rows, t.size))
        for k in range(rows):
            m.compute_temp(m.power_vector(sc.block_power[k]), None, sc.dt)
            s = m.stats()
            dev_ms += s["device_ms"]
            ker_ms += s["kernel_ms"]
            steps += s["rk4_steps"]
            launches += s["launches"]
            tr[k] = t
        avg = m.power_vector(sc.block_power.mean(0))
        sv = m.vector()
        m.steady(avg.copy(), sv)
        sms = []
        for _ in range(3 if form == FORM_FAST else 1):
            m.steady(avg.copy(), sv)
            sms.append(m.stats()["device_ms"])
        temps[name] = (tr, sv.copy())
        cells = m.n_cells
        out[name] = {"cell_steps_per_s": m.n_cells * steps / (dev_ms / 1e3), "ms_per_row": dev_ms / rows,
                     "rk4_steps": steps, "gpu_launches": launches, "steady_ms": statistics.median(sms),
                     "steady_solves_per_s": 1e3 / statistics.median(sms)}
        m.close()
    out["max_dT_K_fast_vs_plain"] = float(np.max(np.abs(temps["fast"][0] - temps["plain_fp64"][0])))
    # the reference's own code on the same rows (the live build, else the oracle's C restatement)
    from oracle import ref as R
    if R.available():
        o, kind = R.RefModel(sc), "reference"
    else:
        from oracle.restatement import OracleModel
        o, kind = OracleModel(sc), "port"
    to = o.vector(333.15)
    o.compute_temp(o.power_vector(sc.block_power[0]), to, 0.0)
    t0 = time.perf_counter()
    worst = 0.0
    for k in range(rows):
        o.compute_temp(o.power_vector(sc.block_power[k]), None, sc.dt)
        worst = max(worst, float(np.max(np.abs(to - temps["plain_fp64"][0][k]))))
    cpu_tr = time.perf_counter() - t0
    so = o.vector()
    t0 = time.perf_counter()
    o.steady(o.power_vector(sc.block_power.mean(0)), so)
    cpu_st = time.perf_counter() - t0
    if hasattr(o, "close"):
        o.close()
    steps = out["plain_fp64"]["rk4_steps"]      # the reference takes the replay's steps (bit-identical)
    out["max_dT_K_plain_vs_reference"] = worst
    out["max_dT_K_steady_plain_vs_reference"] = float(np.max(np.abs(so - temps["plain_fp64"][1])))
    out["cpu_baseline"] = {"kind": kind, "cores": 1, "cell_steps_per_s": cells * steps / cpu_tr,
                           "trace_s": cpu_tr, "steady_s": cpu_st, "steady_solves_per_s": 1.0 / cpu_st,
                           "sample": f"the full {rows} rows and the steady solve, single-threaded"}
    out["speedup_vs_cpu"] = {"fast_transient": out["fast"]["cell_steps_per_s"] / out["cpu_baseline"]["cell_steps_per_s"],
                             "plain_transient": out["plain_fp64"]["cell_steps_per_s"] /
                             out["cpu_baseline"]["cell_steps_per_s"],
                             "fast_steady": cpu_st * 1e3 / out["fast"]["steady_ms"]}
    out["note"] = ("16,384 cells fit L2: every form is latency- and launch-bound here (a few hundred "
                   "microseconds of work per row); no HBM roofline is claimed")
    return out


def leg_microchannel(args):
    """512x512 microchannel steady state by BiCGStab, and the CPU direct solve on 128x128."""
    from hotspot_b200 import FORM_FAST, STEADY_BICGSTAB
    from hotspot_b200 import model as hm
    from hotspot_b200 import workloads as W
    d = tempfile.mkdtemp(prefix="hsb_uchan_")
    out = {}
    for grid in (512, 128):
        kw = {} if grid == 512 else {"die": grid * 20e-6, "blocks": 8}
        sc = W.scenario_microchannel(d, seed=3, grid=grid, **kw)
        m = hm.from_scenario(sc)
        m.set_solver(FORM_FAST, STEADY_BICGSTAB)
        p = m.power_vector(sc.block_power[0])
        s = m.vector()
        m.steady(p.copy(), s)                 # set-up solve: operators, factorisation, graph
        ms = []
        for _ in range(3):
            m.steady(p.copy(), s)
            ms.append(m.stats()["device_ms"])
        st = m.stats()
        rec = {"ms_per_solve": statistics.median(ms), "refinements": st["refinements"],
               "iterations": st["cycles"], "fp64_residual_W": st["residual"], "cells": m.n_cells,
               "flow_ml_min": sc.flow_ml_min}
        if grid == 128:
            from oracle.restatement import OracleModel
            o = OracleModel(sc)
            t0 = time.perf_counter()
            T, Tb = o.steady_direct(p)
            rec["cpu_direct_s"] = time.perf_counter() - t0
            rec["max_dT_K_vs_fp64_direct"] = float(np.max(np.abs(m.grid("steady") - T)))
        out[f"{grid}x{grid}"] = rec
        m.close()
    big = out["512x512"]
    peak, peak_kind = measured_peak()
    # 104 B per cell per BiCGStab iteration (FP32: two operator applications
    # of x read, y write and 5 coefficients, and about 12 vector streams)
    achieved = 104.0 * big["cells"] * big["iterations"] / (big["ms_per_solve"] / 1e3) / 1e9
    return {"workload": "Si 0.1 mm + 0.2 mm water-channel layer (100 um channels, 200 um pitch) + spreader/sink, "
                        "512x512 over 10.24x10.24 mm", "solves_per_s": 1e3 / big["ms_per_solve"],
            "sizes": out,
            "roofline": {"bound": "hbm", "kernel": "BiCGStab iteration (bc_*)", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind, "traffic": None,
                         "note": "104 B per cell per iteration algorithmic (unpreconditioned BiCGStab's streams); "
                                 "the V-cycle preconditioner's plane solves are sequential chains, so the "
                                 "iteration is latency-bound, not HBM-bound"},
            "cpu_baseline": {"kind": "port", "what": "FP64 sparse LU (scipy splu) of the restated system, 1 thread",
                             "sample": "128x128 model", "s_per_solve": out["128x128"]["cpu_direct_s"]}}


def leg_serving(args):
    """The serving mix through hsb_server_run: at the offered 2000 req/s (with
    a probe stream of the latency-SLO class so its p99 rests on >= 200
    samples), and at a sustainable rate where latency reflects service
    rather than queueing."""
    from hotspot_b200.serving import Request, Server, latency_report, serving_mix
    d = tempfile.mkdtemp(prefix="hsb_srv_")
    workers = 8
    srv = Server(workers=workers)
    t0 = time.perf_counter()
    hp = [(256, 4)]              # the latency-SLO class (256x256, 4 chip layers, steady): high priority
    mix = serving_mix(d, srv, seed=4, rate=2000.0, duration=args.serving_seconds, high_priority_classes=hp,
                      replicas=args.serving_replicas, probe_rate=args.serving_probe_rate, probe_class=hp[0])
    calm = serving_mix(d, srv, seed=5, rate=args.serving_calm_rate, duration=args.serving_calm_seconds,
                       high_priority_classes=hp, reuse=mix, replicas=args.serving_replicas)
    if args.serving_batching:
        srv.set_batching(True)
    # every resident model (every member of every pool) serves one request before the clock starts
    warm = []
    for _, mi in mix.classes.items():
        r0 = next((r for r in mix.requests + calm.requests if r.model == mi), None)
        if r0 is None:
            continue
        steps = 1 if r0.kind == 0 else 2
        for _ in range(mix.members.get(mi, 1)):
            warm.append(Request(r0.model, r0.kind, r0.power if steps == 1 else r0.power[:2], 0.0, r0.temp_in,
                                steps, r0.dt, r0.tag))
    srv.run(warm)
    setup_s = time.perf_counter() - t0

    def report(reqs, rate, seconds):
        span = max(r.finish for r in reqs)
        tag = "steady_256_4"
        svc = [(r.finish - r.start) * 1e3 for r in reqs if r.tag == tag]
        return {"offered_req_per_s": rate, "arrival_window_s": seconds, "requests": len(reqs),
                "throughput_req_per_s": len(reqs) / span, "span_s": span,
                "latency_all": latency_report(reqs),
                "latency_steady": latency_report([r for r in reqs if r.kind == 0]),
                "latency_transient": latency_report([r for r in reqs if r.kind == 1]),
                "latency_steady_256x256_4layers": latency_report(reqs, tag),
                "service_ms_steady_256x256_4layers": float(np.median(svc)) if svc else None}
    e0 = srv.batch_stats()
    srv.run(mix.requests)
    e1 = srv.batch_stats()
    loaded = report(mix.requests, 2000.0 + args.serving_probe_rate, args.serving_seconds)
    ticks = e1["ticks"] - e0["ticks"]
    loaded["batch_engine"] = {
        "ticks": ticks,
        "requests_per_tick": ((e1["requests_per_tick"] * e1["ticks"] - e0["requests_per_tick"] * e0["ticks"]) / ticks
                              if ticks else 0.0),
        "request_intervals": e1["request_intervals"] - e0["request_intervals"]}
    srv.run(calm.requests)
    sustainable = report(calm.requests, args.serving_calm_rate, args.serving_calm_seconds)
    res = {"workload": "Poisson arrivals at 2000 req/s: 70% steady (sides 64..1024, 1..8 chip layers), 30% "
                       "500-interval transients (sides 64..256); plus a probe stream of the latency-SLO class "
                       f"(256x256, 4 chip layers, steady) at {args.serving_probe_rate:g} req/s; "
                       f"{args.serving_replicas} resident models per class of side <= 256 (a pool), one above; "
                       "the SLO class in the high-priority class with 2 reserved workers; other requests pause "
                       "between transient chunks and steady refinement passes while it runs; "
                       + ("transients served by the continuous batch engine (every admitted transient of one "
                          "interval length advanced together, a few intervals per launch; requests join and leave "
                          "between launches)" if args.serving_batching else "transients on the workers"),
           "models": len(mix.models), "workers": workers, "offered_2000_req_per_s": loaded,
           "sustainable_rate": sustainable, "setup_s": setup_s}
    srv.close()
    for m in mix.models:
        m.close()
    return res


def run_ours(args):
    import torch
    from hotspot_b200 import FORM_FAST, FORM_PARITY, _abi, replicas
    from hotspot_b200 import model as hm
    from hotspot_b200 import workloads as W

    ws, rank, local = dist()
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as tdist
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = tdist

    def barrier():
        if pg:
            pg.barrier()
        torch.cuda.synchronize()

    K, Wm = args.steps, max(3, args.warmup)
    work = tempfile.mkdtemp(prefix="hsb_bench_")
    LOAD = 4000    # trace rows reserved for the clock-sampling load window
    sc = W.scenario_stack3d(work, seed=100 + rank, grid=args.grid, steps=LOAD + Wm + 2 * K + 1)
    m = hm.from_scenario(sc)
    m.set_solver(FORM_FAST)
    ncell = m.n_cells
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    temp = m.vector(m.config.init_temp)
    m.compute_temp(m.power_vector(sc.block_power[0]), temp, sc.dt)
    for k in range(1, Wm + 1):
        m.compute_temp(m.power_vector(sc.block_power[k]), None, sc.dt)

    # ---- clocks: nvidia-smi samples every 200 ms over a load window of the
    # same workload (about 1 s, untimed) and the timed region that follows
    clocks = Clocks(local)
    barrier()
    clocks.start()
    t_load = time.perf_counter()
    k0 = Wm + 1
    while time.perf_counter() - t_load < 1.0 and k0 < Wm + 1 + LOAD and not args.profile:
        m.compute_temp(m.power_vector(sc.block_power[k0]), None, sc.dt)
        k0 += 1
    barrier()

    # ---- timed: device time of each interval, L2 flushed in between ----
    dev_ms = ker_ms = 0.0
    steps_total = launches = 0
    for k in range(k0, k0 + K):
        flush.fill_(float(k))
        torch.cuda.synchronize()
        m.compute_temp(m.power_vector(sc.block_power[k]), None, sc.dt)
        s = m.stats()
        dev_ms += s["device_ms"]
        ker_ms += s["kernel_ms"]
        steps_total += s["rk4_steps"]
        launches += s["launches"]
    barrier()
    clk = clocks.stop()
    fast_state = m.grid("trans")
    head_kernel = m.transient_kernel()
    if args.profile:
        print(json.dumps({"profile_case": True, "intervals": K, "device_ms": dev_ms,
                          "kernel_ms": ker_ms, "rk4_steps": steps_total}), flush=True)
        m.close()
        return

    # max over ranks of the device time; whole-job cell-steps
    dev_ms_max, cell_steps_all = replicas.reduce_timing(dev_ms, float(ncell * steps_total), pg, "cuda")
    value = cell_steps_all / (dev_ms_max / 1e3)

    # ---- e2e: the C-ABI call with host buffers (copies inside), wall clock ----
    L = _abi.lib()
    powers = [np.ascontiguousarray(m.power_vector(sc.block_power[k0 + k])) for k in range(K)]
    h2d = powers[0].nbytes
    d2h = temp.nbytes
    barrier()
    e2e_steps = 0
    t0 = time.perf_counter()
    for k in range(K):
        L.compute_temp_grid(m.ptr, _abi.dptr(powers[k]), None, sc.dt)
        e2e_steps += m.stats()["rk4_steps"]
    barrier()
    e2e_s = time.perf_counter() - t0
    e2e_max, e2e_work = replicas.reduce_timing(e2e_s, float(ncell * e2e_steps), pg, "cuda")
    e2e_value = e2e_work / e2e_max

    # ---- the same intervals as one multi-interval call (one persistent launch,
    # no host round trip between intervals; block powers copied in inside)
    trows = np.stack([m.power_vector(sc.block_power[k0 + K + k]) for k in range(K)])
    flush.fill_(3.0)
    torch.cuda.synchronize()
    _, tst = m.compute_trace(trows, None, sc.dt)
    trace = {"cell_steps_per_s": ncell * tst["rk4_steps"] / (tst["device_ms"] / 1e3), "intervals": K,
             "device_ms": tst["device_ms"], "kernel_ms": tst["kernel_ms"], "launches": tst["launches"],
             "h2d_bytes": int(trows.nbytes)}

    # ---- steady solves: fast MG-PCG ----
    avg = m.power_vector(sc.block_power[: k0 + K].mean(0))
    st_fast = m.vector()
    for _ in range(2):
        m.steady(avg.copy(), st_fast)
    reps = 5
    fast_ms = []
    for _ in range(reps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        m.steady(avg.copy(), st_fast)
        fast_ms.append(m.stats()["device_ms"])
    steady_fast_residual = m.stats()["residual"]
    steady_fast = 1e3 / statistics.median(fast_ms)
    steady_fast_grid = m.grid("steady")

    extra = {}
    if not args.no_plain:
        # the FP64 forms on the same trace: the replay of the reference's own
        # operation order (bit-identical to it), and the temporally blocked
        # Krylov form with FP64 passes (within 1e-6 K of the replay)
        from hotspot_b200 import FORM_FAST_BLOCKED, FORM_FP64_BLOCKED
        plain = {}
        for name, form in (("replay", FORM_PARITY), ("fp64_blocked", FORM_FP64_BLOCKED),
                           ("fast_blocked", FORM_FAST_BLOCKED)):
            mp_ = hm.from_scenario(sc)
            mp_.set_solver(form)
            tp = mp_.vector(mp_.config.init_temp)
            mp_.compute_temp(mp_.power_vector(sc.block_power[0]), tp, sc.dt)
            for k in range(1, k0):      # the same rows the fast form ran before its timed region
                mp_.compute_temp(mp_.power_vector(sc.block_power[k]), None, sc.dt)
            pdev, psteps, pl = 0.0, 0, 0
            for k in range(k0, k0 + K):
                flush.fill_(float(k))
                torch.cuda.synchronize()
                mp_.compute_temp(mp_.power_vector(sc.block_power[k]), None, sc.dt)
                s = mp_.stats()
                pdev += s["device_ms"]
                psteps += s["rk4_steps"]
                pl += s["launches"]
            plain[name] = {"state": mp_.grid("trans"), "rate": ncell * psteps / (pdev / 1e3), "launches": pl}
            if name == "replay":
                sp = mp_.vector()
                mp_.steady(avg.copy(), sp)
                plain[name]["steady_ms"] = mp_.stats()["device_ms"]
                plain[name]["steady_grid"] = mp_.grid("steady")
            mp_.close()
        rp, fb, tb = plain["replay"], plain["fp64_blocked"], plain["fast_blocked"]
        # the converged FP64 steady solution by sparse direct LU (the oracle's
        # restatement of the steady system, scipy splu)
        from oracle.restatement import OracleModel
        t_dir = time.perf_counter()
        T_direct, _ = OracleModel(sc).steady_direct(avg.copy())
        t_dir = time.perf_counter() - t_dir
        extra = {
            "plain_fp64": {"cell_steps_per_s": rp["rate"], "gpu_launches": rp["launches"],
                           "steady_solves_per_s": 1e3 / rp["steady_ms"],
                           "speedup_fast_vs_plain_transient": value / (rp["rate"] * ws),
                           "speedup_fast_vs_plain_steady": steady_fast * rp["steady_ms"] / 1e3,
                           "what": "the FP64 replay of the reference's RK4 stage by stage (10 stencil kernels per "
                                   "attempt, host step control with the reference's pow); steady: the replay of its "
                                   "nested-iteration Gauss-Seidel, stopping where the reference stops"},
            "fp64_blocked": {"cell_steps_per_s": fb["rate"], "gpu_launches": fb["launches"],
                             "speedup_fast_vs_fp64_blocked_transient": value / (fb["rate"] * ws),
                             "max_dT_K_vs_replay": float(np.max(np.abs(fb["state"] - rp["state"]))),
                             "what": "the temporally blocked Krylov-form kernel with every stencil pass in FP64: "
                                     "the fastest all-FP64 transient here"},
            "fast_blocked": {"cell_steps_per_s": tb["rate"], "gpu_launches": tb["launches"],
                             "max_dT_K_vs_replay": float(np.max(np.abs(tb["state"] - rp["state"]))),
                             "what": "the fast form's arithmetic on the temporally blocked kernel (the fast form's "
                                     "kernel from 2^21 cells up; this chip is below that size)"},
            "max_dT_K": {"transient_fast_vs_fp64_replay": float(np.max(np.abs(fast_state - rp["state"]))),
                         "steady_fast_vs_fp64_replay": float(np.max(np.abs(steady_fast_grid - rp["steady_grid"]))),
                         "steady_fast_vs_fp64_direct": float(np.max(np.abs(steady_fast_grid - T_direct))),
                         "steady_replay_vs_fp64_direct": float(np.max(np.abs(rp["steady_grid"] - T_direct))),
                         "direct_solve_s": t_dir,
                         "note": "the FP64 replay stops where the reference stops (per-sweep change < 1e-6 K), "
                                 "short of the converged fixed point; the fast steady solve converges to the FP64 "
                                 "direct (sparse LU) solution"},
        }

    if rank != 0:
        m.close()
        if pg:
            pg.destroy_process_group()
        return

    peak, peak_kind = measured_peak()
    alg_bytes_launch = ALG_BYTES_FP32 * ncell * steps_total / K
    # the kernel's own events; if the library could not time it, the whole interval
    kernel_timed = ker_ms > 0
    achieved = alg_bytes_launch / (((ker_ms if kernel_timed else dev_ms) / K) / 1e3) / 1e9
    kname = {"passes": "rk4_krylov_kernel", "blocked": "rk4_tb_kernel"}.get(head_kernel, head_kernel)
    traffic = profiled_traffic(f"{kname}_stack256.md")
    line = {
        "metric": METRIC, "value": value, "unit": "cell-steps/s", "n_gpus": ws, "steps": K,
        "warmup": Wm, "ms_per_step": dev_ms_max / K, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
        "config": headline_config(args.grid, ncell, ws),
        "e2e": {"value": e2e_value, "unit": "cell-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "steady_solves_per_s": {"fast": steady_fast, "unit": "solves/s",
                                "fast_final_fp64_residual_W": steady_fast_residual},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peak,
                     "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic,
                     "alg_bytes_per_launch": alg_bytes_launch,
                     "note": "one launch = one sampling interval; 108 B per cell-step algorithmic (the pass-by-"
                             "pass form's FP32 stage fields + FP64 state r/w + FP32 power); the fast form runs the "
                             "pass-by-pass kernel below 2^21 cells, and the 393k-cell working set fits the 126 MB "
                             "L2, so the launch is bound by latency and grid barriers, not HBM" +
                             ("" if kernel_timed else "; kernel events unavailable: duration = the whole interval's "
                                                      "device time")},
        "gpu_launches": launches,
        "trace": dict(trace, note="K intervals through hsb_dev_transient_trace: one persistent launch, device "
                                  "time including the copy of the K block-power rows"),
        "clocks": dict(clk, window="nvidia-smi every 200 ms over ~1 s of this workload just before the timed "
                                  "region and over the timed region"),
        "rk4_steps_per_interval": steps_total / K,
    }
    line.update(extra)
    if ws == 1:
        procs = max(1, min(os.cpu_count() or 1, 16))
        rate, cores, kind, cs, el = cpu_throughput(args.grid, 2, procs)
        line["cpu_baseline"] = {"value": rate, "unit": "cell-steps/s", "cores": cores, "kind": kind,
                                "sample": f"2 rows of the same workload x {cores} independent "
                                          "single-threaded replicas"}
    if ws == 1 and not args.headline_only:
        legs = set(args.legs.split(","))
        for name, fn in (("chip2d", lambda: leg_chip2d(args, flush)), ("batched", lambda: leg_batched(args, flush)),
                         ("microchannel", lambda: leg_microchannel(args)), ("serving", lambda: leg_serving(args))):
            if name not in legs:
                continue
            try:
                line[name] = fn()
            except Exception as e:      # a failed leg is reported, the headline still prints
                line[name] = {"error": f"{type(e).__name__}: {e}"}
        # per-request latency of the reference on the host, from the 2-D chip
        # leg's single-threaded reference runs (the serving mix's smallest
        # class, 64x64): a steady request, and a 500-interval transient
        c0, sv = line.get("chip2d", {}), line.get("serving", {})
        cb = c0.get("cpu_baseline") if isinstance(c0, dict) else None
        if cb and isinstance(sv, dict) and "error" not in sv:
            sv["cpu_reference_per_request"] = {
                "steady_64x64_s": cb["steady_s"],
                "transient_500_intervals_64x64_s": cb["trace_s"] * 500.0 / args.chip2d_rows,
                "cores": 1,
                "sample": f"the 2-D chip leg's reference runs: one steady solve, {args.chip2d_rows} rows scaled to "
                          "500; larger classes take longer in proportion to their cells"}
    print(json.dumps(line), flush=True)
    m.close()
    if pg:
        pg.destroy_process_group()


def profile_case(args):
    """Small cases of the batched transient, the MG steady solve of the
    serving latency class and the BiCGStab solver, sized for ncu (a few GB on
    the device at most)."""
    from hotspot_b200 import FORM_FAST, STEADY_BICGSTAB
    from hotspot_b200 import model as hm
    from hotspot_b200 import workloads as W
    d = tempfile.mkdtemp(prefix="hsb_prof_")
    if args.profile_case == "batch":
        from hotspot_b200.batch import Batch
        rng = np.random.default_rng(7)
        # 16 x 256x256x10 + 8 x 128x128x6 + 8 x 64x64x4: 11.4M cells, 180 MB
        # of FP64 state and candidate buffers, above the 126 MB L2
        specs = [(256, 8)] * 16 + [(128, 4)] * 8 + [(64, 2)] * 8
        scs = [W.scenario_random_chip(d, rng, f"p{i}", side=s, chip_layers=l, steps=8)
               for i, (s, l) in enumerate(specs)]
        models = []
        for sc in scs:
            m = hm.from_scenario(sc)
            m.set_solver(FORM_FAST)
            t = m.vector(m.config.init_temp)
            m.compute_temp(m.power_vector(sc.block_power[0]), t, 0.0)
            models.append(m)
        bt = Batch(models)
        bt.set_schedule(0, 1.0)
        out = []
        for k in range(1, 4):
            st = bt.transient([m.power_vector(sc.block_power[k]) for sc, m in zip(scs, models)], scs[0].dt)
            out.append({"kernel_ms": st["kernel_ms"], "rk4_steps": st["rk4_steps"]})
        print(json.dumps({"profile_case": "batch", "cells": int(sum(m.n_cells for m in models)), "intervals": out}))
        bt.close()
    elif args.profile_case == "steady":
        # the serving latency class: one 256x256 chip with 4 chip layers, MG-PCG to 1e-5 K
        sc = W.scenario_random_chip(d, np.random.default_rng([0, 256, 4, 1]), "p", side=256, chip_layers=4, steps=0)
        m = hm.from_scenario(sc)
        m.set_solver(FORM_FAST, steady_tol=1e-5)
        nblk = sum(m.layer_units[l] for l in range(m.n_layers) if m.layer_power[l])
        p = m.power_vector(np.random.default_rng(1).uniform(0.5, 20.0, nblk))
        s = m.vector()
        m.steady(p.copy(), s)
        st = m.stats()
        print(json.dumps({"profile_case": "steady", "cells": m.n_cells, "device_ms": st["device_ms"],
                          "refinements": st["refinements"], "cycles": st["cycles"]}))
        m.close()
    else:
        sc = W.scenario_microchannel(d, seed=3, grid=128, die=128 * 20e-6, blocks=8)
        m = hm.from_scenario(sc)
        m.set_solver(FORM_FAST, STEADY_BICGSTAB)
        p = m.power_vector(sc.block_power[0])
        s = m.vector()
        res = []
        for _ in range(2):
            m.steady(p.copy(), s)
            res.append(m.stats()["device_ms"])
        print(json.dumps({"profile_case": "microchannel", "cells": m.n_cells, "device_ms": res}))
        m.close()


def main():
    args = parse()
    if args.profile_case:
        profile_case(args)
        return
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
