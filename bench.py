#!/usr/bin/env python
"""Throughput of the B200 Saint-Venant RK time step.

Workload: the single large catchment. It is 4096 x 4096 cells at dx = 2 m, with a
diamond-square bed (Hurst 0.8, 100 m relief) plus a 0.005 regional slope. Rainfall is a
lognormal field (mean 30 mm/h, sigma_log 0.5, smoothed over 200 m) for 1800 s. Manning n comes
from Voronoi land classes, and every edge is an outflow. The scheme is classic RK4 at CFL 0.5.

The metric: batched FP32 vs plain FP64 cell-updates/s at <= 1 mm depth error, with p50/p99
latency.

- `value` is the FP32 path (FP32 state and arithmetic, bed as FP32 offsets from FP64 tile
  datums, FP64 reductions and dt control). It counts cell-updates/s: cells x accepted
  timesteps per device second.
- `fp64` is the plain FP64 path, which is bit-identical to the reference arithmetic.
- `precision` gives the FP32 paths' max depth error against FP64 on a dam break over a 350 m
  bed (the wet/dry-front precision study).
- `serving` gives p50/p95/p99 latency of a continuous-batching run.
- `batched` gives the throughput of an ensemble of uneven catchments advancing in shared
  launches.

One "step" is one accepted RK4 timestep of the whole grid. Inputs are seeded synthetic fields
with the workload's shapes and statistics. Before timing, the plain FP64 path runs the first
60 s step from dry (at most --spinup-cap timesteps); every precision starts from that state.
Every FP64 state field (134 MB) is larger than the 126 MB L2.

Every phase is bounded by a count of timesteps rather than by simulated seconds. On this bed
the reference's velocity formulation blows up in finite time: a cell holding a 2 mm film beside
a nearly dry cell reaches |u| ~ 1e3 m/s, du/dt grows faster than the control number lets dt
shrink, and simulated time converges on a limit it never passes (t ~ 91 s in the 1024 x 1024
window). A loop run to a later step boundary would never end, in the reference as here.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank runs an independent replica on its own GPU: one catchment never
spans GPUs. The time is the max over ranks, and the value sums the ranks' work.
--impl reference times the CPU oracle on a bounded window of the same workload, with OpenMP
on all host cores. The oracle restates the reference's arithmetic in C++ at the reference's
shipped FP32 precision. Rank 0 alone runs it.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Batched FP32 vs plain FP64 cell-updates/s at ≤1mm depth err; p50/p99 latency"
UNIT = "cell-updates/s"
# algorithmic HBM values per cell-update, one pass per RK stage (classic RK4):
# 52 (state in/out, accumulator, bed) + 4 (per-cell Manning n) + 4 (per-cell rain pattern)
VALUES_PER_CELL_UPDATE = 60


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=100)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--precision", default="f32_datum64", choices=["f32_datum64", "f32", "f64"],
                   help="precision of the headline value")
    p.add_argument("--size", type=int, default=4096)
    p.add_argument("--spinup-cap", type=int, default=4000,
                   help="most timesteps of the FP64 run through the first 60 s step before timing")
    p.add_argument("--error-span", type=float, default=10.0,
                   help="simulated seconds both precisions advance from the common state for the headline error")
    p.add_argument("--cpu-seconds", type=float, default=12.0)
    p.add_argument("--window-steps", type=int, default=1,
                   help="60 s steps from dry of the 1024^2 window both CPU baselines are timed on")
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the fp64, precision, serving, batched parts")
    p.add_argument("--variant", default="auto", help="stage-kernel variant 0-13, or auto (autotune)")
    return p.parse_args()


_T0 = time.perf_counter()


def log(msg):
    """Progress on stderr (the JSON line alone goes to stdout)."""
    print(f"[bench {time.perf_counter() - _T0:7.1f} s] {msg}", file=sys.stderr, flush=True)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = [r for r in self.rows if len(r) >= 9]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def reduce_over_ranks(ms, work, dist, device="cpu"):
    """Replicas only: the job's time is the slowest rank's device time, its work the sum of
    the ranks' accepted cell-updates. No simulation data crosses ranks."""
    if dist is None:
        return ms, work
    import torch
    t_max = torch.tensor([ms], dtype=torch.float64, device=device)
    w_sum = torch.tensor([work], dtype=torch.float64, device=device)
    dist.all_reduce(t_max, op=dist.ReduceOp.MAX)
    dist.all_reduce(w_sum, op=dist.ReduceOp.SUM)
    return float(t_max.item()), float(w_sum.item())


def workload(size):
    from mfcm_b200 import synth
    return synth.config2(size, size, 2.0, seed=2)


def rain_series():
    from mfcm_b200 import TimeSeries
    # uniform time profile of the spatial rain field: on for the first 1800 s
    return TimeSeries([0.0, 1800.0, 1800.001, 1e7], [1.0, 1.0, 0.0, 0.0])


def make_solver(w, precision, device, step_duration=60.0, **kw):
    from mfcm_b200 import SaintVenantSolver
    s = SaintVenantSolver(w["nx"], w["ny"], w["dx"], precision=precision, cn_target=0.5,
                          rain_mode="physical", step_duration=step_duration, initial_dt=1.0, device=device, **kw)
    zeros = np.zeros((w["ny"], w["nx"]))
    s.set_field("Z", w["z"])
    for f in ("H", "U", "V"):
        s.set_field(f, zeros)
    s.set_field("N_SHALLOW", w["n"])
    s.set_field("N_DEEP", w["n"])
    s.set_field("RAIN_PATTERN", w["rain"])
    return s


def forcing_at(t, L):
    from mfcm_b200 import start_new_step_forcing, RAIN_PATTERN
    return start_new_step_forcing(t, L, rain=rain_series(), rain_kind=RAIN_PATTERN, head=0.0, head_edges=15)


class Runner:
    """Drives TypedTemporalScheme::solve timestep by timestep: start_new_step at each step
    boundary, device-controlled timesteps in between."""

    def __init__(self, solver, t0=0.0):
        self.s = solver
        self.t_step = t0
        self.L = solver.step_duration
        self.need_begin = True

    def run(self, n, timing=False, stop_at_boundary=False):
        """Run n timesteps (accepted or repeated), crossing step boundaries as needed (or
        stopping at the first one)."""
        tot = {"total_ms": 0.0, "stage_ms": 0.0, "finalize_ms": 0.0, "stage_launches": 0, "finalize_launches": 0,
               "begin_launches": 0, "timesteps": 0}
        last = self.s.stats()
        done_so_far = 0
        while done_so_far < n:
            if self.need_begin:
                self.s.set_forcing(forcing_at(self.t_step, self.L))
            st, done, tm = self.s.run_timesteps(n - done_so_far, begin=self.need_begin, timing=timing)
            tot["begin_launches"] += 1
            if tm:
                for k in ("total_ms", "stage_ms", "finalize_ms", "stage_launches", "finalize_launches"):
                    tot[k] += tm[k]
            self.need_begin = done
            if done:
                self.t_step += self.L
            ran = (st["accepted"] + st["repeated"]) - (last["accepted"] + last["repeated"])
            last = st
            done_so_far += ran
            if ran == 0 or (done and stop_at_boundary):
                break
        tot["timesteps"] = done_so_far
        return last, tot

    def run_step(self, cap, chunk=50):
        """Run the current step to its end, at most `cap` timesteps (accepted or repeated):
        the reference's velocity formulation can blow up in thin films on steep cells, where dt
        shrinks without bound and the step would never end. Returns True when the step ended."""
        ran = 0
        start = self.t_step
        while ran < cap and self.t_step == start:
            _, tot = self.run(min(chunk, cap - ran), stop_at_boundary=True)
            if tot["timesteps"] == 0:
                break
            ran += tot["timesteps"]
            log(f"  t_step {start:.0f} s: {ran} timesteps, dt {self.s.get_dt():.3g} s")
        return self.t_step != start


def common_state(w, args, device):
    """The state every precision is timed from: the plain FP64 path (bit for bit the
    reference arithmetic) run from dry through the first 60 s step, a step boundary from which
    a solver of either precision starts the next step. If the step does not end within
    --spinup-cap timesteps the state at the cap is used and the line says so."""
    s = make_solver(w, "f64", device)
    r = Runner(s)
    ended = r.run_step(args.spinup_cap)
    st = s.stats()
    state = {"h": s.get_field("H"), "u": s.get_field("U"), "v": s.get_field("V"), "dt": s.get_dt(),
             "t_step": r.t_step if ended else 0.0, "step_ended": ended,
             "spinup_accepted": st["accepted"], "spinup_repeated": st["repeated"]}
    s.close()
    return state


def solver_at(w, precision, state, device, step_duration=60.0):
    """A solver of `precision` holding the common state (FP64 values rounded once to FP32 for
    the FP32 paths) and its next timestep."""
    s = make_solver(w, precision, device, step_duration=step_duration)
    for f in ("H", "U", "V"):
        s.set_field(f, state[f.lower()])
    s.set_dt(state["dt"])
    return s


def headline_error(w, state, precision, device, span, cap=3000):
    """Error of the FP32 headline against FP64 on the headline workload itself: from the common
    state both advance one step of `span` simulated seconds (device-controlled timesteps, at
    most `cap` each), then the depth fields and FP64 volumes are compared."""
    out = {}
    for prec in ("f64", precision):
        s = solver_at(w, prec, state, device, step_duration=span)
        r = Runner(s, t0=state["t_step"])
        ended = r.run_step(cap)
        st = s.stats()
        out[prec] = (s.get_field("H"), st["volume"], st["accepted"], st["repeated"], ended)
        s.close()
    if not (out["f64"][4] and out[precision][4]):
        return {"case": f"{span:g} s from the common state at t = {state['t_step']:.0f} s",
                "reached": {p: out[p][4] for p in out}, "cap_timesteps": cap}
    d = np.abs(out[precision][0] - out["f64"][0])
    wet = out["f64"][0] > 1e-3
    return {"case": f"{span:g} s from the common state at t = {state['t_step']:.0f} s",
            "max_depth_err_m": float(d.max()), "p99_depth_err_m": float(np.percentile(d, 99)),
            "mean_depth_err_m": float(d.mean()), "cells_over_1mm_fraction": float((d > 1e-3).mean()),
            "max_depth_err_wet_m": float(d[wet].max()) if wet.any() else None,
            "rel_volume_err": abs(out[precision][1] - out["f64"][1]) / out["f64"][1],
            "accepted": {precision: out[precision][2], "f64": out["f64"][2]},
            "repeated": {precision: out[precision][3], "f64": out["f64"][3]}}


def profile_traffic(name, key="bytes_per_cell_per_launch"):
    """Per-launch DRAM bytes (or warp instructions) per cell of a stage kernel from a committed
    ncu capture."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", name)))[key]
    except Exception:
        return None


def measured_peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def dominant_kernel(variant, precision):
    """The stage kernel that does most of a variant's work on the benchmark mesh, whose
    interior strips (all but the edge strips) run the interior form of the column sweep."""
    if variant < 4 or variant == 11:
        return "stage_kernel"
    if precision != "f64" and variant == 8:
        return "sweep_batch_kernel"  # FP32 with the batches' variant runs the batched sweep as a batch of one
    if variant in (12, 13):
        return "sweep_pair_kernel"
    return "sweep_interior_kernel"


def timed_run(w, precision, args, device, barrier, dist, state):
    """From the common state: pick the kernel, then time args.steps timesteps with per-kernel
    events."""
    solver = solver_at(w, precision, state, device)
    runner = Runner(solver, t0=state["t_step"])
    if args.variant == "auto":
        variant = solver.autotune()
        tune = solver.autotune_ms()
    else:
        variant = int(args.variant)
        tune = None
        solver.set_kernel_variant(variant)
    runner.run(max(3, args.warmup))
    st0 = solver.stats()
    barrier()
    sampler = ClockSampler(device)
    sampler.start()
    _, tm = runner.run(args.steps, timing=True)
    barrier()
    clocks = sampler.stop()
    st1 = solver.stats()
    ncells = w["nx"] * w["ny"]
    accepted = st1["accepted"] - st0["accepted"]
    repeated = st1["repeated"] - st0["repeated"]
    ms_max, work = reduce_over_ranks(tm["total_ms"], float(accepted * ncells), dist, f"cuda:{device}")
    bpv = 8 if precision == "f64" else 4
    alg_bytes_launch = VALUES_PER_CELL_UPDATE / 4.0 * bpv * ncells
    stage_avg_s = tm["stage_ms"] * 1e-3 / max(1, solver.nstages * tm["timesteps"])
    achieved = alg_bytes_launch / stage_avg_s / 1e9
    peak, peak_kind = measured_peaks()
    kernel = dominant_kernel(variant, precision)
    traffic_pc = profile_traffic(f"{kernel}_{precision}_2048_traffic.json")
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": (traffic_pc * ncells if traffic_pc else None), "peak_kind": peak_kind,
            "traffic_source": (f"profiles/{kernel}_{precision}_2048_traffic.json scaled to {w['nx']}x{w['ny']} cells"
                               if traffic_pc else None),
            "kernel": f"{kernel} (variant {variant})", "alg_bytes_per_launch": alg_bytes_launch,
            "stage_launch_ms": stage_avg_s * 1e3, "stage_share_of_step": tm["stage_ms"] / max(1e-9, tm["total_ms"])}
    # the bound that holds: instruction issue. Warp instructions per cell from the same ncu
    # capture; each of the 148 SMs' 4 schedulers issues at most one per cycle at the SM clock
    # sampled during the timed region
    inst_pc = profile_traffic(f"{kernel}_{precision}_2048_traffic.json", "warp_inst_per_cell_per_launch")
    if inst_pc and clocks.get("sm_mhz"):
        issue_ms = inst_pc * ncells / (148 * 4 * clocks["sm_mhz"] * 1e6) * 1e3
        roof["issue"] = {"warp_inst_per_cell": inst_pc, "issue_limited_ms": issue_ms,
                         "frac": issue_ms / (stage_avg_s * 1e3), "sm_mhz": clocks["sm_mhz"]}
    res = {"value": work / (ms_max * 1e-3), "ms": ms_max, "accepted": accepted, "repeated": repeated,
           "variant": variant, "autotune_ms": tune, "roofline": roof, "clocks": clocks, "timesteps": tm["timesteps"],
           "sim_time_s": runner.t_step, "ms_per_timestep": tm["total_ms"] / max(1, tm["timesteps"]),
           "stage_ms": stage_avg_s * 1e3,
           "launches": int(tm["stage_launches"] + tm["finalize_launches"] + tm["begin_launches"])}
    return solver, res


def precision_study(device, nx=8192, ny=1024, dx=0.5, seconds=60.0, h0=1.0, cap=20000):
    """Dam break on a flat bed at 350 m (8192 x 1024 cells, dx = 0.5 m, h = h0 for x below the
    centre, dry beyond, frictionless, no rain, 60 s): max depth error and relative volume
    error of the FP32 paths against FP64, the front position of each against Ritter's
    2 sqrt(g h0) t, and the depth and velocity at the dam against Ritter's 4/9 h0 and
    2/3 sqrt(g h0). The depth error is given over the whole grid and away from the moving
    bore (cells more than 20 m from FP64's front), because a bore that arrives one timestep
    earlier or later differs there by up to its own height whatever the precision. Each run
    stops after `cap` timesteps if it has not reached the end by then (reached_end)."""
    from mfcm_b200 import SaintVenantSolver, synth
    z, h = synth.dam_break(nx, ny, 350.0, h0)
    out = {}
    mid = nx // 2
    for prec in ("f64", "f32", "f32_datum64"):
        s = SaintVenantSolver(nx, ny, dx, precision=prec, cn_target=0.5, step_duration=seconds, manning=False,
                              initial_dt=0.01, device=device)
        s.set_field("Z", z)
        s.set_field("H", h)
        t0 = time.perf_counter()
        st, reached, _ = s.run_timesteps(cap, begin=True)  # the whole span unless dt collapses
        el = time.perf_counter() - t0
        hf, uf = s.get_field("H"), s.get_field("U")
        wet = np.where(hf[ny // 2, mid:] > 1e-3)[0]
        out[prec] = {"h": hf, "volume": s.stats()["volume"], "front_m": (wet.max() + 1) * dx if wet.size else 0.0,
                     "h_dam": float(hf[ny // 2, mid]), "u_dam": float(uf[ny // 2, mid]), "accepted": st["accepted"],
                     "repeated": st["repeated"], "seconds": el, "reached_end": reached}
        s.close()
    h64, v64 = out["f64"]["h"], out["f64"]["volume"]
    c0 = math.sqrt(9.81 * h0)
    res = {"case": f"dam break {nx}x{ny}, dx={dx} m, bed 350 m, h0 = {h0} m, {seconds:.0f} s, no friction",
           "ritter_front_m": 2.0 * c0 * seconds, "ritter_h_dam": 4.0 / 9.0 * h0, "ritter_u_dam": 2.0 / 3.0 * c0}
    x = (np.arange(nx) + 0.5) * dx - mid * dx
    away = np.abs(x - out["f64"]["front_m"]) > 20.0
    for prec in ("f64", "f32", "f32_datum64"):
        o = out[prec]
        r = {k: o[k] for k in ("front_m", "h_dam", "u_dam", "accepted", "repeated", "seconds", "reached_end")}
        if prec != "f64":
            d = np.abs(o["h"] - h64)
            r["max_depth_err_m"] = float(d.max())
            r["max_depth_err_away_from_bore_m"] = float(d[:, away].max())
            r["mean_depth_err_m"] = float(d.mean())
            r["rel_volume_err"] = abs(o["volume"] - v64) / v64
            r["within_1mm"] = r["max_depth_err_m"] <= 1e-3
        res[prec] = r
    return res


SERVING_RATES = (5.0, 10.0, 20.0, 50.0, 100.0, 200.0)


def serving_sweep(device, count=24, horizon_scale=1.0 / 60.0, precision="f32_datum64", persistent=False,
                  time_limit=30.0, step_s=10.0, step_limit=400):
    """The serving stream at every arrival rate of SERVING_RATES: `count` requests with mesh sides
    log-uniform on [128, 4096] (multiples of 32), dx in {1, 2, 5} m, raw fractal beds (Hurst 0.8,
    relief U(10, 150) m), triangular hyetographs (peak U(20, 120) mm/h, duration U(900, 7200) s),
    Manning n = 0.035, outflow on every edge, FP32 state with FP64 reductions, admitted against
    a 150 GB device-memory budget, in steps of `step_s` simulated seconds (admission happens at
    step boundaries). Horizons are U(1, 6) h scaled by `horizon_scale` (so that one rate's
    stream runs in about `time_limit` seconds); the same requests arrive at every rate, as a
    fresh Poisson stream. A request whose dt collapses (the reference scheme's thin-film blow-up
    on steep cells: more than `step_limit` timesteps in one step, a mean dt below
    step_s / step_limit) is failed and counted as failed; requests still running at the time
    limit are counted as unfinished."""
    from mfcm_b200.serving import FloodServer, make_requests, at_rate
    base = make_requests(1.0, count, seed=11, side=(128, 4096), dxs=(1.0, 2.0, 5.0),
                         horizon=(3600.0 * horizon_scale, 21600.0 * horizon_scale), relief_m=(10.0, 150.0),
                         peak=(20.0, 120.0), duration=(900.0, 7200.0), multiple=32)
    per_rate = []
    log("serving requests generated")
    for rate in SERVING_RATES:
        reqs = at_rate(base, rate, seed=int(rate))
        srv = FloodServer(budget_bytes=150e9, precision=precision, device=device, persistent=persistent,
                          steps_per_advance=1, step_limit=step_limit, step_duration=step_s)
        summary = srv.run(reqs, time_limit=time_limit)
        srv.close()
        log(f"serving at {rate:g}/s: {summary['completed']} completed, {summary['failed']} failed, "
            f"p50 {summary['p50_s']}")
        summary["arrival_rate_per_s"] = rate
        summary["unfinished"] = summary["requests"] - summary["completed"] - summary["failed"]
        per_rate.append(summary)
    cells = [r.nx * r.ny for r in base]
    return {"requests_per_rate": count, "mesh_side": [128, 4096], "dx_m": [1, 2, 5], "relief_m": [10, 150],
            "horizon_s": [3600.0 * horizon_scale, 21600.0 * horizon_scale], "horizon_scale": horizon_scale,
            "horizon_note": "U(1, 6) h scaled down by the stated factor at every rate",
            "step_s": step_s, "time_limit_s": time_limit, "step_limit": step_limit,
            "cells_per_request": [min(cells), max(cells)], "kernel": "persistent batch kernel" if persistent
            else "batched launches per stage", "per_rate": per_rate}


def ensemble_members(count=64, seed=13):
    """The batched ensemble: `count` catchments with sides log-uniform on [256, 2048] rounded
    to multiples of 32, aspect U(0.5, 2), dx = 2 m, catchment beds (0.5-3 % regional slope
    plus smoothed fractal relief of 1-3 % of the catchment length), a 1 cm initial film,
    uniform rain U(10, 100) mm/h and Manning n U(0.02, 0.08)."""
    from mfcm_b200 import synth
    from mfcm_b200.serving import catchment_bed
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        side = math.exp(rng.uniform(math.log(256), math.log(2048)))
        asp = rng.uniform(0.5, 2.0)
        nx = max(32, int(round(side * math.sqrt(asp) / 32)) * 32)
        ny = max(32, int(round(side / math.sqrt(asp) / 32)) * 32)
        z = catchment_bed(nx, ny, 2.0, rng.uniform(0.005, 0.03), rng.uniform(0.01, 0.03), 1000 + i)
        out.append({"nx": nx, "ny": ny, "z": z, "n": rng.uniform(0.02, 0.08),
                    "rate": rng.uniform(10, 100) * synth.MM_PER_H})
    return out


def batched_run(device, members, precision, steps=6, per_call=3, step_s=10.0, persistent=True, perturb=0.0):
    """The ensemble advanced together, `per_call` queued steps per call (each member at its own
    pace): in one persistent launch per call, or in one launch per RK stage and timestep.
    Members that fail leave; only members that complete a step count toward the throughput.
    `perturb` multiplies each member's initial film by 1 + perturb * N(0, 1) (the noise-floor
    run). Returns the summary and each surviving member's final depth."""
    from mfcm_b200 import start_new_step_forcing, RAIN_UNIFORM
    from mfcm_b200.batch import SaintVenantBatch
    import torch
    b = SaintVenantBatch(precision, device=device)
    b.set_step_limit(2000)   # 10-s steps: a member whose dt falls below 5 ms has blown up
    if persistent:
        b.set_persistent(True, 0, 900.0)  # a call runs 5 steps of 64 catchments: allow minutes
    rng = np.random.default_rng(77)
    live = []
    for i, d in enumerate(members):
        m = b.add(d["nx"], d["ny"], 2.0, cn_target=0.5, step_duration=step_s, rain_mode="physical")
        m.set_field("Z", d["z"])
        film = np.full((d["ny"], d["nx"]), 0.01)
        if perturb:
            film = film * (1.0 + perturb * rng.standard_normal(film.shape))
        m.set_field("H", film)
        m.set_manning(d["n"], d["n"], 0.1, 0.3)
        live.append((i, m))
    v0 = {i: m.stats()["volume"] for i, m in live}
    cells = sum(d["nx"] * d["ny"] for d in members)
    failed = []
    k0 = 0

    def run(nsteps):
        nonlocal live, k0
        res = b.advance_steps({m: [start_new_step_forcing(step_s * (k0 + j), step_s, rain=members[i]["rate"],
                                                          rain_kind=RAIN_UNIFORM, head=0.0, head_edges=15)
                                   for j in range(nsteps)] for i, m in live}, raise_on_error=False)
        k0 += nsteps
        keep, work = [], 0
        for i, m in live:
            r = res[m.slot]
            if r["status"] != 0:
                failed.append(i)
                b.remove(m)
            else:
                work += sum(st["accepted"] for st in r["steps"]) * members[i]["nx"] * members[i]["ny"]
                keep.append((i, m))
        live = keep
        return work

    run(1)  # warm-up step (builds the launch graph)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    work = 0
    for _ in range(steps // per_call):
        work += run(per_call)
    torch.cuda.synchronize(device)
    el = time.perf_counter() - t0
    final = {}
    for i, m in live:
        st = m.stats()
        # mass balance of the whole run: V_end - (V_0 + rain in - outflow + wall flow), FP64
        closure = (st["volume"] - (v0[i] + st["rain_in"] - st["outflow"] + st["wall_in"])) / st["volume"]
        final[i] = (m.get_field("H"), st["volume"], closure)
    b.close()
    return ({"precision": precision, "catchments": len(members), "cells": cells, "steps": steps + 1,
             "timed_steps": steps, "step_s": step_s, "steps_per_call": per_call, "persistent": persistent,
             "cell_updates_per_s": work / el,
             "seconds": el, "failed_members": sorted(failed),
             "max_mass_balance_err": max((abs(f[2]) for f in final.values()), default=None)}, final)


def batched_ensemble(device, precision="f32_datum64"):
    """The ensemble in `precision` and in plain FP64, each in the persistent batch kernel; the
    FP32 run's max depth error and relative volume error against FP64 over the members that
    finished in both, member by member next to that member's noise floor: the FP64 run again
    from an initial film perturbed by 1e-7 relative (FP32 rounding size). The FP32 ensemble in
    one launch per stage is timed too, for comparison."""
    members = ensemble_members()
    r32, f32 = batched_run(device, members, precision)
    log(f"ensemble {precision}: {r32['cell_updates_per_s']:.3e}")
    r64, f64 = batched_run(device, members, "f64")
    log(f"ensemble f64: {r64['cell_updates_per_s']:.3e}")
    _, p64 = batched_run(device, members, "f64", perturb=1e-7)
    log("ensemble noise floor done")
    g32, _ = batched_run(device, members, precision, persistent=False)
    log(f"ensemble {precision} per-stage launches: {g32['cell_updates_per_s']:.3e}")
    both = sorted(set(f32) & set(f64))
    per_member = []
    for i in both:
        e = float(np.max(np.abs(f32[i][0] - f64[i][0])))
        floor = float(np.max(np.abs(p64[i][0] - f64[i][0]))) if i in p64 else None
        per_member.append({"member": i, "cells": members[i]["nx"] * members[i]["ny"], "max_depth_err_m": e,
                           "fp64_noise_floor_m": floor,
                           "within_noise_floor": bool(floor is not None and e <= max(floor, 1e-3)),
                           "rel_volume_diff": abs(f32[i][1] - f64[i][1]) / f64[i][1]})
    diffs = [np.abs(f32[i][0] - f64[i][0]) for i in both]
    over = sum(int((d > 1e-3).sum()) for d in diffs)
    ncmp = sum(d.size for d in diffs)
    r32.update({"fp64": r64, "fp32_over_fp64": r32["cell_updates_per_s"] / r64["cell_updates_per_s"],
                "compared_members": len(both),
                "max_depth_err_m": max((float(d.max()) for d in diffs), default=None),
                "p99_depth_err_m": max((float(np.percentile(d, 99)) for d in diffs), default=None),
                "mean_depth_err_m": float(sum(float(d.sum()) for d in diffs) / ncmp) if ncmp else None,
                "cells_over_1mm_fraction": over / ncmp if ncmp else None,
                "max_rel_volume_diff_vs_fp64": max((abs(f32[i][1] - f64[i][1]) / f64[i][1] for i in both),
                                                   default=None),
                "members_within_1mm": sum(1 for m in per_member if m["max_depth_err_m"] <= 1e-3),
                "members_within_noise_floor": sum(1 for m in per_member if m["within_noise_floor"]),
                "per_member": per_member, "launch_per_stage": g32,
                "persistent_over_launch_per_stage": r32["cell_updates_per_s"] / g32["cell_updates_per_s"],
                "note": "pointwise maxima sit on moving bores, where the FP64 scheme itself moves by millimetres "
                        "under a 1e-7 relative perturbation of the initial state (fp64_noise_floor_m per member)"})
    return r32


def window_workload(w, n=1024):
    """The top-left n x n window of the catchment's bed, Manning and rain fields, as a
    catchment of its own (outflow on its edges)."""
    n = min(n, w["nx"], w["ny"])
    sl = (slice(0, n), slice(0, n))
    return {"nx": n, "ny": n, "dx": w["dx"], "z": w["z"][sl], "n": w["n"][sl], "rain": w["rain"][sl]}


def window_state(w, steps, device=None):
    """The state both CPU baselines (this arm's and the reference arm's) are timed on: the
    1024 x 1024 window run from dry for `steps` whole 60 s steps in plain FP64 -- on the GPU
    here, on the oracle in the reference arm (which has no GPU). The two FP64 paths are bit for
    bit the same, so both arms time the CPU on the same state. The first step takes 37
    timesteps; the second never ends (the thin-film blow-up near 91 s), so `steps` is 1 or 0."""
    ww = window_workload(w)
    if device is not None:
        s = make_solver(ww, "f64", device)
    else:
        from oracle.sv_oracle_py import OracleSolver
        s = OracleSolver(ww["nx"], ww["ny"], ww["dx"], cn_target=0.5, rain_mode="physical", step_duration=60.0,
                         initial_dt=1.0, openmp=True, threads=os.cpu_count() or 1)
        zeros = np.zeros((ww["ny"], ww["nx"]))
        s.set_field("Z", ww["z"])
        for f in ("H", "U", "V"):
            s.set_field(f, zeros)
        s.set_field("N_SHALLOW", ww["n"])
        s.set_field("N_DEEP", ww["n"])
        s.set_field("RAIN_PATTERN", ww["rain"])
    if steps > 1:
        raise ValueError("the window's second 60 s step never ends under the reference scheme")
    acc = 0
    for k in range(steps):
        s.set_forcing(forcing_at(60.0 * k, 60.0))
        acc = s.advance()["accepted"]
    state = {"h": s.get_field("H"), "u": s.get_field("U"), "v": s.get_field("V"), "dt": s.get_dt(),
             "t_step": 60.0 * steps, "spinup_accepted": acc}
    s.close()
    return state


def cpu_baseline(w, state, cpu_seconds, precision):
    """The oracle (the reference's arithmetic restated in C++, OpenMP, all host threads) on the
    1024 x 1024 window of the catchment (window_workload), at the window state of
    window_state; timed over whole accepted timesteps."""
    from oracle.sv_oracle_py import OracleSolver, threads_available
    threads = os.cpu_count() or 1
    n = min(1024, w["nx"])
    sl = (slice(0, n), slice(0, n))
    o = OracleSolver(n, n, w["dx"], precision=precision, cn_target=0.5, rain_mode="physical", step_duration=60.0,
                     tallies=False, openmp=True, threads=threads)
    o.set_field("Z", w["z"][sl])
    o.set_field("H", state["h"][sl])
    o.set_field("U", state["u"][sl])
    o.set_field("V", state["v"][sl])
    o.set_field("N_SHALLOW", w["n"][sl])
    o.set_field("N_DEEP", w["n"][sl])
    o.set_field("RAIN_PATTERN", w["rain"][sl])
    o.set_forcing(forcing_at(state["t_step"], 60.0))
    dt = state["dt"]
    cn, rep, nd = o.do_timestep(0.0, dt)  # one untimed warm-up timestep
    if not rep:
        o.accept()
    dt = nd
    acc = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < cpu_seconds:
        cn, rep, nd = o.do_timestep(0.0, dt)
        if not rep:
            o.accept()
            acc += 1
        dt = nd
    el = time.perf_counter() - t0
    used = threads_available(True)
    return {"value": acc * n * n / el, "unit": UNIT, "cores": used, "kind": "port",
            "sample": f"{acc} accepted RK4 timesteps of the {n}x{n} window of the {w['nx']}x{w['ny']} catchment, "
                      f"from its FP64 state after {state['t_step']:.0f} s from dry "
                      f"(oracle {precision}, {el:.1f} s, OpenMP {used} threads)"}


def source_terms_cost(w, state, precision, variant, device, timesteps=20):
    """Stage-kernel time on the spun-up catchment with and without the energy-loss and
    infiltration terms (per-cell fx, fy, rate and a capacity read and written each stage:
    5 more values per cell per stage)."""
    ncells = w["nx"] * w["ny"]
    out = {}
    for on in (False, True):
        s = make_solver(w, precision, device)
        s.set_kernel_variant(variant)
        for f in ("H", "U", "V"):
            s.set_field(f, state[f.lower()])
        s.set_dt(state["dt"])
        if on:
            for name, val in (("ELOSS_FX", 0.05), ("ELOSS_FY", 0.05), ("INFIL_RATE", 2e-6), ("INFIL_CAP", 0.05)):
                s.set_field(name, np.full((w["ny"], w["nx"]), val))
        r = Runner(s, t0=state["t_step"])
        r.run(3)
        _, tm = r.run(timesteps, timing=True)
        out["with" if on else "without"] = tm["stage_ms"] / max(1, tm["stage_launches"])
        s.close()
    bpv = 8 if precision == "f64" else 4
    alg = (VALUES_PER_CELL_UPDATE + 4 * 5) / 4.0 * bpv * ncells
    peak, _ = measured_peaks()
    return {"terms": "energy loss + infiltration", "stage_ms_without": out["without"], "stage_ms_with": out["with"],
            "extra_values_per_cell_stage": 5,
            "roofline_frac_with": alg / (out["with"] * 1e-3) / 1e9 / peak}


def oracle_precision(p):
    return "f64" if p == "f64" else "f32"


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    w = workload(args.size)
    # the window state the GPU arm's CPU baseline is timed on, spun up here on the oracle
    state = window_state(w, args.window_steps)
    prec = oracle_precision(args.precision)
    # each step is a bounded sample (about 1 s of CPU work; at least one whole timestep)
    per_step = max(0.6, min(2.0, 120.0 / max(1, args.steps)))
    vals = []
    cpu_baseline(w, state, per_step, prec)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_baseline(w, state, per_step, prec))
    el = time.perf_counter() - t0
    v = statistics.median([x["value"] for x in vals])
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / max(1, args.steps), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": prec, "data": "synthetic", "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "config": {"workload": f"1024x1024 window of the {w['nx']}x{w['ny']} dx=2 m catchment from its FP64 "
                                   f"state after {state['t_step']:.0f} s from dry, oracle port of the reference "
                                   "arithmetic (the reference's SYCL build cannot be built here; the oracle is pinned "
                                   "bit for bit to the reference's kernels compiled on the CPU)",
                       "scheme": "classic RK4", "cn_target": 0.5, "same_state_as": "the b200 arm's cpu_baseline"}}
    print(json.dumps(line), flush=True)
    return 0


def measure_e2e(w, args, device, state, variant, precision, reps=3):
    """End to end through the public API from host arrays: upload the inputs (bed, state,
    Manning n, rain pattern) from pinned host memory, run the same number of timesteps, read
    the state back; wall clock with the device synchronised on both sides. Each repetition is
    a whole end-to-end run with a new solver; the median is reported, every run is listed."""
    import torch
    from mfcm_b200 import SaintVenantSolver
    pinned = {}
    for k, a in (("z", w["z"]), ("n", w["n"]), ("rain", w["rain"]), ("h", state["h"]), ("u", state["u"]),
                 ("v", state["v"])):
        pinned[k] = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory().numpy()
    results = {f: torch.empty(w["ny"] * w["nx"], dtype=torch.float64).pin_memory().numpy() for f in ("H", "U", "V")}
    ncells = w["nx"] * w["ny"]
    runs = []
    for _ in range(reps):
        s = SaintVenantSolver(w["nx"], w["ny"], w["dx"], precision=precision, cn_target=0.5, rain_mode="physical",
                              step_duration=60.0, initial_dt=state["dt"], device=device)
        s.set_kernel_variant(variant)
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        s.set_field("Z", pinned["z"])
        s.set_field("H", pinned["h"])
        s.set_field("U", pinned["u"])
        s.set_field("V", pinned["v"])
        s.set_field("N_SHALLOW", pinned["n"])
        s.set_field("N_DEEP", pinned["n"])
        s.set_field("RAIN_PATTERN", pinned["rain"])
        r = Runner(s, t0=state["t_step"])
        r.run(args.steps)
        st = s.stats()
        out = [s.get_field(f, out=results[f]) for f in ("H", "U", "V")]
        torch.cuda.synchronize(device)
        el = time.perf_counter() - t0
        s.close()
        del out
        runs.append((st["accepted"] * ncells / el, el, st["accepted"]))
    value, el, acc = sorted(runs)[len(runs) // 2]
    return {"value": value, "unit": UNIT,
            "h2d_bytes_per_step": 6 * ncells * 8 / max(1, args.steps),
            "d2h_bytes_per_step": (3 * ncells * 8 + 40) / max(1, args.steps),
            "seconds": el, "accepted": acc, "runs": [r[0] for r in runs], "runs_seconds": [r[1] for r in runs],
            "what": "upload bed/state/n/rain (FP64 host arrays) from pinned memory, run the timesteps, read h/u/v back "
                    "into pinned memory; median of the listed whole runs"}


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, local_rank, world = dist_env()
    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = local_rank
    torch.cuda.set_device(device)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)

    w = workload(args.size)
    log("workload ready")
    state = common_state(w, args, device)
    log(f"common FP64 state at t = {state['t_step']:.0f} s ({state['spinup_accepted']} accepted, "
        f"{state['spinup_repeated']} repeated timesteps; step ended: {state['step_ended']})")
    solver, main_res = timed_run(w, args.precision, args, device, barrier, dist, state)
    solver.close()
    log(f"{args.precision} timed: {main_res['value']:.3e} cell-updates/s, variant {main_res['variant']}")
    extras = {}
    if not args.no_extras and args.precision != "f64":
        s64, r64 = timed_run(w, "f64", args, device, barrier, dist, state)
        s64.close()
        log(f"f64 timed: {r64['value']:.3e} cell-updates/s, variant {r64['variant']}")
        extras["fp64"] = {"value": r64["value"], "ms_per_step": r64["ms"] / max(1, args.steps),
                          "ms_per_timestep": r64["ms_per_timestep"], "stage_ms": r64["stage_ms"],
                          "accepted": r64["accepted"], "repeated": r64["repeated"], "kernel_variant": r64["variant"],
                          "autotune_stage_ms": r64["autotune_ms"],
                          "roofline": r64["roofline"], "clocks": r64["clocks"]}
        # both arms start from the same state; the throughput ratio counts accepted timesteps,
        # so it also carries the two arms' accept/repeat decisions, which the per-timestep and
        # per-stage ratios do not
        extras["fp32_over_fp64"] = main_res["value"] / r64["value"]
        extras["fp32_over_fp64_per_timestep"] = r64["ms_per_timestep"] / main_res["ms_per_timestep"]
        extras["fp32_over_fp64_per_stage"] = r64["stage_ms"] / main_res["stage_ms"]
        if rank == 0:
            extras["headline_error_vs_fp64"] = headline_error(w, state, args.precision, device, args.error_span)
            log("headline error done")
    wstate = None
    if rank == 0 and world == 1 and not args.no_cpu:
        wstate = window_state(w, args.window_steps, device=device)
        log("window state done")
        if "fp64" in extras:
            extras["fp64"]["cpu_baseline"] = cpu_baseline(w, wstate, args.cpu_seconds, "f64")
    if rank == 0 and not args.no_extras:
        extras["precision"] = precision_study(device)
        # the same on a 2 cm dam: levels near 350 m then carry the depth in their last bits
        extras["precision_thin"] = precision_study(device, h0=0.02)
        log("precision studies done")
        extras["serving"] = serving_sweep(device)
        log("serving sweep done")
        extras["batched"] = batched_ensemble(device, args.precision)
        log("ensemble done")
    e2e = None
    if rank == 0 and not args.no_e2e:
        e2e = measure_e2e(w, args, device, state, main_res["variant"], args.precision)
        log("e2e done")
    if rank == 0 and not args.no_extras:
        extras["source_terms"] = source_terms_cost(w, state, args.precision, main_res["variant"], device)
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline(w, wstate, args.cpu_seconds, oracle_precision(args.precision))

    if rank == 0:
        line = {"metric": METRIC, "value": main_res["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": main_res["ms"] / max(1, args.steps), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "f64" else "f32",
                "data": "synthetic",
                "config": {"workload": f"single catchment {w['nx']}x{w['ny']}, dx=2 m (diamond-square H0.8 100 m + "
                                       "0.005 slope, lognormal rain field 30 mm/h, Voronoi n, outflow all edges)",
                           "scheme": "classic RK4", "cn_target": 0.5, "precision": args.precision,
                           "spinup_timesteps": state["spinup_accepted"] + state["spinup_repeated"],
                           "spinup_step_ended": state["step_ended"], "sim_time_s": main_res["sim_time_s"],
                           "start": f"common FP64 state at t = {state['t_step']:.0f} s for every precision",
                           "l2": "inputs larger than L2 (each FP64 state field 134 MB; FP32 67 MB x 13 fields)",
                           "parallelism": f"replicas x{world}", "kernel_variant": main_res["variant"],
                           "autotune_stage_ms": main_res["autotune_ms"],
                           "accepted": main_res["accepted"], "repeated": main_res["repeated"]},
                "roofline": main_res["roofline"], "cpu_baseline": cb, "e2e": e2e, "clocks": main_res["clocks"],
                "gpu_launches": main_res["launches"]}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
