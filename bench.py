#!/usr/bin/env python
"""Throughput of the B200 Saint-Venant RK time step on the single large catchment:
4096 x 4096 cells, dx = 2 m, diamond-square bed (Hurst 0.8, 100 m relief) + 0.005 slope,
lognormal rainfall field (mean 30 mm/h) for 1800 s, Voronoi Manning classes, outflow on
every edge, classic RK4, CFL target 0.5.

One "step" of this benchmark is one accepted RK4 timestep of the whole grid; the metric is
cell-updates/s (cells x accepted timesteps / device seconds). Inputs are seeded synthetic
fields with the workload's shapes and statistics. Before timing, the catchment is spun up
from dry for --spinup timesteps so the timed timesteps see wet/dry fronts and channel
flow. Every state field (134 MB in FP64) is larger than the 126 MB L2.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Under torchrun each rank runs an independent replica on its own GPU (replicas only: one
catchment never spans GPUs); timing is the max over ranks, value sums the ranks' work.
--impl reference times the CPU oracle (the reference's arithmetic restated in C++, OpenMP on
all host cores) on a bounded sample of the same workload; rank 0 alone runs it.
"""
import argparse
import json
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
# algorithmic HBM bytes per cell-update, one pass per RK stage (classic RK4):
# 52 values (state in/out, accumulator, bed) + 4 (per-cell n) + 4 (per-cell rain pattern)
VALUES_PER_CELL_UPDATE = 60


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=200)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--precision", default="f64", choices=["f64", "f32"])
    p.add_argument("--size", type=int, default=4096)
    p.add_argument("--spinup", type=int, default=600, help="timesteps run from dry before timing")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--variant", default="auto", help="stage-kernel variant 0-6, or auto (autotune)")
    return p.parse_args()


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
    nx = ny = size
    w = synth.config2(nx, ny, 2.0, seed=2)
    return w


def rain_series():
    from mfcm_b200 import TimeSeries
    # uniform time profile of the spatial field: on for the first 1800 s
    return TimeSeries([0.0, 1800.0, 1800.001, 1e7], [1.0, 1.0, 0.0, 0.0])


def make_solver(w, precision, device):
    from mfcm_b200 import SaintVenantSolver
    s = SaintVenantSolver(w["nx"], w["ny"], w["dx"], precision=precision, cn_target=0.5,
                          rain_mode="physical", step_duration=60.0, initial_dt=1.0, device=device)
    upload(s, w)
    return s


def upload(s, w):
    zeros = np.zeros((w["ny"], w["nx"]))
    s.set_field("Z", w["z"])
    s.set_field("H", zeros)
    s.set_field("U", zeros)
    s.set_field("V", zeros)
    s.set_field("N_SHALLOW", w["n"])
    s.set_field("N_DEEP", w["n"])
    s.set_field("RAIN_PATTERN", w["rain"])


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

    def run(self, n, timing=False):
        """Run n timesteps (accepted or repeated), crossing step boundaries as needed."""
        tot = {"total_ms": 0.0, "stage_ms": 0.0, "finalize_ms": 0.0, "stage_launches": 0, "finalize_launches": 0,
               "begin_launches": 0, "timesteps": 0}
        st0 = self.s.stats()
        done_so_far = 0
        last = st0
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
            if ran == 0:
                break
        tot["timesteps"] = done_so_far
        return last, tot

    def spinup(self, timesteps):
        """Spin up by a count of timesteps, not simulated seconds: the reference's velocity
        formulation can blow up in thin films on steep cells, where dt shrinks without bound
        and a fixed simulated span would never end."""
        if timesteps > 0:
            self.run(timesteps)


def roofline_traffic(precision):
    """Per-launch DRAM bytes of the stage kernel from the committed ncu capture, scaled to
    the 4096^2 grid (None when no capture was committed)."""
    p = os.path.join(ROOT, "profiles", f"stage_kernel_{precision}_traffic.json")
    try:
        d = json.load(open(p))
        return d["bytes_per_cell_per_launch"]
    except Exception:
        return None


def measured_peaks():
    try:
        d = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(w, state, cpu_seconds, precision="f64"):
    """The oracle (reference arithmetic restated in C++, OpenMP, all host threads) on a
    1024 x 1024 window of the spun-up catchment; timed over whole accepted timesteps."""
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
    o.set_forcing(forcing_at(600.0, 60.0))
    o.set_dt(state["dt"])
    t_local, dt = 0.0, state["dt"]
    # one untimed warm-up timestep, then whole accepted timesteps until the budget is used
    cn, rep, nd = o.do_timestep(t_local, dt)
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
            "sample": f"{acc} accepted RK4 timesteps of a {n}x{n} window of the spun-up 4096^2 catchment "
                      f"({precision}, {el:.1f} s, OpenMP {used} threads)"}


def run_reference(args):
    rank, _, world = dist_env()
    if rank != 0:
        return 0
    w = workload(min(args.size, 1024))
    zeros = np.zeros((w["ny"], w["nx"]))
    # state: a thin film stands in for the spun-up state (no GPU on this arm)
    state = {"h": zeros + 0.02, "u": zeros, "v": zeros, "dt": 0.5}
    per_step = max(2.0, args.cpu_seconds / max(1, args.steps))
    vals = []
    for _ in range(args.warmup if args.warmup < 2 else 1):
        cpu_baseline(w, state, min(per_step, 2.0), args.precision)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        vals.append(cpu_baseline(w, state, per_step, args.precision))
    el = time.perf_counter() - t0
    v = statistics.median([x["value"] for x in vals])
    cb = dict(vals[-1])
    cb["value"] = v
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / max(1, args.steps), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
            "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "config": {"workload": f"{w['nx']}x{w['ny']} window of the 4096x4096 dx=2 m catchment (oracle port, "
                                   "reference not buildable here)", "scheme": "classic RK4", "cn_target": 0.5}}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    rank, local_rank, world = dist_env()
    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    device = local_rank
    torch.cuda.set_device(device)

    w = workload(args.size)
    ncells = w["nx"] * w["ny"]
    solver = make_solver(w, args.precision, device)
    runner = Runner(solver)
    if args.variant == "auto":
        # tune on a partly spun-up state, then finish the spin-up with the chosen kernel
        first = min(50, args.spinup)
        runner.spinup(first)
        variant = solver.autotune()
        runner.spinup(args.spinup - first)
    else:
        variant = int(args.variant)
        solver.set_kernel_variant(variant)
        runner.spinup(args.spinup)
    # warm-up timesteps (untimed)
    runner.run(max(3, args.warmup))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)

    sampler = ClockSampler(device)
    barrier()
    st0 = solver.stats()
    sampler.start()
    last, tm = runner.run(args.steps, timing=True)
    barrier()
    clocks = sampler.stop()
    st1 = solver.stats()
    accepted = st1["accepted"] - st0["accepted"]
    repeated = st1["repeated"] - st0["repeated"]
    ms_max, work = reduce_over_ranks(tm["total_ms"], float(accepted * ncells), dist, f"cuda:{device}")
    value = work / (ms_max * 1e-3)

    # roofline of the dominant kernel (the fused stage kernel)
    bpv = 8 if args.precision == "f64" else 4
    alg_bytes_launch = VALUES_PER_CELL_UPDATE / 4.0 * bpv * ncells
    real_stage_launches = solver.nstages * tm["timesteps"]
    stage_avg_s = tm["stage_ms"] * 1e-3 / max(1, real_stage_launches)
    achieved = alg_bytes_launch / stage_avg_s / 1e9
    peak, peak_kind = measured_peaks()
    traffic_pc = roofline_traffic(args.precision)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": (traffic_pc * ncells if traffic_pc else None), "peak_kind": peak_kind,
            "alg_bytes_per_launch": alg_bytes_launch, "stage_launch_ms": stage_avg_s * 1e3,
            "stage_share_of_step": tm["stage_ms"] / max(1e-9, tm["total_ms"])}

    state = None
    if rank == 0 and (not args.no_cpu or not args.no_e2e):
        state = {"h": solver.get_field("H"), "u": solver.get_field("U"), "v": solver.get_field("V"),
                 "dt": solver.get_dt()}

    e2e = None
    if not args.no_e2e:
        e2e = measure_e2e(w, args, device, state)
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline(w, state, args.cpu_seconds, args.precision)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / max(1, args.steps), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
                "config": {"workload": f"single catchment {w['nx']}x{w['ny']}, dx=2 m (diamond-square H0.8 100 m + "
                                       "0.005 slope, lognormal rain field 30 mm/h, Voronoi n, outflow all edges)",
                           "scheme": "classic RK4", "cn_target": 0.5, "precision": args.precision,
                           "spinup_timesteps": args.spinup, "sim_time_s": runner.t_step, "l2": "inputs larger than L2 (each state field 134 MB)",
                           "parallelism": f"replicas x{world}", "kernel_variant": variant, "accepted": accepted, "repeated": repeated},
                "roofline": roof, "cpu_baseline": cb, "e2e": e2e, "clocks": clocks,
                "gpu_launches": int(tm["stage_launches"] + tm["finalize_launches"] + tm["begin_launches"])}
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    solver.close()
    return 0


def measure_e2e(w, args, device, state):
    """End to end through the public API from host arrays: upload the inputs (bed, state,
    Manning n, rain pattern) from pinned host memory, run the same number of timesteps, read
    the state back; wall clock with the device synchronised on both sides."""
    import torch
    from mfcm_b200 import SaintVenantSolver
    pinned = {}
    for k, a in (("z", w["z"]), ("n", w["n"]), ("rain", w["rain"]),
                 ("h", state["h"] if state else np.zeros_like(w["z"])),
                 ("u", state["u"] if state else np.zeros_like(w["z"])),
                 ("v", state["v"] if state else np.zeros_like(w["z"]))):
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).pin_memory()
        pinned[k] = t.numpy()
    s = SaintVenantSolver(w["nx"], w["ny"], w["dx"], precision=args.precision, cn_target=0.5, rain_mode="physical",
                          step_duration=60.0, initial_dt=state["dt"] if state else 1.0, device=device)
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    s.set_field("Z", pinned["z"])
    s.set_field("H", pinned["h"])
    s.set_field("U", pinned["u"])
    s.set_field("V", pinned["v"])
    s.set_field("N_SHALLOW", pinned["n"])
    s.set_field("N_DEEP", pinned["n"])
    s.set_field("RAIN_PATTERN", pinned["rain"])
    r = Runner(s, t0=600.0)
    r.run(args.steps)
    st = s.stats()
    out_h = s.get_field("H")
    out_u = s.get_field("U")
    out_v = s.get_field("V")
    torch.cuda.synchronize(device)
    el = time.perf_counter() - t0
    ncells = w["nx"] * w["ny"]
    h2d = 6 * ncells * 8
    d2h = 3 * ncells * 8 + 40
    s.close()
    del out_h, out_u, out_v
    return {"value": st["accepted"] * ncells / el, "unit": UNIT,
            "h2d_bytes_per_step": h2d / max(1, args.steps), "d2h_bytes_per_step": d2h / max(1, args.steps),
            "seconds": el, "accepted": st["accepted"],
            "what": "upload bed/state/n/rain from pinned host memory, run the timesteps, read h/u/v back"}


if __name__ == "__main__":
    sys.exit(main())
