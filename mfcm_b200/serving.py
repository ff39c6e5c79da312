"""Continuous-batching flood-solve server.

Requests (a catchment, its rainfall and a simulated horizon) arrive at wall-clock times. Each
request is prepared as soon as a slot and its device memory fit under the budget: a thread
creates its solver and uploads its bed while the batch (mfcm_b200.batch) advances the others.
The batch advances every running request by a few steps per call (`steps_per_advance`), each
request at its own pace; prepared requests join it between calls (sv_batch_adopt), so
requests that arrive while others are on the GPU join the next launches without waiting for
their own set-up. A request leaves the batch when its horizon is reached, freeing its memory
for the queue. Each request's results are bit-identical whether it runs alone or in the mix
(members never share state).

A request whose solve fails is failed alone: a member whose time turns NaN, or which takes
more than `step_limit` timesteps within one step (the reference's thin-film velocity
blow-up on steep beds, where dt shrinks without bound), is removed with its reason recorded
while the rest of the batch completes the same step.

The reference has no serving layer; this is a production serving pattern built on the same
step (one `step()` of TypedTemporalScheme per batch advance, per member).
"""
import collections
import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import synth, SaintVenantSolver, TimeSeries, start_new_step_forcing, RAIN_UNIFORM
from .batch import SaintVenantBatch
from ._abi import SV_E_NONFINITE


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the server starts
    nx: int
    ny: int
    dx: float
    z: np.ndarray
    rain: TimeSeries        # m/s, uniform over the catchment
    horizon: float          # simulated seconds
    n: float = 0.035
    head_edges: int = 15    # outflow on every edge
    # filled in by the server
    admitted: float = math.nan
    finished: float = math.nan
    error: str = None       # why the solve failed (None: completed)
    cell_updates: int = 0
    steps: int = 0
    result_h: np.ndarray = None
    stats: dict = field(default_factory=dict)

    @property
    def latency(self):
        return self.finished - self.arrival


def triangular_hyetograph(peak_mm_h, duration_s, end=1e9):
    """Rain rate rising linearly to peak at duration/2 and back to zero at duration."""
    p = peak_mm_h * synth.MM_PER_H
    return TimeSeries([0.0, duration_s / 2.0, duration_s, end], [0.0, p, 0.0, 0.0])


def catchment_bed(nx, ny, dx, slope, relief_frac, seed, hurst=0.8, smooth_m=10.0):
    """A catchment bed: a regional `slope` toward +x plus fractal relief of `relief_frac`
    times the catchment's longer side, smoothed over `smooth_m` metres (bed slopes of a few
    to twenty-odd percent, like gridded terrain at metre resolution)."""
    r = relief_frac * max(nx, ny) * dx
    z = synth.gaussian_smooth(synth.diamond_square(nx, ny, hurst, r, seed=seed), smooth_m / dx)
    return z + synth.regional_slope(nx, ny, dx, slope)


def fractal_bed(nx, ny, relief_m, seed, hurst=0.8):
    """A seeded diamond-square bed of `relief_m` metres (max - min) and Hurst exponent `hurst`,
    unsmoothed."""
    return synth.diamond_square(nx, ny, hurst, relief_m, seed=seed)


def make_requests(rate, count, seed=0, side=(64, 512), dxs=(1.0, 2.0, 5.0), horizon=(120.0, 600.0),
                  slope=(0.005, 0.03), relief=(0.01, 0.03), peak=(20.0, 120.0), duration=(900.0, 7200.0),
                  hurst=0.8, relief_m=None, multiple=1):
    """Poisson arrivals at `rate` requests/s; mesh side log-uniform on `side` (rounded to a
    multiple of `multiple`); beds from `catchment_bed` with regional slope U(`slope`) and relief
    U(`relief`) x length, or, with `relief_m` = (lo, hi), raw fractal beds (`fractal_bed`) of
    relief U(relief_m) metres."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        s = int(round(math.exp(rng.uniform(math.log(side[0]), math.log(side[1]))) / multiple)) * multiple
        s = max(s, multiple)
        dx = float(rng.choice(dxs))
        if relief_m is None:
            z = catchment_bed(s, s, dx, float(rng.uniform(*slope)), float(rng.uniform(*relief)), seed * 100003 + i,
                              hurst)
        else:
            z = fractal_bed(s, s, float(rng.uniform(*relief_m)), seed * 100003 + i, hurst)
        rain = triangular_hyetograph(float(rng.uniform(*peak)), float(rng.uniform(*duration)))
        out.append(Request(i, t, s, s, dx, z, rain, float(rng.uniform(*horizon))))
    return out


def at_rate(requests, rate, seed=0):
    """The same requests (same catchments, rain and horizons) arriving as a Poisson stream of
    `rate` requests/s: fresh copies whose arrival times are redrawn, timings cleared."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for r in requests:
        t += rng.exponential(1.0 / rate)
        out.append(Request(r.rid, t, r.nx, r.ny, r.dx, r.z, r.rain, r.horizon, r.n, r.head_edges))
    return out


class FloodServer:
    """Requests are prepared off the batch's path: a preparation thread creates each arriving
    request's solver and uploads its bed and roughness on the solver's own stream while the
    batch advances; between advances the main loop adopts every prepared solver into the
    batch (sv_batch_adopt), so an arrival waits for the current advance to end, not for its
    own preparation. persistent: each batch advance is one persistent cooperative launch
    (every running request at its own dt, idle warps taking work from any request); else one
    launch per RK stage and one per timestep's reductions, replayed as a graph."""

    def __init__(self, budget_bytes=150e9, max_slots=512, precision="f32", step_duration=60.0, cn_target=0.5,
                 device=0, step_limit=20000, steps_per_advance=4, persistent=False):
        self.batch = SaintVenantBatch(precision, "classic", device)
        self.batch.set_step_limit(step_limit)
        if persistent:
            self.batch.set_persistent(True)
        self.precision = precision
        self.device = int(device)
        # steps each running request advances per batched launch sequence: members run them
        # back to back at their own pace; new arrivals are adopted between sequences
        self.steps_per_advance = int(steps_per_advance)
        self.budget = float(budget_bytes)
        self.max_slots = int(max_slots)
        self.L = float(step_duration)
        self.cn_target = float(cn_target)
        self.value_bytes = 8 if precision == "f64" else 4

    def estimate_bytes(self, req):
        """Device memory of one member: 15 cell fields (two states, two stage buffers, bed and
        its slopes), the per-cell Manning field, and the per-tile partial sums. Field uploads
        stage through one FP64 buffer (8 bytes per cell of the largest mesh) that the library's
        pool holds outside this estimate."""
        cells = req.nx * req.ny
        tiles = math.ceil(req.nx / 32) * math.ceil(req.ny / 8)
        return cells * self.value_bytes * 16 + tiles * 11 * 8 + 4096

    def _prepare(self, req):
        """The request as a solver of its own: bed and roughness uploaded on its own stream; the
        state starts dry and still (the library zeroes it)."""
        s = SaintVenantSolver(req.nx, req.ny, req.dx, precision=self.precision, cn_target=self.cn_target,
                              step_duration=self.L, rain_mode="physical", device=self.device)
        s.set_field("Z", req.z)
        s.set_manning(req.n, req.n, 0.1, 0.3)
        return s

    def run(self, requests, time_limit=None):
        """Serve `requests` (sorted by arrival). Returns a summary dict; the requests carry
        their own timings and results."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        ready = []                     # (request, solver) prepared, waiting for adoption
        lock = threading.Lock()
        wake, freed, stop = threading.Event(), threading.Event(), threading.Event()
        shared = {"used": 0.0, "slots": 0, "error": None}
        t0 = time.perf_counter()

        def preparer():
            try:
                while pending and not stop.is_set():
                    req = pending[0]
                    delay = req.arrival - (time.perf_counter() - t0)
                    if delay > 0:
                        stop.wait(min(delay, 0.05))
                        continue
                    need = self.estimate_bytes(req)
                    with lock:  # a request larger than the budget still runs once nothing else holds memory
                        fits = shared["slots"] < self.max_slots and (
                            shared["used"] + need <= self.budget or shared["slots"] == 0)
                        if fits:
                            shared["used"] += need
                            shared["slots"] += 1
                    if not fits:
                        freed.wait(0.05)
                        freed.clear()
                        continue
                    pending.popleft()
                    solver = self._prepare(req)
                    with lock:
                        ready.append((req, solver))
                    wake.set()
            except Exception as e:  # reported by the main loop
                shared["error"] = e
                wake.set()

        worker = threading.Thread(target=preparer, daemon=True)
        worker.start()
        active = {}   # slot -> [request, member, simulated time]
        total_updates = 0
        max_active = 0
        try:
            while True:
                now = time.perf_counter() - t0
                if time_limit is not None and now > time_limit:
                    break
                if shared["error"] is not None:
                    raise shared["error"]
                with lock:
                    joining = list(ready)
                    ready.clear()
                for req, solver in joining:
                    m = self.batch.adopt(solver)
                    req.admitted = now
                    active[m.slot] = [req, m, 0.0]
                max_active = max(max_active, len(active))
                if not active:
                    if not pending and not ready and not worker.is_alive():
                        break
                    wake.wait(0.05)
                    wake.clear()
                    continue
                queued = {}
                for slot, (req, m, t) in active.items():
                    left = max(1, math.ceil((req.horizon - t) / self.L - 1e-9))
                    queued[m] = [start_new_step_forcing(t + i * self.L, self.L, rain=req.rain,
                                                        rain_kind=RAIN_UNIFORM, head=0.0, head_edges=req.head_edges)
                                 for i in range(min(self.steps_per_advance, left))]
                res = self.batch.advance_steps(queued, raise_on_error=False)
                done = []
                for slot, entry in active.items():
                    req, m, t = entry
                    r = res[slot]
                    for st in r["steps"]:
                        req.cell_updates += st["accepted"] * req.nx * req.ny
                        total_updates += st["accepted"] * req.nx * req.ny
                    req.steps += len(r["steps"])
                    entry[2] = t + self.L * len(r["steps"])
                    if r["status"] != 0:
                        req.error = ("time became NaN" if r["status"] == SV_E_NONFINITE else
                                     "step limit reached (dt collapsed)")
                        req.stats = m.stats()
                        req.finished = time.perf_counter() - t0
                        done.append(slot)
                    elif entry[2] >= req.horizon - 1e-9:
                        req.result_h = m.get_field("H")
                        req.stats = m.stats()
                        req.finished = time.perf_counter() - t0
                        done.append(slot)
                for slot in done:
                    req, m, _ = active.pop(slot)
                    self.batch.remove(m)
                    with lock:
                        shared["used"] -= self.estimate_bytes(req)
                        shared["slots"] -= 1
                    freed.set()
        finally:
            stop.set()
            worker.join()
            with lock:
                leftover = list(ready)
                ready.clear()
            for _, solver in leftover:  # prepared but never adopted (time limit)
                solver.close()
        wall = time.perf_counter() - t0
        lat = np.array([r.latency for r in requests if not math.isnan(r.finished) and r.error is None])
        failures = {}
        for r in requests:
            if r.error is not None:
                failures[r.error] = failures.get(r.error, 0) + 1
        admit_wait = [r.admitted - r.arrival for r in requests if not math.isnan(r.admitted)]
        return {
            "requests": len(requests), "completed": int(lat.size),
            "failed": sum(1 for r in requests if r.error is not None), "wall_s": wall,
            "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "p95_s": float(np.percentile(lat, 95)) if lat.size else None,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else None,
            "admission_wait_p50_s": float(np.percentile(admit_wait, 50)) if admit_wait else None,
            "cell_updates_per_s": total_updates / wall if wall > 0 else 0.0,
            "max_concurrent": max_active, "failures": failures,
        }

    def close(self):
        self.batch.close()
