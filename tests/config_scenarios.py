"""The benchmark configurations at full size, as runs that record one digest per output time.

Shared by tests/golden/make_config_golden.py (which runs them on the oracle and commits the
digests) and tests/test_gpu_parity_configs.py (which runs them on the CUDA path and compares).

  plane256_*     256 x 256, dx = 5 m, plane of slope 0.01 plus 8 Gaussian bumps (seed 1),
                 rain 50 mm/h for 600 s (ramped to zero over the next 60 s step), Manning
                 n = 0.03, walls plus an outflow strip on the lowest edge, control-number target
                 0.5, 3600 s, outputs every 600 s, in three modes: the reference rain clamp from
                 dry (max dt 10 s: from a dry, still state the reference's next dt is infinite;
                 no cell ever holds water, and the ramp-down step drains some below zero),
                 the reference clamp on a 1 mm film, and the physical clamp from dry
  fractal1024    1024 x 1024 window of the 4096 x 4096, dx = 2 m catchment (diamond-square bed,
                 Hurst 0.8, 100 m relief, plus a 0.005 slope; lognormal rain field, mean
                 30 mm/h; Voronoi Manning classes; outflow on every edge), 60 s from dry
  dambreak8192   8192 x 1024, dx = 0.5 m, bed 350 m, 1 m of water upstream of the centre,
                 frictionless, walls, 2 s in steps of 1 s
"""
import hashlib

import numpy as np

from mfcm_b200 import solve, synth
from tests.scenarios import rain_series, setup

SCENARIOS = {
    "plane256_reference_dry": dict(kind="plane", mode="reference_dry"),
    "plane256_reference_film": dict(kind="plane", mode="reference_film"),
    "plane256_physical_dry": dict(kind="plane", mode="physical_dry"),
    "fractal1024": dict(kind="fractal"),
    "dambreak8192": dict(kind="dambreak"),
}


def digest(fields):
    """SHA-256 of FP64 fields with -0.0 folded into +0.0 and NaNs made canonical."""
    h = hashlib.sha256()
    for a in fields:
        a = np.asarray(a, dtype=np.float64)
        a = np.where(np.isnan(a), np.nan, a + 0.0)
        h.update(np.ascontiguousarray(a, dtype="<f8").tobytes())
    return h.hexdigest()


def _record(solver, t0, t1, every, **kw):
    outs = []

    def on_step(t, s):
        if abs((t - t0) / every - round((t - t0) / every)) < 1e-9:
            st = s.stats()
            f = [s.get_field(n) for n in ("H", "U", "V")]
            outs.append(dict(t=t, accepted=int(st["accepted"]), repeated=int(st["repeated"]),
                             volume=float(st["volume"]), max_h=float(np.nanmax(f[0])), digest=digest(f)))

    solve(solver, t0, t1, on_step=on_step, **kw)
    return outs


def run(name, make):
    """Run scenario `name` on a backend made by make(nx, ny, dx, **params); returns the record."""
    sc = SCENARIOS[name]
    if sc["kind"] == "plane":
        c = synth.config1()
        nx, ny, dx, z = c["nx"], c["ny"], c["dx"], c["z"]
        mode = sc["mode"]
        kw = dict(cn_target=0.5, rain_mode="physical" if mode == "physical_dry" else "reference",
                  step_duration=60.0, initial_dt=1.0, max_dt=10.0 if mode == "reference_dry" else 0.0)
        b = make(nx, ny, dx, **kw)
        h = np.full((ny, nx), 1e-3 if mode == "reference_film" else 0.0)
        setup(b, z, h, np.zeros_like(h), np.zeros_like(h), n=(c["n"], c["n"], 0.1, 0.3))
        outs = _record(b, 0.0, 3600.0, 600.0, rain=rain_series(c["rain_rate"], stop=600.0), head=0.0,
                       head_edges=c["edges"])
    elif sc["kind"] == "fractal":
        nx = ny = 1024
        c = synth.config2(nx=nx, ny=ny)
        kw = dict(cn_target=0.5, rain_mode="physical", step_duration=60.0, initial_dt=1.0)
        b = make(nx, ny, c["dx"], **kw)
        h = np.zeros((ny, nx))
        setup(b, c["z"], h, h, h, n=(0.03, 0.03, 0.1, 0.3), n_field=c["n"])
        b.set_field("RAIN_PATTERN", c["rain"])
        # SV_RAIN_PATTERN with scale 1: every cell takes its own rain rate
        outs = _record(b, 0.0, 60.0, 60.0, rain=1.0, rain_kind=3, head=0.0, head_edges=c["edges"])
    else:
        nx, ny, dx = 8192, 1024, 0.5
        z, h = synth.dam_break(nx, ny, 350.0, 1.0)
        kw = dict(cn_target=0.5, rain_mode="reference", step_duration=1.0, initial_dt=0.01, manning=False)
        b = make(nx, ny, dx, **kw)
        setup(b, z, h, np.zeros_like(h), np.zeros_like(h))
        outs = _record(b, 0.0, 2.0, 1.0)
    rec = dict(outputs=outs, dt=float(b.get_dt()))
    b.close()
    return rec
