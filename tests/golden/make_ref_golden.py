"""Regenerate the golden fixtures made by the reference's own code (tests/golden/ref_*.npz).

The fixtures are outputs of the reference's hot-path sources compiled by
oracle/ref_pin/build.py (its kernels, state arithmetic and RungeKuttaSolver step loop, run on
the CPU through a host-only SYCL stand-in). They let the oracle (CPU) and the CUDA path (GPU)
be checked against the reference where the reference tree is not available, bit for bit.
Needs the reference source tree:

    python tests/golden/make_ref_golden.py [fixture names]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mfcm_b200 import synth  # noqa: E402
from oracle.ref_pin import refpin  # noqa: E402
from tests.scenarios import wet_dry_state  # noqa: E402


def case_dudt(prec):
    """One update_dUdt on a 23 x 17 mesh with coded-out cells, per-cell Manning values,
    discharge values on most cells and head values on some (head listed first)."""
    nx, ny, dx, dy = 23, 17, 3.0, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=41, nan_cells=6)
    rng = np.random.default_rng(42)
    man = (rng.uniform(0.02, 0.05, (ny, nx)), rng.uniform(0.03, 0.3, (ny, nx)), np.full((ny, nx), 0.1),
           np.full((ny, nx), 0.3))
    q = (rng.uniform(0, 3e-5, (ny, nx)) * (rng.uniform(size=(ny, nx)) > 0.3), rng.uniform(0, 3e-5, (ny, nx)))
    hb0 = np.where(rng.uniform(size=(ny, nx)) > 0.8, rng.uniform(0, 0.1, (ny, nx)), np.nan)
    hb = (hb0, np.where(np.isnan(hb0), np.nan, 0.02))
    t, dt, L = 7.5, 0.37, 60.0
    dt_ = np.float64 if prec == "f64" else np.float32
    r = refpin.dudt(z, h, u, v, dx, dy, manning=man, q=q, head=hb, head_first=True, time_now=t, timestep=dt,
                    step_length=L, precision=prec)
    out = dict(nx=nx, ny=ny, dx=dx, dy=dy, z=z.astype(dt_), h=h.astype(dt_), u=u.astype(dt_), v=v.astype(dt_),
               n_shallow=man[0].astype(dt_), n_deep=man[1].astype(dt_), d_shallow=man[2].astype(dt_),
               d_deep=man[3].astype(dt_), qbdy0=q[0].astype(dt_), qbdy1=q[1].astype(dt_), hbdy0=hb[0].astype(dt_),
               hbdy1=hb[1].astype(dt_), head_first=1, t_sub=t, dt=dt, step_duration=L)
    out.update(r)
    return out


def case_dudt_terms(prec):
    """One update_dUdt on a 23 x 17 mesh with coded-out cells and every further term: energy
    loss, infiltration (its capacity consumed in place), Smagorinsky eddy viscosity and a stage
    boundary on some cells (listed before the discharge), beside Manning roughness and the
    discharge boundary; momentum terms in the order eddy viscosity, roughness, energy loss."""
    nx, ny, dx, dy = 23, 17, 3.0, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=43, nan_cells=5)
    rng = np.random.default_rng(44)
    man = (rng.uniform(0.02, 0.05, (ny, nx)), rng.uniform(0.03, 0.3, (ny, nx)), np.full((ny, nx), 0.1),
           np.full((ny, nx), 0.3))
    q = (rng.uniform(0, 3e-5, (ny, nx)) * (rng.uniform(size=(ny, nx)) > 0.3), rng.uniform(0, 3e-5, (ny, nx)))
    eloss = (rng.uniform(0.0, 0.5, (ny, nx)), rng.uniform(0.0, 0.5, (ny, nx)))
    infil = (rng.uniform(0.0, 2e-5, (ny, nx)), rng.uniform(0.0, 2e-3, (ny, nx)))
    sel = rng.uniform(size=(ny, nx)) > 0.7
    zf = np.nan_to_num(z, nan=0.0)
    stage = (np.where(sel, zf + rng.uniform(-0.05, 0.2, (ny, nx)), np.nan), np.where(sel, zf + 0.03, np.nan))
    order = (3, 1, 2)
    t, dt, L = 7.5, 0.37, 60.0
    dt_ = np.float64 if prec == "f64" else np.float32
    r = refpin.dudt_terms(z, h, u, v, dx, dy, manning=man, eloss=eloss, infil=infil, eddy=("smagorinsky", 0.05, 0.5),
                          q=q, stage=stage, stage_first=True, order=order, time_now=t, timestep=dt, step_length=L,
                          precision=prec)
    out = dict(nx=nx, ny=ny, dx=dx, dy=dy, z=z.astype(dt_), h=h.astype(dt_), u=u.astype(dt_), v=v.astype(dt_),
               n_shallow=man[0].astype(dt_), n_deep=man[1].astype(dt_), d_shallow=man[2].astype(dt_),
               d_deep=man[3].astype(dt_), qbdy0=q[0].astype(dt_), qbdy1=q[1].astype(dt_),
               hbdy0=stage[0].astype(dt_), hbdy1=stage[1].astype(dt_), eloss_fx=eloss[0].astype(dt_),
               eloss_fy=eloss[1].astype(dt_), infil_rate=infil[0].astype(dt_), infil_cap0=infil[1].astype(dt_),
               mu_const=0.05, mu_smag=0.5, order=np.array(order), stage_first=1, t_sub=t, dt=dt, step_duration=L)
    out.update({k: a for k, a in r.items()})
    return out


def case_solve(prec, rk):
    """Two 30 s steps through RungeKuttaSolver::solve: 45 x 30 plane with bumps, 1 mm film,
    Manning roughness, uniform rain 2e-5 m/s, outflow strip on the lowest edge."""
    nx, ny, dx = 45, 30, 4.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=3)
    h = np.full((ny, nx), 1e-3)
    zero = np.zeros_like(h)
    man = (0.03, 0.05, 0.1, 0.3)
    rain = 2e-5
    edges = synth.lowest_edge(z)
    rh, ru, rv, n = refpin.solve(z, h, zero, zero, dx, manning=man, rain=([0.0, 1e6], [rain, rain]),
                                 head_edges=edges, rk_method=rk, end=60.0, step_length=30.0, initial_dt=1.0,
                                 precision=prec)
    dt_ = np.float64 if prec == "f64" else np.float32
    return dict(nx=nx, ny=ny, dx=dx, z=z.astype(dt_), h=h.astype(dt_), manning=np.array(man), rain=rain,
                edges=edges, rk_method=rk, end_time=60.0, step_duration=30.0, initial_dt=1.0, timesteps=n,
                h_new=rh, u_new=ru, v_new=rv)


def main():
    cases = [("ref_dudt_23x17_coded_out_f64", lambda: case_dudt("f64")),
             ("ref_dudt_23x17_coded_out_f32", lambda: case_dudt("f32")),
             ("ref_dudt_terms_23x17_f64", lambda: case_dudt_terms("f64")),
             ("ref_dudt_terms_23x17_f32", lambda: case_dudt_terms("f32")),
             ("ref_solve_45x30_classic_f64", lambda: case_solve("f64", "classic")),
             ("ref_solve_45x30_kutta3_f64", lambda: case_solve("f64", "kutta3")),
             ("ref_solve_45x30_classic_f32", lambda: case_solve("f32", "classic"))]
    only = sys.argv[1:]
    for name, fn in cases:
        if only and name not in only:
            continue
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **fn())
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
