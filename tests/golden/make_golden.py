"""Regenerate the golden fixtures of the oracle (the CPU restatement of the reference's
arithmetic). The reference itself ships no fixtures and cannot be built here, so these pin
the oracle against later edits and give the CUDA path committed vectors to match.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from mfcm_b200 import solve, synth, EDGE_XMAX, EDGE_YMIN, EDGE_XMIN  # noqa: E402
from oracle.sv_oracle_py import OracleSolver  # noqa: E402
from tests.scenarios import wet_dry_state, setup, forcing, rain_series  # noqa: E402

FIELDS_SLOPE = ["DHDX", "DUDX", "DVDX", "DHDY", "DUDY", "DVDY", "DZDX", "DZDY"]
FIELDS_FACE = ["FLUX_H", "FLUX_U", "FLUX_V", "FLUX_Z", "FLUX_BRANCH"]
FIELDS_K = ["DHDT", "DUDT", "DVDT"]


def case_dudt():
    nx, ny, dx = 17, 13, 3.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=nx * 31 + ny, nan_cells=5)
    o = OracleSolver(nx, ny, dx, rain_mode="reference")
    setup(o, z, h, u, v, n=(0.03, 0.05, 0.1, 0.3))
    o.set_forcing(forcing((2e-5, 1e-5), head=(0.05, 0.0), edges=EDGE_XMAX | EDGE_YMIN))
    o.eval_dudt(0, 7.5, 0.37)
    out = dict(nx=nx, ny=ny, dx=dx, z=z, h=h, u=u, v=v, manning=np.array([0.03, 0.05, 0.1, 0.3]),
               rain=np.array([2e-5, 1e-5]), head=np.array([0.05, 0.0]), edges=EDGE_XMAX | EDGE_YMIN,
               t_sub=7.5, dt=0.37)
    for f in FIELDS_SLOPE + FIELDS_FACE + FIELDS_K:
        out[f] = o.get_field(f)
    return out


def case_timestep():
    nx, ny, dx = 37, 21, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=7)
    o = OracleSolver(nx, ny, dx)
    setup(o, z, h, u, v)
    o.set_forcing(forcing((3e-5, 3e-5), head=(0.0, 0.0), edges=EDGE_XMIN))
    cn, rep, nd = o.do_timestep(1.25, 0.05)
    return dict(nx=nx, ny=ny, dx=dx, z=z, h=h, u=u, v=v, rain=np.array([3e-5, 3e-5]), edges=EDGE_XMIN,
                t_local=1.25, dt=0.05, cn=cn, repeat=int(rep), new_dt=nd,
                h_new=o.get_field(112), u_new=o.get_field(113), v_new=o.get_field(114))


def case_steps():
    nx, ny, dx = 45, 30, 4.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=3)
    h = np.full((ny, nx), 1e-3)
    o = OracleSolver(nx, ny, dx, cn_target=0.5, rain_mode="physical", step_duration=30.0)
    setup(o, z, h, np.zeros_like(h), np.zeros_like(h))
    edges = synth.lowest_edge(z)
    per = solve(o, 0.0, 120.0, rain=rain_series(50.0 * synth.MM_PER_H, stop=60.0), head=0.0, head_edges=edges)
    s = o.stats()
    return dict(nx=nx, ny=ny, dx=dx, z=z, h=h, edges=edges, rain_rate=50.0 * synth.MM_PER_H, rain_stop=60.0,
                end_time=120.0, step_duration=30.0, accepted=np.array([p["accepted"] for p in per]),
                repeated=np.array([p["repeated"] for p in per]), h_new=o.get_field("H"), u_new=o.get_field("U"),
                v_new=o.get_field("V"), volume=s["volume"], rain_in=s["rain_in"], outflow=s["outflow"],
                dt=o.get_dt())


def main():
    for name, fn in (("dudt_17x13_coded_out", case_dudt), ("timestep_37x21_classic", case_timestep),
                     ("steps_45x30_rain_outflow", case_steps)):
        path = os.path.join(HERE, name + ".npz")
        np.savez_compressed(path, **fn())
        print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
