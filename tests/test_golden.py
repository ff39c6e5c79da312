"""The committed golden fixtures (tests/golden/*.npz, made by tests/golden/make_golden.py from
the oracle) against the oracle on the CPU and against the CUDA path on the GPU, bit for bit."""
import os

import numpy as np
import pytest

from mfcm_b200 import solve, EDGE_XMAX, EDGE_YMIN
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import setup, forcing, rain_series, same

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
SLOPE = ["DHDX", "DUDX", "DVDX", "DHDY", "DUDY", "DVDY", "DZDX", "DZDY"]
FACE = ["FLUX_H", "FLUX_U", "FLUX_V", "FLUX_Z", "FLUX_BRANCH"]
KS = ["DHDT", "DUDT", "DVDT"]


def load(name):
    return dict(np.load(os.path.join(GOLD, name + ".npz")))


def backend(kind, nx, ny, dx, **kw):
    if kind == "gpu":
        from mfcm_b200 import SaintVenantSolver
        return SaintVenantSolver(nx, ny, dx, **kw)
    return OracleSolver(nx, ny, dx, **kw)


def check_dudt(kind):
    g = load("dudt_17x13_coded_out")
    b = backend(kind, int(g["nx"]), int(g["ny"]), float(g["dx"]), rain_mode="reference")
    setup(b, g["z"], g["h"], g["u"], g["v"], n=tuple(g["manning"]))
    b.set_forcing(forcing(tuple(g["rain"]), head=tuple(g["head"]), edges=int(g["edges"])))
    b.eval_dudt(0, float(g["t_sub"]), float(g["dt"]))
    for f in SLOPE + FACE + KS:
        assert same(b.get_field(f), g[f]), f


def check_timestep(kind):
    g = load("timestep_37x21_classic")
    b = backend(kind, int(g["nx"]), int(g["ny"]), float(g["dx"]))
    setup(b, g["z"], g["h"], g["u"], g["v"])
    b.set_forcing(forcing(tuple(g["rain"]), head=(0.0, 0.0), edges=int(g["edges"])))
    cn, rep, nd = b.do_timestep(float(g["t_local"]), float(g["dt"]))
    assert (cn, int(rep), nd) == (float(g["cn"]), int(g["repeat"]), float(g["new_dt"]))
    for k, f in enumerate(("h_new", "u_new", "v_new")):
        assert same(b.get_field(112 + k), g[f]), f


def check_steps(kind):
    g = load("steps_45x30_rain_outflow")
    nx, ny = int(g["nx"]), int(g["ny"])
    b = backend(kind, nx, ny, float(g["dx"]), cn_target=0.5, rain_mode="physical",
                step_duration=float(g["step_duration"]))
    setup(b, g["z"], g["h"], np.zeros((ny, nx)), np.zeros((ny, nx)))
    per = solve(b, 0.0, float(g["end_time"]), rain=rain_series(float(g["rain_rate"]), stop=float(g["rain_stop"])),
                head=0.0, head_edges=int(g["edges"]))
    assert [p["accepted"] for p in per] == list(g["accepted"])
    assert [p["repeated"] for p in per] == list(g["repeated"])
    for f, n in (("H", "h_new"), ("U", "u_new"), ("V", "v_new")):
        assert same(b.get_field(f), g[n]), f
    s = b.stats()
    assert abs(s["volume"] - float(g["volume"])) <= 1e-12 * float(g["volume"])
    assert abs(s["rain_in"] - float(g["rain_in"])) <= 1e-12 * float(g["rain_in"])
    assert abs(s["outflow"] - float(g["outflow"])) <= 1e-12 * max(1e-300, float(g["outflow"]))
    assert b.get_dt() == float(g["dt"])


@pytest.mark.parametrize("check", [check_dudt, check_timestep, check_steps])
def test_oracle_matches_golden(check):
    check("cpu")


@pytest.mark.gpu
@pytest.mark.parametrize("check", [check_dudt, check_timestep, check_steps])
def test_cuda_path_matches_golden(check):
    check("gpu")
