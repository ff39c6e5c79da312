"""Eddy viscosity (constant, per-cell and Smagorinsky coefficients) in any position among the
momentum source terms: FP64 equals the oracle bit for bit per function and over whole steps,
in the tiled and column-sweep kernels and in a batch; FP32 stays within a millimetre."""
import numpy as np
import pytest

from mfcm_b200 import SaintVenantSolver, synth
from mfcm_b200.batch import SaintVenantBatch
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import wet_dry_state, forcing, first_diff

pytestmark = pytest.mark.gpu

KS = ["DHDT", "DUDT", "DVDT"]
ORDERS = [None, ["eddy viscosity", "manning", "energy loss"], ["energy loss", "eddy viscosity", "manning"]]


def _assert_same(g, o, name):
    d = first_diff(g, o)
    assert d is None, f"{name}: first mismatch at {d[0]}: gpu {d[1]!r} oracle {d[2]!r} ({d[3]} differ)"


def _eddy(b, mode, mu_field):
    if mode == "smagorinsky":
        b.set_eddy_viscosity("smagorinsky", mu_const=0.05, mu_smag=0.5)
    elif mode == "field":
        b.set_field("EDDY_MU", mu_field)
        b.set_eddy_viscosity("constant", mu=2.0)
    else:
        b.set_eddy_viscosity("constant", mu=0.7)


@pytest.mark.parametrize("mode", ["constant", "field", "smagorinsky"])
@pytest.mark.parametrize("order", ORDERS)
def test_stage_derivative_with_eddy_viscosity(mode, order):
    nx, ny, dx = 37, 21, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=7)
    rng = np.random.default_rng(3)
    fx, fy = rng.uniform(0.0, 0.5, (ny, nx)), rng.uniform(0.0, 0.5, (ny, nx))
    mu = rng.uniform(0.0, 3.0, (ny, nx))
    out = []
    for cls in (SaintVenantSolver, OracleSolver):
        b = cls(nx, ny, dx, rain_mode="physical")
        for name, a in (("Z", z), ("H", h), ("U", u), ("V", v), ("ELOSS_FX", fx), ("ELOSS_FY", fy)):
            b.set_field(name, a)
        b.set_manning(0.03, 0.05, 0.1, 0.3)
        _eddy(b, mode, mu)
        if order:
            b.set_source_order(order)
        b.set_forcing(forcing((2e-5, 1e-5)))
        b.eval_dudt(0, 7.5, 0.37)
        out.append({k: b.get_field(k) for k in KS})
    for k in KS:
        _assert_same(out[0][k], out[1][k], k)


def _catchment(nx, ny, dx):
    z = synth.plane_with_gaussians(nx, ny, dx, seed=3)
    rng = np.random.default_rng(2)
    h = rng.uniform(0.0, 0.05, (ny, nx))
    u = rng.normal(0.0, 0.3, (ny, nx))
    v = rng.normal(0.0, 0.3, (ny, nx))
    return z, h, u, v


@pytest.mark.parametrize("variant", [1, 3, 5, 8])
@pytest.mark.parametrize("mode", ["field", "smagorinsky"])
def test_steps_with_eddy_viscosity(variant, mode):
    """Three whole steps in the tiled (1, 3) and column-sweep (5, 8) kernels."""
    nx, ny, dx, L = 61, 43, 2.0, 10.0
    z, h, u, v = _catchment(nx, ny, dx)
    mu = np.random.default_rng(5).uniform(0.0, 2.0, (ny, nx))
    res = []
    for cls in (SaintVenantSolver, OracleSolver):
        b = cls(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical")
        if cls is SaintVenantSolver:
            b.set_kernel_variant(variant)
        for name, a in (("Z", z), ("H", h), ("U", u), ("V", v)):
            b.set_field(name, a)
        b.set_manning(0.03, 0.05, 0.1, 0.3)
        _eddy(b, mode, mu)
        b.set_source_order(["eddy viscosity", "manning"])
        for i in range(3):
            b.set_forcing(forcing((3e-5, 3e-5), head=(0.0, 0.0), edges=2))
            b.advance()
        res.append(({k: b.get_field(k) for k in ("H", "U", "V")}, b.stats()))
    for k in ("H", "U", "V"):
        _assert_same(res[0][0][k], res[1][0][k], k)
    assert res[0][1]["accepted"] == res[1][1]["accepted"] > 0


def test_batch_member_with_eddy_viscosity_equals_its_solo_run():
    nx, ny, dx, L = 40, 24, 2.0, 10.0
    z, h, u, v = _catchment(nx, ny, dx)
    batch = SaintVenantBatch("f64")
    plain = batch.add(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical")   # without the term
    m = batch.add(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical")
    s = SaintVenantSolver(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical")
    for x in (plain, m, s):
        for name, a in (("Z", z), ("H", h), ("U", u), ("V", v)):
            x.set_field(name, a)
    for x in (m, s):
        x.set_eddy_viscosity("smagorinsky")
    for i in range(2):
        for x in (plain, m, s):
            x.set_forcing(forcing((2e-5, 2e-5), head=(0.0, 0.0), edges=2))
        batch.advance()
        s.advance()
    for k in ("H", "U", "V"):
        _assert_same(m.get_field(k), s.get_field(k), k)
    assert not np.array_equal(plain.get_field("U"), m.get_field("U"))
    batch.close()
    s.close()


def _gentle(nx, ny, dx):
    """Deep water over a gently sloping bed with smooth waves and currents: no fronts, so the
    FP64 scheme itself is insensitive to rounding here (on thin films and moving fronts it moves
    by millimetres under a 1e-7 perturbation, with or without eddy viscosity)."""
    y, x = np.mgrid[0:ny, 0:nx] * dx
    z = 0.002 * x
    h = 1.0 + 0.02 * np.sin(x / 17.0) * np.cos(y / 13.0)
    u = 0.1 * np.sin(y / 11.0)
    v = 0.1 * np.cos(x / 9.0)
    return z, h, u, v


@pytest.mark.parametrize("precision", ["f32", "f32_datum64"])
def test_eddy_viscosity_in_fp32(precision):
    nx, ny, dx, L = 64, 40, 2.0, 10.0
    z, h, u, v = _gentle(nx, ny, dx)
    out = {}
    for prec, eddy in (("f64", True), (precision, True), (precision, False)):
        s = SaintVenantSolver(nx, ny, dx, precision=prec, cn_target=0.5, step_duration=L, rain_mode="physical")
        for name, a in (("Z", z), ("H", h), ("U", u), ("V", v)):
            s.set_field(name, a)
        if eddy:
            s.set_eddy_viscosity("smagorinsky")
        for i in range(3):
            s.set_forcing(forcing((3e-5, 3e-5)))
            s.advance()
        out[(prec, eddy)] = (s.get_field("H"), s.get_field("U"))
        s.close()
    for k in (0, 1):
        assert np.max(np.abs(out[(precision, True)][k] - out[("f64", True)][k])) <= 1e-3
    assert np.max(np.abs(out[(precision, True)][1] - out[(precision, False)][1])) > 1e-5   # the term acts
