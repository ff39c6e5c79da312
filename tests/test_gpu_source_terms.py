"""The further source and boundary terms of the reference: energy loss (either side of the
roughness term), infiltration with its capacity consumed at every stage evaluation, and the
stage boundary (water-level targets). FP64 must equal the oracle bit for bit, per function and
over whole steps, in every kernel variant and in a batch."""
import numpy as np
import pytest

from mfcm_b200 import SaintVenantSolver, solve, synth, EDGE_XMAX, EDGE_YMIN, STAGE_EDGES, STAGE_FIELDS
from mfcm_b200.batch import SaintVenantBatch
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import wet_dry_state, forcing, same, first_diff, rain_series

pytestmark = pytest.mark.gpu

KS = ["DHDT", "DUDT", "DVDT"]


def _fields(nx, ny, dx, seed):
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=seed)
    rng = np.random.default_rng(seed)
    shape = (ny, nx)
    extra = {"ELOSS_FX": rng.uniform(0.0, 0.5, shape), "ELOSS_FY": rng.uniform(0.0, 0.5, shape),
             "INFIL_RATE": rng.uniform(0.0, 2e-5, shape), "INFIL_CAP": rng.uniform(0.0, 2e-3, shape)}
    return z, h, u, v, extra


def _setup(b, z, h, u, v, extra):
    for name, a in (("Z", z), ("H", h), ("U", u), ("V", v)):
        b.set_field(name, a)
    for name, a in extra.items():
        b.set_field(name, a)
    b.set_manning(0.03, 0.05, 0.1, 0.3)


def _assert_same(g, o, name):
    d = first_diff(g, o)
    assert d is None, f"{name}: first mismatch at {d[0]}: gpu {d[1]!r} oracle {d[2]!r} ({d[3]} differ)"


@pytest.mark.parametrize("eloss_first", [False, True])
@pytest.mark.parametrize("shape", [(37, 21), (64, 9)])
def test_stage_derivative_with_every_term(eloss_first, shape):
    nx, ny = shape
    z, h, u, v, extra = _fields(nx, ny, 2.0, seed=nx + ny)
    level = (float(np.median(z)) + 0.05, float(np.median(z)))
    out = []
    for cls in (SaintVenantSolver, OracleSolver):
        b = cls(nx, ny, 2.0, rain_mode="physical", eloss_first=eloss_first)
        _setup(b, z, h, u, v, extra)
        f = forcing((2e-5, 1e-5), head=level, edges=EDGE_XMAX | EDGE_YMIN)
        f.head_kind = STAGE_EDGES
        b.set_forcing(f)
        b.eval_dudt(0, 7.5, 0.37)
        out.append({k: b.get_field(k) for k in KS + ["INFIL_CAP"]})
    for k in KS + ["INFIL_CAP"]:
        _assert_same(out[0][k], out[1][k], k)


@pytest.mark.parametrize("variant", [1, 5, 8])
def test_steps_with_every_term(variant):
    """Three whole steps: infiltration capacity, energy loss and a per-cell stage boundary,
    in the tiled and the column-sweep kernels."""
    nx, ny, dx, L = 45, 30, 4.0, 20.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=3)
    h = np.full((ny, nx), 2e-3)
    rng = np.random.default_rng(1)
    extra = {"ELOSS_FX": rng.uniform(0.0, 0.3, (ny, nx)), "ELOSS_FY": rng.uniform(0.0, 0.3, (ny, nx)),
             "INFIL_RATE": np.full((ny, nx), 5e-6), "INFIL_CAP": rng.uniform(0.0, 1e-3, (ny, nx))}
    l0 = np.full((ny, nx), np.nan)
    l0[:, -1] = z[:, -1] + 0.01                      # stage (water level) targets on the last column
    res = []
    for cls in (SaintVenantSolver, OracleSolver):
        b = cls(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical")
        if cls is SaintVenantSolver:
            b.set_kernel_variant(variant)
        _setup(b, z, h, np.zeros_like(h), np.zeros_like(h), extra)
        b.set_field("HBDY0", l0)
        b.set_field("HBDY1", l0)
        for i in range(3):
            f = forcing((3e-5, 3e-5))
            f.head_kind = STAGE_FIELDS
            b.set_forcing(f)
            b.advance()
        res.append(({k: b.get_field(k) for k in ("H", "U", "V", "INFIL_CAP")}, b.stats()))
    for k in ("H", "U", "V", "INFIL_CAP"):
        _assert_same(res[0][0][k], res[1][0][k], k)
    assert res[0][1]["accepted"] == res[1][1]["accepted"]
    assert res[0][1]["volume"] == res[1][1]["volume"]


def test_autotune_leaves_the_infiltration_capacity_alone():
    nx, ny = 64, 48
    z, h, u, v, extra = _fields(nx, ny, 2.0, seed=9)
    s = SaintVenantSolver(nx, ny, 2.0, rain_mode="physical")
    _setup(s, z, h, u, v, extra)
    before = s.get_field("INFIL_CAP")
    s.autotune()
    assert same(s.get_field("INFIL_CAP"), before)


def test_stage_boundary_on_a_high_bed_in_every_precision():
    """Stage targets are water levels: on a bed at 350 m the depth target is level - bed,
    which the datum path forms in FP64; all precisions agree within 1 mm."""
    nx, ny, dx = 96, 16, 1.0
    z = 350.0 + synth.plane_with_gaussians(nx, ny, dx, slope=0.01, n_bumps=0, seed=1)
    h = np.full((ny, nx), 0.05)
    out = {}
    for prec in ("f64", "f32", "f32_datum64"):
        s = SaintVenantSolver(nx, ny, dx, precision=prec, cn_target=0.5, step_duration=10.0, rain_mode="physical")
        s.set_field("Z", z)
        s.set_field("H", h)
        s.set_manning(0.03, 0.03, 0.1, 0.3)
        for k in range(3):
            f = forcing((0.0, 0.0), head=(float(z[0, -1]) + 0.02, float(z[0, -1]) + 0.02), edges=EDGE_XMAX)
            f.head_kind = STAGE_EDGES
            s.set_forcing(f)
            s.advance()
        out[prec] = s.get_field("H")
        s.close()
    assert abs(out["f64"][0, -1] - 0.02) < 5e-3        # the outlet column sits near the 2 cm target
    for prec in ("f32", "f32_datum64"):
        assert np.max(np.abs(out[prec] - out["f64"])) <= 1e-3, prec


def test_batch_member_with_source_terms_equals_its_solo_run():
    nx, ny, dx, L = 40, 24, 2.0, 10.0
    z, h, u, v, extra = _fields(nx, ny, dx, seed=5)
    b = SaintVenantBatch("f64")
    m = b.add(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical", eloss_first=True)
    _setup(m, z, h, u, v, extra)
    s = SaintVenantSolver(nx, ny, dx, cn_target=0.5, step_duration=L, rain_mode="physical", eloss_first=True)
    _setup(s, z, h, u, v, extra)
    for i in range(2):
        for x in (m, s):
            x.set_forcing(forcing((2e-5, 2e-5), head=(0.0, 0.0), edges=EDGE_XMAX))
        b.advance()
        s.advance()
    for k in ("H", "U", "V", "INFIL_CAP"):
        _assert_same(m.get_field(k), s.get_field(k), k)
    b.close()
