"""The oracle against the reference's own code (CPU; needs the reference source tree).

oracle/ref_pin/build.py compiles the reference's hot-path sources -- its mesh, field and state
classes, the Minmod3 slope operator, the flux, temporal-derivative, Manning, discharge and head
kernels, the control-number reduction, the state arithmetic of the stage combination and the
RungeKuttaSolver / TypedTemporalScheme step loop with the named tableaux -- against a host-only
SYCL stand-in. Every check here is bit for bit, in FP64 and in FP32 (the reference's shipped
precision, whose times are FP32 too). Without the reference tree the tests skip; the golden
fixtures made from it (tests/golden/make_ref_golden.py) carry the same checks everywhere.
"""
import numpy as np
import pytest

from mfcm_b200 import synth, solve, Forcing, TimeSeries, RK_METHODS, RAIN_FIELDS, HEAD_FIELDS, STAGE_FIELDS
from oracle.ref_pin import refpin
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import wet_dry_state, setup, first_diff

pytestmark = pytest.mark.skipif(not refpin.available(), reason="reference source tree not present")

PRECISIONS = ["f64", "f32"]


def assert_same(a, b, what):
    d = first_diff(np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64))
    assert d is None, f"{what}: first mismatch at {d[0]}: reference {d[1]!r} oracle {d[2]!r} ({d[3]} differ)"


def boundary_fields(nx, ny, seed):
    rng = np.random.default_rng(seed)
    ns = rng.uniform(0.02, 0.05, (ny, nx))
    nd = rng.uniform(0.03, 0.3, (ny, nx))
    ds = np.full((ny, nx), 0.1)
    dd = np.full((ny, nx), 0.3)
    q0 = rng.uniform(0, 3e-5, (ny, nx)) * (rng.uniform(size=(ny, nx)) > 0.3)
    q1 = rng.uniform(0, 3e-5, (ny, nx))
    hb0 = np.where(rng.uniform(size=(ny, nx)) > 0.8, rng.uniform(0, 0.1, (ny, nx)), np.nan)
    hb1 = np.where(np.isnan(hb0), np.nan, 0.02)
    return (ns, nd, ds, dd), (q0, q1), (hb0, hb1)


def oracle_dudt(prec, nx, ny, dx, dy, z, h, u, v, man, q, hb, head_first, rain_mode, t, dt, L):
    o = OracleSolver(nx, ny, dx, dy, precision=prec, rain_mode=rain_mode, step_duration=L, head_first=head_first)
    setup(o, z, h, u, v)
    f = Forcing()
    f.rain_kind, f.head_kind = RAIN_FIELDS, HEAD_FIELDS
    o.set_forcing(f)  # per-cell boundary values are uploaded after the forcing
    for name, a in zip(("N_SHALLOW", "N_DEEP", "D_SHALLOW", "D_DEEP", "QBDY0", "QBDY1", "HBDY0", "HBDY1"),
                       man + q + hb):
        o.set_field(name, a)
    o.eval_dudt(0, t, dt)
    return o


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("shape,dxy,nan_cells,head_first", [
    ((23, 17), (3.0, 3.0), 0, False), ((23, 17), (3.0, 3.0), 7, True), ((8, 8), (2.0, 5.0), 0, False),
    ((1, 9), (1.5, 1.5), 0, False), ((9, 1), (1.5, 1.5), 0, True), ((40, 3), (0.5, 0.25), 4, False)])
def test_stage_derivative_matches_reference_kernels(prec, shape, dxy, nan_cells, head_first):
    """Slopes, bed slopes, face fluxes and branches, dU/dt with Manning roughness, discharge
    and head boundaries: every field of one update_dUdt."""
    nx, ny = shape
    dx, dy = dxy
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=nx * 7 + ny, nan_cells=nan_cells)
    man, q, hb = boundary_fields(nx, ny, seed=nx + ny)
    t, dt, L = 7.5, 0.37, 60.0
    ref = refpin.dudt(z, h, u, v, dx, dy, manning=man, q=q, head=hb, head_first=head_first, time_now=t, timestep=dt,
                      step_length=L, precision=prec)
    o = oracle_dudt(prec, nx, ny, dx, dy, z, h, u, v, man, q, hb, head_first, "reference", t, dt, L)
    for name, a in ref.items():
        assert_same(a, o.get_field(name), name)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_rain_clamp_on_dry_cells(prec):
    """The discharge clamp h - q dt <= 0 => q = -h / dt, which drains dry and nearly dry cells."""
    nx, ny, dx = 16, 12, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=2)
    h = h * (np.arange(nx * ny).reshape(ny, nx) % 3 == 0)  # many dry cells
    man, q, hb = boundary_fields(nx, ny, seed=9)
    q = (np.full((ny, nx), 2e-5), np.full((ny, nx), 3e-5))
    ref = refpin.dudt(z, h, u, v, dx, q=q, time_now=10.0, timestep=0.5, step_length=30.0, precision=prec)
    o = OracleSolver(nx, ny, dx, precision=prec, rain_mode="reference", step_duration=30.0, manning=False)
    setup(o, z, h, u, v)
    f = Forcing()
    f.rain_kind = RAIN_FIELDS
    o.set_forcing(f)
    o.set_field("QBDY0", q[0])
    o.set_field("QBDY1", q[1])
    o.eval_dudt(0, 10.0, 0.5)
    for name in ("DHDT", "DUDT", "DVDT"):
        assert_same(ref[name], o.get_field(name), name)


@pytest.mark.parametrize("prec", PRECISIONS)
def test_control_number_matches_reference_reduction(prec):
    nx, ny, dx = 31, 19, 2.5
    _, h, u, v = wet_dry_state(nx, ny, dx, seed=4)
    o = OracleSolver(nx, ny, dx, precision=prec, cn_target=1.0)
    z = np.zeros_like(h)
    setup(o, z, h, u, v)
    cn, _, _ = o.do_timestep(0.0, 0.2)
    N = o.nstages
    hn, un, vn = (o.get_field(100 + 3 * N + k) for k in range(3))
    ref = refpin.control_number(hn, un, vn, dx, timestep=np.float32(0.2) if prec == "f32" else 0.2, precision=prec)
    assert float(ref) == cn


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("rk", RK_METHODS)
def test_stage_combination_matches_reference_state_arithmetic(prec, rk):
    """Every stage input Y_s and U_[N] of one timestep from the oracle's own k's, recombined by
    the reference's state operators in update_y's order."""
    from mfcm_b200._abi import RK_STAGES
    nx, ny, dx = 13, 11, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=8)
    o = OracleSolver(nx, ny, dx, precision=prec, rk_method=rk, cn_target=1.0)
    setup(o, z, h, u, v)
    dt = 0.05
    o.do_timestep(0.0, dt)
    N = RK_STAGES[RK_METHODS.index(rk)]
    tab = TABLEAUX[rk]
    U0 = np.stack([o.get_field(100 + k) for k in range(3)])
    ks = [np.stack([o.get_field(200 + 3 * j + k) for k in range(3)]) for j in range(N)]
    tdt = float(np.float32(dt)) if prec == "f32" else dt
    for s in range(1, N + 1):
        coefs = tab[s][1:s + 1]  # a(s+1, 1..s); for s = N the b row
        y = refpin.update_y(U0, ks[:s], coefs, tdt, precision=prec)
        for k in range(3):
            assert_same(y[k], o.get_field(100 + 3 * s + k), f"stage {s} field {k}")


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("rk", RK_METHODS)
def test_whole_solves_match_reference_step_loop(prec, rk):
    """Two 30 s steps through the reference's RungeKuttaSolver::solve (its tableau table,
    do_timestep and step(), control-number target 1.0 as it hard-codes) with Manning roughness,
    rain and an outflow strip: the number of timesteps and the final state."""
    nx, ny, dx = 45, 30, 4.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=3)
    h = np.full((ny, nx), 1e-3)
    zero = np.zeros_like(h)
    rain = ([0.0, 1e6], [2e-5, 2e-5])
    edges = synth.lowest_edge(z)
    man = (0.03, 0.05, 0.1, 0.3)
    rh, ru, rv, nts = refpin.solve(z, h, zero, zero, dx, manning=man, rain=rain, head_edges=edges, rk_method=rk,
                                   end=60.0, step_length=30.0, initial_dt=1.0, precision=prec)
    o = OracleSolver(nx, ny, dx, precision=prec, rk_method=rk, cn_target=1.0, rain_mode="reference",
                     step_duration=30.0, initial_dt=1.0)
    setup(o, z, h, zero, zero, n=man)
    st = solve(o, 0.0, 60.0, rain=TimeSeries(*rain), head=0.0, head_edges=edges)
    assert nts == sum(s["accepted"] + s["repeated"] for s in st)
    for name, a in (("H", rh), ("U", ru), ("V", rv)):
        assert_same(a, o.get_field(name), name)


# the named tableaux as (c_i, a_i1..) rows, last row (0, b_1..b_N), RungeKutta.cpp:54-115
TABLEAUX = {
    "euler": [[0.0], [0.0, 1.0]],
    "midpoint": [[0.0], [0.5, 0.5], [0.0, 0.0, 1.0]],
    "heun2": [[0.0], [1.0, 1.0], [0.0, 0.5, 0.5]],
    "ralston2": [[0.0], [2.0 / 3.0, 2.0 / 3.0], [0.0, 0.25, 0.75]],
    "kutta3": [[0.0], [0.5, 0.5], [1.0, -1.0, 2.0], [0.0, 1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0]],
    "heun3": [[0.0], [1.0 / 3.0, 1.0 / 3.0], [2.0 / 3.0, 0.0, 2.0 / 3.0], [0.0, 0.25, 0.0, 0.75]],
    "wray3": [[0.0], [8.0 / 15.0, 8.0 / 15.0], [2.0 / 3.0, 0.25, 5.0 / 12.0], [0.0, 0.25, 0.0, 0.75]],
    "ralston3": [[0.0], [0.5, 0.5], [0.75, 0.0, 0.75], [0.0, 2.0 / 9.0, 1.0 / 3.0, 4.0 / 9.0]],
    "ssprk3": [[0.0], [1.0, 1.0], [0.5, 0.25, 0.25], [0.0, 1.0 / 6.0, 1.0 / 6.0, 2.0 / 3.0]],
    "classic": [[0.0], [0.5, 0.5], [0.5, 0.0, 0.5], [1.0, 0.0, 0.0, 1.0], [0.0, 1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]],
    "ralston4": [[0.0], [0.4, 0.4], [0.45573725, 0.29697761, 0.15875964], [1.0, 0.21810040, -3.05096516, 3.83286476],
                 [0.0, 0.17476028, -0.55148066, 1.20553560, 0.17118478]],
    "3/8rule": [[0.0], [1.0 / 3.0, 1.0 / 3.0], [2.0 / 3.0, -1.0 / 3.0, 1.0], [1.0, 1.0, -1.0, 1.0],
                [0.0, 1.0 / 8.0, 3.0 / 8.0, 3.0 / 8.0, 1.0 / 8.0]],
}


TERM_NAMES = {1: "manning", 2: "energy loss", 3: "eddy viscosity"}


def _oracle_terms(prec, nx, ny, dx, dy, z, h, u, v, man, eloss, infil, eddy, q, stage, stage_first, order, t, dt, L):
    o = OracleSolver(nx, ny, dx, dy, precision=prec, rain_mode="reference", step_duration=L, head_first=stage_first,
                     manning=man is not None)
    for name, a in (("Z", z), ("H", h), ("U", u), ("V", v)):
        o.set_field(name, a)
    f = Forcing()
    f.rain_kind = RAIN_FIELDS if q else 0
    f.head_kind = STAGE_FIELDS if stage else 0
    o.set_forcing(f)  # per-cell boundary values are uploaded after the forcing
    fields = []
    if man:
        fields += list(zip(("N_SHALLOW", "N_DEEP", "D_SHALLOW", "D_DEEP"), man))
    if q:
        fields += [("QBDY0", q[0]), ("QBDY1", q[1])]
    if stage:
        fields += [("HBDY0", stage[0]), ("HBDY1", stage[1])]
    if eloss:
        fields += [("ELOSS_FX", eloss[0]), ("ELOSS_FY", eloss[1])]
    if infil:
        fields += [("INFIL_RATE", infil[0]), ("INFIL_CAP", infil[1])]
    for name, a in fields:
        o.set_field(name, a)
    if eddy and eddy[0] == "field":
        o.set_eddy_viscosity("constant", mu=0.7)
        o.set_field("EDDY_MU", eddy[1])
    elif eddy:
        o.set_eddy_viscosity("smagorinsky", mu_const=eddy[1], mu_smag=eddy[2])
    o.set_source_order([TERM_NAMES[k] for k in order])
    o.eval_dudt(0, t, dt)
    return o


@pytest.mark.parametrize("prec", PRECISIONS)
@pytest.mark.parametrize("shape,dxy,nan_cells,eddy_mode,order,stage_first", [
    ((23, 17), (3.0, 3.0), 0, "smagorinsky", (1, 2, 3), False),
    ((23, 17), (3.0, 3.0), 6, "field", (3, 1, 2), True),
    ((19, 12), (2.0, 5.0), 0, "smagorinsky", (2, 3, 1), False),
    ((1, 9), (1.5, 1.5), 0, "field", (2, 1, 3), True),
    ((9, 1), (1.5, 1.5), 0, "smagorinsky", (3, 2, 1), False),
    ((40, 3), (0.5, 0.25), 4, "smagorinsky", (1, 3, 2), True)])
def test_further_terms_match_reference_kernels(prec, shape, dxy, nan_cells, eddy_mode, order, stage_first):
    """dU/dt with energy loss, infiltration (and its capacity, consumed in place), eddy
    viscosity (a coefficient field or the Smagorinsky coefficient) and a stage boundary, beside
    Manning roughness and the discharge boundary, in the configured order of the momentum terms:
    the reference's EnergyLoss, Infiltration, EddyViscosity, SmagorinskyCoefficient and
    StageBoundary kernels against the oracle."""
    nx, ny = shape
    dx, dy = dxy
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=nx * 5 + ny, nan_cells=nan_cells)
    man, q, _ = boundary_fields(nx, ny, seed=nx + ny + 1)
    rng = np.random.default_rng(nx * ny)
    eloss = (rng.uniform(0.0, 0.5, (ny, nx)), rng.uniform(0.0, 0.5, (ny, nx)))
    infil = (rng.uniform(0.0, 2e-5, (ny, nx)), rng.uniform(0.0, 2e-3, (ny, nx)) * (rng.uniform(size=(ny, nx)) > 0.2))
    eddy = ("field", rng.uniform(0.0, 2.0, (ny, nx))) if eddy_mode == "field" else ("smagorinsky", 0.05, 0.5)
    sel = rng.uniform(size=(ny, nx)) > 0.7
    zf = np.nan_to_num(z, nan=0.0)
    stage = (np.where(sel, zf + rng.uniform(-0.05, 0.2, (ny, nx)), np.nan), np.where(sel, zf + 0.03, np.nan))
    t, dt, L = 7.5, 0.37, 60.0
    ref = refpin.dudt_terms(z, h, u, v, dx, dy, manning=man, eloss=eloss, infil=infil, eddy=eddy, q=q, stage=stage,
                            stage_first=stage_first, order=order, time_now=t, timestep=dt, step_length=L,
                            precision=prec)
    o = _oracle_terms(prec, nx, ny, dx, dy, z, h, u, v, man, eloss, infil, eddy, q, stage, stage_first, order, t, dt, L)
    for name, a in ref.items():
        assert_same(a, o.get_field(name), name)


def test_num_steps_matches_reference():
    """TimeParameters::num_steps: whole steps within 1e-6 s of the duration count as whole, any
    other remainder adds a step; the package's restatement (used by solve() and the decks)."""
    from mfcm_b200 import num_steps
    rng = np.random.default_rng(3)
    cases = [(0.0, 3600.0, 60.0), (0.0, 3600.0000001, 60.0), (0.0, 3600.000002, 60.0), (0.0, 3601.0, 60.0),
             (0.0, 59.9999995, 60.0), (10.0, 70.0, 60.0), (0.0, 0.3, 0.1), (0.0, 1.0, 0.1), (0.0, 7200.0, 7.0),
             (5.5, 5.5, 60.0), (0.0, 1e9, 60.0)]
    for _ in range(300):
        step = float(rng.choice([0.1, 1.0, 7.5, 30.0, 60.0, 600.0, 3600.0, 0.37]))
        k = int(rng.integers(0, 500))
        start = float(rng.choice([0.0, rng.uniform(0, 1e5)]))
        end = start + k * step + float(rng.choice([0.0, 1e-7, -1e-7, 2e-6, -2e-6, rng.uniform(0, step)]))
        cases.append((start, end, step))
    for start, end, step in cases:
        assert num_steps(start, end, step) == refpin.num_steps(start, end, step), (start, end, step)
