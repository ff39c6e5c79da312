"""The C++ oracle against the independent numpy restatement of the same reference lines
(oracle/sv_oracle_np.py): slopes, face fluxes and branches, and dU/dt with roughness and both
boundaries must agree bit for bit (up to the sign of an exact zero), on wet/dry states with
coded-out cells, ragged and one-cell-wide grids, dx != dy, both rain clamps and both
boundary orders. No GPU is needed."""
import numpy as np
import pytest

from mfcm_b200 import EDGE_XMAX, EDGE_XMIN, EDGE_YMAX, EDGE_YMIN, STAGE_EDGES
from oracle import sv_oracle_np as onp
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import wet_dry_state, forcing, same, first_diff

SLOPES = {"DHDX": "dhdx", "DUDX": "dudx", "DVDX": "dvdx", "DHDY": "dhdy", "DUDY": "dudy", "DVDY": "dvdy",
          "DZDX": "dzdx", "DZDY": "dzdy"}
FACES = {"FLUX_H": "flux_h", "FLUX_U": "flux_u", "FLUX_V": "flux_v", "FLUX_Z": "flux_z",
         "FLUX_BRANCH": "flux_branch"}
KS = {"DHDT": "dhdt", "DUDT": "dudt", "DVDT": "dvdt"}


def _check(o, ref, fields):
    for name, key in fields.items():
        got = o.get_field(name)
        want = ref[key].reshape(got.shape)
        d = first_diff(got, want)
        assert d is None, f"{name}: first mismatch at {d[0]}: oracle {d[1]!r} numpy {d[2]!r} ({d[3]} differ)"


CASES = [  # nx, ny, dx, dy, nan cells, seed
    (17, 13, 3.0, 3.0, 0, 1),
    (33, 17, 2.0, 5.0, 6, 2),
    (1, 9, 3.0, 3.0, 0, 3),
    (9, 1, 3.0, 3.0, 0, 4),
    (40, 3, 0.5, 0.5, 4, 5),
    (24, 24, 4.0, 1.0, 10, 6),
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("rain_mode,head_first", [("reference", False), ("physical", False), ("physical", True)])
def test_oracle_matches_numpy_restatement(case, rain_mode, head_first):
    nx, ny, dx, dy, nan_cells, seed = case
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=seed, nan_cells=nan_cells if nx * ny >= 20 else 0)
    n = (0.03, 0.05, 0.1, 0.3)
    q = (2e-5, 1e-5)
    head, edges = (0.05, 0.0), EDGE_XMAX | EDGE_YMIN
    t_now, ts, L = 7.5, 0.37, 60.0
    o = OracleSolver(nx, ny, dx, dy, rain_mode=rain_mode, head_first=head_first, step_duration=L)
    o.set_field("Z", z)
    o.set_field("H", h)
    o.set_field("U", u)
    o.set_field("V", v)
    o.set_manning(*n)
    o.set_forcing(forcing(q, head=head, edges=edges))
    o.eval_dudt(0, t_now, ts)
    shape = (ny, nx)
    hb = onp.edge_strips(nx, ny, edges, *head)
    assert same(o.get_field("HBDY0"), hb[0]) and same(o.get_field("HBDY1"), hb[1])
    ref = onp.update_dudt(h, u, v, z, dx, dy, manning=tuple(np.full(shape, x) for x in n),
                          qbdy=(np.full(shape, q[0]), np.full(shape, q[1])), hbdy=hb, time_now=t_now, timestep=ts,
                          step_length=L, rain_mode=rain_mode, head_first=head_first)
    _check(o, ref, SLOPES)
    _check(o, ref, FACES)
    _check(o, ref, KS)


def test_numpy_restatement_sees_every_branch():
    """The wet/dry scenario drives all four flux branches (both step cases of branch 2)."""
    nx, ny, dx = 33, 17, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=2)
    ref = onp.update_dudt(h, u, v, z, dx, dx)
    assert {1.0, 2.25, 2.75, 3.0, 4.0} <= set(np.unique(ref["flux_branch"]).tolist())


def test_numpy_pow43_matches_the_shared_routine():
    from oracle.sv_oracle_py import pow43
    rng = np.random.default_rng(1)
    x = np.exp(rng.uniform(np.log(1e-9), np.log(1e4), 5000))
    assert np.array_equal(onp.pow43(x), np.array([pow43(t) for t in x]))


def test_mirror_in_y_is_not_a_symmetry_of_the_reference_slopes():
    """The y slope takes the north (row + 1) neighbour as its left operand, so dU/dy is
    minus the row-wise derivative: a linear ramp rising with the row index has a negative
    reference slope."""
    ny, nx = 6, 4
    f = np.tile(np.arange(ny, dtype=float)[:, None], (1, nx))
    s = onp.slope_y(f, 1.0)
    assert np.all(s[1:-1] == -1.0)


@pytest.mark.parametrize("method", ["classic", "ralston4", "3/8rule"])
@pytest.mark.parametrize("case", CASES[:2] + CASES[4:5])
def test_oracle_timestep_matches_numpy_restatement(method, case):
    """A whole timestep: every stage, the left-to-right stage combination, the control number
    and the dt controller."""
    nx, ny, dx, dy, nan_cells, seed = case
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=seed + 50, nan_cells=0)
    n = (0.03, 0.05, 0.1, 0.3)
    q = (2e-5, 3e-5)
    head, edges = (0.02, 0.01), EDGE_XMIN | EDGE_YMAX
    t0, dt, L, tgt = 4.0, 0.05, 30.0, 0.5
    o = OracleSolver(nx, ny, dx, dy, rk_method=method, cn_target=tgt, rain_mode="physical", step_duration=L)
    for name, a in (("Z", z), ("H", h), ("U", u), ("V", v)):
        o.set_field(name, a)
    o.set_manning(*n)
    o.set_forcing(forcing(q, head=head, edges=edges))
    cn, rep, nd = o.do_timestep(t0, dt)
    shape = (ny, nx)
    (hN, uN, vN), cn2, rep2, nd2 = onp.do_timestep(
        h, u, v, z, dx, dy, t0, dt, method=method, cn_target=tgt,
        manning=tuple(np.full(shape, x) for x in n), qbdy=(np.full(shape, q[0]), np.full(shape, q[1])),
        hbdy=onp.edge_strips(nx, ny, edges, *head), step_length=L, rain_mode="physical")
    assert cn == cn2 and bool(rep) == rep2 and nd == nd2, ((cn, rep, nd), (cn2, rep2, nd2))
    N = o.nstages
    for k, want in enumerate((hN, uN, vN)):
        got = o.get_field(100 + 3 * N + k)
        d = first_diff(got, want)
        assert d is None, f"U_[N] field {k}: first mismatch at {d[0]}: oracle {d[1]!r} numpy {d[2]!r}"


@pytest.mark.parametrize("case", CASES[:2] + CASES[5:])
@pytest.mark.parametrize("eloss_first", [False, True])
def test_oracle_source_terms_match_numpy(case, eloss_first):
    """Energy loss (either side of the roughness term), infiltration with its in-place
    capacity, and a stage boundary on edge strips, against the numpy restatement."""
    nx, ny, dx, dy, nan_cells, seed = case
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=seed + 11, nan_cells=0)
    rng = np.random.default_rng(seed)
    shape = (ny, nx)
    fx, fy = rng.uniform(0.0, 0.5, shape), rng.uniform(0.0, 0.5, shape)
    rate, cap = rng.uniform(0.0, 2e-3, shape), rng.uniform(0.0, 1e-3, shape)
    n = (0.03, 0.05, 0.1, 0.3)
    q = (2e-5, 1e-5)
    level, edges = (float(np.median(z)) + 0.05, float(np.median(z))), EDGE_XMAX | EDGE_YMIN
    t_now, ts, L = 7.5, 0.37, 60.0
    o = OracleSolver(nx, ny, dx, dy, rain_mode="physical", step_duration=L, eloss_first=eloss_first)
    for name, a in (("Z", z), ("H", h), ("U", u), ("V", v), ("ELOSS_FX", fx), ("ELOSS_FY", fy),
                    ("INFIL_RATE", rate), ("INFIL_CAP", cap)):
        o.set_field(name, a)
    o.set_manning(*n)
    f = forcing(q, head=level, edges=edges)
    f.head_kind = STAGE_EDGES
    o.set_forcing(f)
    o.eval_dudt(0, t_now, ts)
    ref = onp.update_dudt(h, u, v, z, dx, dy, manning=tuple(np.full(shape, x) for x in n),
                          qbdy=(np.full(shape, q[0]), np.full(shape, q[1])),
                          hbdy=onp.edge_strips(nx, ny, edges, *level), stage=True, time_now=t_now, timestep=ts,
                          step_length=L, rain_mode="physical", eloss=(fx, fy), eloss_first=eloss_first,
                          infil=(rate, cap))
    _check(o, ref, KS)
    assert same(o.get_field("INFIL_CAP"), ref["infil_cap"])


def test_infiltration_capacity_is_consumed_by_every_stage():
    nx, ny, dx, dy = 24, 18, 2.0, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=4)
    shape = (ny, nx)
    rate, cap = np.full(shape, 1e-3), np.full(shape, 5e-4)
    o = OracleSolver(nx, ny, dx, rain_mode="physical", cn_target=0.5)
    for name, a in (("Z", z), ("H", h), ("U", u), ("V", v), ("INFIL_RATE", rate), ("INFIL_CAP", cap)):
        o.set_field(name, a)
    cn, rep, nd = o.do_timestep(0.0, 0.2)
    out = {}
    (hN, uN, vN), cn2, rep2, nd2 = onp.do_timestep(h, u, v, z, dx, dy, 0.0, 0.2, cn_target=0.5,
                                                   manning=tuple(np.full(shape, x) for x in (0.03, 0.3, 0.1, 0.3)),
                                                   infil=(rate, cap), rain_mode="physical", terms_out=out)
    assert (cn, bool(rep), nd) == (cn2, rep2, nd2)
    assert same(o.get_field(100 + 3 * o.nstages), hN)
    assert same(o.get_field("INFIL_CAP"), out["infil"][1])
    # the four classic RK stages each took up to rate * dt = 2e-4 m: more than one stage's
    # worth is gone, and deep cells emptied their 5e-4 m capacity
    taken = cap - o.get_field("INFIL_CAP")
    assert taken.max() > 2e-4 and np.any(o.get_field("INFIL_CAP") == 0.0)


EDDY_ORDERS = [None, ["eddy viscosity", "manning", "energy loss"], ["energy loss", "eddy viscosity", "manning"]]


def _eddy_setup(o, mode, shape, rng):
    if mode == "smagorinsky":
        o.set_eddy_viscosity("smagorinsky", mu_const=0.05, mu_smag=0.5)
        return ("smagorinsky", 0.05, 0.5)
    if mode == "field":
        mu = rng.uniform(0.0, 3.0, shape)
        o.set_field("EDDY_MU", mu)
        o.set_eddy_viscosity("constant", mu=2.0)    # the field takes precedence
        return ("constant", mu)
    o.set_eddy_viscosity("constant", mu=0.7)
    return ("constant", 0.7)


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("mode", ["constant", "field", "smagorinsky"])
@pytest.mark.parametrize("order", EDDY_ORDERS)
def test_oracle_eddy_viscosity_matches_numpy(case, mode, order):
    """Eddy viscosity (constant, per-cell and Smagorinsky coefficients) in any position among
    the momentum terms, against the numpy restatement."""
    nx, ny, dx, dy, nan_cells, seed = case
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=seed + 3, nan_cells=nan_cells)   # coded-out cells too
    rng = np.random.default_rng(seed + 100)
    shape = (ny, nx)
    fx, fy = rng.uniform(0.0, 0.5, shape), rng.uniform(0.0, 0.5, shape)
    n = (0.03, 0.05, 0.1, 0.3)
    o = OracleSolver(nx, ny, dx, dy, rain_mode="physical")
    for name, a in (("Z", z), ("H", h), ("U", u), ("V", v), ("ELOSS_FX", fx), ("ELOSS_FY", fy)):
        o.set_field(name, a)
    o.set_manning(*n)
    eddy = _eddy_setup(o, mode, shape, rng)
    if order:
        o.set_source_order(order)
    o.eval_dudt(0, 7.5, 0.37)
    ref = onp.update_dudt(h, u, v, z, dx, dy, manning=tuple(np.full(shape, x) for x in n), time_now=7.5,
                          timestep=0.37, rain_mode="physical", eloss=(fx, fy), eddy=eddy, order=order)
    _check(o, ref, KS)
    base = onp.update_dudt(h, u, v, z, dx, dy, manning=tuple(np.full(shape, x) for x in n), time_now=7.5,
                           timestep=0.37, rain_mode="physical", eloss=(fx, fy))
    if nx > 2 and ny > 2:
        assert not same(ref["dudt"], base["dudt"])      # the term acts


def test_oracle_eddy_viscosity_steps_match_numpy():
    nx, ny, dx = 30, 22, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=21)
    shape = (ny, nx)
    o = OracleSolver(nx, ny, dx, rain_mode="physical", cn_target=0.5)
    for name, a in (("Z", z), ("H", h), ("U", u), ("V", v)):
        o.set_field(name, a)
    o.set_eddy_viscosity("smagorinsky", mu_const=0.05, mu_smag=0.5)
    o.set_source_order(["eddy viscosity", "manning"])
    cn, rep, nd = o.do_timestep(0.0, 0.2)
    (hN, uN, vN), cn2, rep2, nd2 = onp.do_timestep(
        h, u, v, z, dx, dx, 0.0, 0.2, cn_target=0.5, manning=tuple(np.full(shape, x) for x in (0.03, 0.3, 0.1, 0.3)),
        rain_mode="physical", eddy=("smagorinsky", 0.05, 0.5), order=["eddy viscosity", "manning"])
    assert (cn, bool(rep), nd) == (cn2, rep2, nd2)
    for k, a in zip((0, 1, 2), (hN, uN, vN)):
        assert same(o.get_field(100 + 3 * o.nstages + k), a)


def test_source_order_is_validated():
    o = OracleSolver(4, 4, 1.0)
    for bad in (["manning", "manning"],):
        with pytest.raises(Exception):
            o.set_source_order(bad)
    with pytest.raises(ValueError):
        o.set_eddy_viscosity("laminar")
