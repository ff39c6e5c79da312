"""CPU checks of the oracle (the CPU restatement of the reference's arithmetic) and of the
host-side logic. None of these needs a GPU."""
import math

import numpy as np
import pytest

from mfcm_b200 import TimeSeries, num_steps, solve, synth, EDGE_XMAX, RAIN_UNIFORM
from oracle.sv_oracle_py import OracleSolver, pow43, minmod3
from tests.scenarios import wet_dry_state, setup, forcing, same, rain_series

NAN = float("nan")


# ---------------------------------------------------------------- pow(x, 4/3) routine
def _pow43_np(x):
    """numpy restatement of sv_math::pow43 (same operation order, IEEE double)."""
    C = (-0.019273, 0.18161161, -0.63413856, 1.48409885)
    third = 1.0 / 3.0
    m, e = np.frexp(x)
    q = np.floor_divide(e, 3)
    r = e - 3 * q
    w = np.ldexp(m, r)
    y = ((C[0] * w + C[1]) * w + C[2]) * w + C[3]
    for _ in range(3):
        y3 = (y * y) * y
        y = y + (y * (1.0 - w * y3)) * third
    cb = (w * y) * y
    cb = cb - ((cb * cb) * cb - w) * ((y * y) * third)
    return x * np.ldexp(cb, q)


def test_pow43_matches_its_numpy_restatement_and_libm():
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.uniform(1e-3, 16, 4000), np.exp(rng.uniform(np.log(1e-7), np.log(1e3), 4000))])
    got = np.array([pow43(v) for v in x])
    assert np.array_equal(got, _pow43_np(x))
    lib = np.power(x, 4.0 / 3.0)
    assert np.max(np.abs(got - lib) / np.spacing(lib)) <= 12.0
    exact = np.power(x.astype(np.longdouble), np.longdouble(4) / np.longdouble(3))
    ulp = np.abs(got.astype(np.longdouble) - exact) / np.spacing(got).astype(np.longdouble)
    assert float(ulp.max()) <= 1.7


def test_pow43_special_values():
    assert math.isnan(pow43(NAN))
    assert pow43(0.0) == 0.0
    assert pow43(math.inf) == math.inf
    assert pow43(8.0) == 16.0


# ---------------------------------------------------------------- Minmod3
@pytest.mark.parametrize("args,expected", [
    ((1.0, 2.0, 2.0, 2.0, 4.0), 0.5),        # interior: min(2*0.5, 2*1, 0.75) = 0.75? see below
    ((4.0, 2.0, 2.0, 2.0, 1.0), -0.5),
    ((1.0, 2.0, 3.0, 2.0, 2.0), 0.0),        # extremum: opposite one-sided slopes
    ((2.0, 0.0, 2.0, 2.0, 3.0), 0.5),        # west edge (dx_l = 0): one-sided
    ((1.0, 2.0, 3.0, 0.0, 3.0), 1.0),        # east edge (dx_r = 0)
    ((5.0, 0.0, 5.0, 0.0, 5.0), 0.0),        # single cell: central = 0
])
def test_minmod3_known_answers(args, expected):
    ul, dxl, uc, dxr, ur = args
    # recompute the expected value from Minmod3.hpp:34-82 by hand for the interior cases
    if dxl > 0 and dxr > 0:
        lhs, rhs, c = 2 * (uc - ul) / dxl, 2 * (ur - uc) / dxr, (ur - ul) / (dxl + dxr)
        sgn = lambda v: (v > 0) - (v < 0)
        outer = 0.5 * (sgn(lhs) + sgn(rhs)) * min(abs(lhs), abs(rhs))
        expected = 0.5 * (sgn(outer) + sgn(c)) * min(abs(outer), abs(c))
    assert minmod3(*args) == expected


def test_minmod3_nan_rules():
    # NaN centre: both one-sided differences NaN -> the central difference is returned
    assert minmod3(1.0, 2.0, NAN, 2.0, 3.0) == (3.0 - 1.0) / 4.0
    # NaN left neighbour: outer = rhs, central NaN -> sign(outer)/2 * |outer| (sycl::min(x, NaN) = x)
    assert minmod3(NAN, 2.0, 1.0, 2.0, 2.0) == 0.5 * (2 * (2.0 - 1.0) / 2.0)


# ---------------------------------------------------------------- whole-solver properties
def _run_steps(openmp, steps=2):
    nx, ny, dx = 40, 28, 3.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=5)
    o = OracleSolver(nx, ny, dx, cn_target=0.5, step_duration=10.0, rain_mode="physical", openmp=openmp, threads=4)
    setup(o, z, np.full((ny, nx), 2e-3), np.zeros((ny, nx)), np.zeros((ny, nx)))
    solve(o, 0.0, 10.0 * steps, rain=rain_series(60 * synth.MM_PER_H, stop=15.0), head=0.0,
          head_edges=synth.lowest_edge(z))
    return [o.get_field(f) for f in ("H", "U", "V")], o.stats()


def test_serial_and_openmp_oracles_agree_bit_for_bit():
    a, sa = _run_steps(False)
    b, sb = _run_steps(True)
    for x, y in zip(a, b):
        assert same(x, y)
    assert sa["accepted"] == sb["accepted"] and sa["volume"] == sb["volume"]


def test_x_mirror_symmetry_of_depth_and_v_but_not_u():
    """Flipping the domain in x (and the sign of u) mirrors dh/dt and dv/dt exactly. dU/dt
    of u is not mirror-symmetric at one-sided (wet/dry) faces: branch 4 adds +g*h_p to the
    u-flux (FluxKernel.cpp:277-278) where branch 1 subtracts it (FluxKernel.cpp:218-219)."""
    nx, ny, dx = 33, 20, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=3)
    a = OracleSolver(nx, ny, dx, step_duration=5.0)
    b = OracleSolver(nx, ny, dx, step_duration=5.0)
    setup(a, z, h, u, v)
    setup(b, z[:, ::-1], h[:, ::-1], -u[:, ::-1], v[:, ::-1])
    a.eval_dudt(0, 0.0, 0.01)
    b.eval_dudt(0, 0.0, 0.01)
    assert same(a.get_field("DHDT"), b.get_field("DHDT")[:, ::-1])
    assert same(a.get_field("DVDT"), b.get_field("DVDT")[:, ::-1])
    br = a.get_field("FLUX_BRANCH")
    assert np.any((br == 3) | (br == 4))
    assert not same(a.get_field("DUDT"), -b.get_field("DUDT")[:, ::-1])


def test_dry_domain_without_rain_stays_dry():
    nx, ny = 16, 12
    o = OracleSolver(nx, ny, 5.0, step_duration=10.0)
    o.set_field("Z", synth.plane_with_gaussians(nx, ny, 5.0, seed=2))
    o.advance()
    assert np.all(o.get_field("H") == 0.0)


def test_reference_rain_on_dry_bed_adds_nothing_and_dt_becomes_infinite():
    """DischargeBoundarySourceTerm.cpp:62-64 turns positive rain on a dry cell into -h/dt = 0,
    and do_timestep's dt/cn with cn = 0 (RungeKutta.cpp:166) gives an infinite next dt."""
    nx, ny = 16, 12
    o = OracleSolver(nx, ny, 5.0, step_duration=60.0, rain_mode="reference")
    o.set_field("Z", synth.plane_with_gaussians(nx, ny, 5.0, seed=2))
    f = forcing((1e-5, 1e-5))
    o.set_forcing(f)
    o.advance()
    assert np.all(o.get_field("H") == 0.0)
    assert o.get_dt() == math.inf
    # the physical clamp lets the same rain in
    p = OracleSolver(nx, ny, 5.0, step_duration=60.0, rain_mode="physical")
    p.set_field("Z", synth.plane_with_gaussians(nx, ny, 5.0, seed=2))
    p.set_forcing(f)
    p.advance()
    assert p.stats()["volume"] > 0.0


def test_rain_tally_equals_the_volume_gain_when_no_face_carries_flux():
    """Flat bed, uniform still water, uniform rain: every face flux is zero, so the volume
    gained equals the FP64 rain tally to round-off."""
    nx, ny, dx = 24, 18, 2.0
    o = OracleSolver(nx, ny, dx, cn_target=0.5, step_duration=10.0, rain_mode="physical")
    setup(o, np.full((ny, nx), 3.0), np.full((ny, nx), 1e-2), np.zeros((ny, nx)), np.zeros((ny, nx)))
    v0 = o.stats()["volume"]
    solve(o, 0.0, 30.0, rain=rain_series(50 * synth.MM_PER_H, stop=15.0))
    s = o.stats()
    assert s["rain_in"] > 0 and s["outflow"] == 0.0
    assert abs(s["volume"] - v0 - s["rain_in"]) <= 1e-12 * s["volume"]


# ---------------------------------------------------------------- host logic
def test_time_series_linear_interpolation():
    ts = TimeSeries([0.0, 600.0, 600.001, 3600.0], [1.0, 1.0, 0.0, 0.0])
    assert ts.at(0.0) == 1.0 and ts.at(300.0) == 1.0
    assert ts.at(600.0005) == pytest.approx(0.5)
    assert ts.at(5000.0) == 0.0  # past the last knot: last segment extrapolated


def test_num_steps():
    assert num_steps(0.0, 3600.0, 60.0) == 60
    assert num_steps(0.0, 3600.0000001, 60.0) == 60
    assert num_steps(0.0, 3601.0, 60.0) == 61


def test_mass_balance_closes_with_the_wall_tally():
    """Volume = initial + rain in - outflow + wall flow, to rounding: the wall tally counts
    what the reference's y-walls let through (closed box, no outflow boundary) and what
    crosses the edge faces of head-boundary strips."""
    nx, ny, dx = 30, 24, 2.0
    for edges in (0, EDGE_XMAX):
        o = OracleSolver(nx, ny, dx, cn_target=0.5, step_duration=10.0, rain_mode="physical")
        setup(o, synth.plane_with_gaussians(nx, ny, dx, seed=8), np.full((ny, nx), 1e-3), np.zeros((ny, nx)),
              np.zeros((ny, nx)))
        v0 = o.stats()["volume"]
        solve(o, 0.0, 60.0, rain=rain_series(40 * synth.MM_PER_H, stop=1e4), head=0.0 if edges else None,
              head_edges=edges)
        s = o.stats()
        assert s["wall_in"] < 0.0                     # water left through the walls
        closure = s["volume"] - (v0 + s["rain_in"] - s["outflow"] + s["wall_in"])
        assert abs(closure) <= 1e-12 * s["volume"], closure
