"""Parity of the CUDA path (through the C-ABI) with the CPU oracle, FP64 bit for bit.

Each reference kernel is checked on its own through sv_eval_dudt (slopes, face fluxes and
branches, dU/dt), then the fused path through whole timesteps and whole steps. Grids that are
not multiples of the CTA tile, strips, wet/dry fronts, coded-out (NaN bed) cells, every named
Runge-Kutta tableau and both boundary orders are covered."""
import numpy as np
import pytest

from mfcm_b200 import SaintVenantSolver, solve, EDGE_XMAX, EDGE_XMIN, EDGE_YMIN, EDGE_YMAX, RK_METHODS, synth
from oracle.sv_oracle_py import OracleSolver
from tests.scenarios import wet_dry_state, setup, rain_series, forcing, same, first_diff

pytestmark = pytest.mark.gpu

SLOPES = ["DHDX", "DUDX", "DVDX", "DHDY", "DUDY", "DVDY", "DZDX", "DZDY"]
FACES = ["FLUX_H", "FLUX_U", "FLUX_V", "FLUX_Z", "FLUX_BRANCH"]
KS = ["DHDT", "DUDT", "DVDT"]


def pair(nx, ny, dx, **kw):
    return SaintVenantSolver(nx, ny, dx, **kw), OracleSolver(nx, ny, dx, **kw)


def assert_same(g, o, what):
    d = first_diff(g, o)
    assert d is None, f"{what}: first mismatch at {d[0]}: gpu {d[1]!r} oracle {d[2]!r} ({d[3]} cells differ)"


@pytest.mark.parametrize("shape", [(17, 13), (8, 8), (1, 9), (9, 1), (40, 3), (33, 17)])
@pytest.mark.parametrize("nan_cells", [0, 5])
def test_per_function_parity(shape, nan_cells):
    nx, ny = shape
    if nan_cells and nx * ny < 20:
        pytest.skip("too small for coded-out cells")
    z, h, u, v = wet_dry_state(nx, ny, 3.0, seed=nx * 31 + ny, nan_cells=nan_cells)
    g, o = pair(nx, ny, 3.0, rain_mode="reference")
    for b in (g, o):
        setup(b, z, h, u, v, n=(0.03, 0.05, 0.1, 0.3))
        b.set_forcing(forcing((2e-5, 1e-5), head=(0.05, 0.0), edges=EDGE_XMAX | EDGE_YMIN))
        b.eval_dudt(0, 7.5, 0.37)
    for f in SLOPES + FACES + KS:
        assert_same(g.get_field(f), o.get_field(f), f)


@pytest.mark.parametrize("rk", RK_METHODS)
def test_one_timestep_every_tableau(rk):
    nx, ny, dx = 37, 21, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=7)
    g, o = pair(nx, ny, dx, rk_method=rk)
    N = g.nstages
    for b in (g, o):
        setup(b, z, h, u, v)
        b.set_forcing(forcing((3e-5, 3e-5), head=(0.0, 0.0), edges=EDGE_XMIN))
    rg = g.do_timestep(1.25, 0.05)
    ro = o.do_timestep(1.25, 0.05)
    assert rg[0] == ro[0] and rg[1] == ro[1] and rg[2] == ro[2], (rg, ro)
    for f in range(3):
        assert_same(g.get_field(100 + 3 * N + f), o.get_field(100 + 3 * N + f), f"U_[N] field {f}")


@pytest.mark.parametrize("rain_mode,head_first", [("reference", False), ("physical", False), ("physical", True)])
def test_steps_match(rain_mode, head_first):
    nx, ny, dx = 45, 30, 4.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=3)
    h = np.full((ny, nx), 1e-3)
    g, o = pair(nx, ny, dx, cn_target=0.5, rain_mode=rain_mode, head_first=head_first, step_duration=30.0)
    for b in (g, o):
        setup(b, z, h, np.zeros_like(h), np.zeros_like(h))
    rain = rain_series(50.0 * synth.MM_PER_H, stop=60.0)
    sg = solve(g, 0.0, 120.0, rain=rain, head=0.0, head_edges=synth.lowest_edge(z))
    so = solve(o, 0.0, 120.0, rain=rain, head=0.0, head_edges=synth.lowest_edge(z))
    for a, b in zip(sg, so):
        assert a["accepted"] == b["accepted"] and a["repeated"] == b["repeated"]
        assert abs(a["volume"] - b["volume"]) <= 1e-12 * abs(b["volume"])
        assert abs(a["rain_in"] - b["rain_in"]) <= 1e-12 * abs(b["rain_in"]) + 1e-300
        assert abs(a["outflow"] - b["outflow"]) <= 1e-12 * abs(b["outflow"]) + 1e-300
    for f in ("H", "U", "V"):
        assert_same(g.get_field(f), o.get_field(f), f)
    assert g.get_dt() == o.get_dt()


def test_fields_forcing_and_pattern():
    nx, ny, dx = 50, 34, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=11)
    rng = np.random.default_rng(5)
    pat = rng.uniform(0.5, 1.5, size=(ny, nx))
    nfield = rng.choice([0.02, 0.035, 0.05, 0.1], size=(ny, nx))
    g, o = pair(nx, ny, dx, rain_mode="physical", step_duration=20.0)
    for b in (g, o):
        setup(b, z, h, u, v, n_field=nfield)
        b.set_field("RAIN_PATTERN", pat)
        b.set_forcing(forcing((1e-5, 2e-5), rain_kind=3, head=(0.0, 0.0), edges=15))
        b.advance()
    for f in ("H", "U", "V"):
        assert_same(g.get_field(f), o.get_field(f), f)


def test_fp32_close_to_fp64_oracle():
    nx, ny, dx = 64, 48, 5.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=1)
    h = np.full((ny, nx), 1e-3)
    g = SaintVenantSolver(nx, ny, dx, precision="f32", cn_target=0.5, rain_mode="physical")
    o = OracleSolver(nx, ny, dx, cn_target=0.5, rain_mode="physical")
    for b in (g, o):
        setup(b, z, h, np.zeros_like(h), np.zeros_like(h))
    rain = rain_series(50.0 * synth.MM_PER_H, stop=600.0)
    solve(g, 0.0, 240.0, rain=rain, head=0.0, head_edges=synth.lowest_edge(z))
    solve(o, 0.0, 240.0, rain=rain, head=0.0, head_edges=synth.lowest_edge(z))
    err = np.max(np.abs(g.get_field("H") - o.get_field("H")))
    vg, vo = g.stats()["volume"], o.stats()["volume"]
    assert err <= 1e-3, err
    assert abs(vg - vo) <= 1e-6 * vo, (vg, vo)


@pytest.mark.parametrize("variant", range(4, 11))
@pytest.mark.parametrize("nan_cells", [0, 6])
def test_interior_strips_every_sweep_variant(variant, nan_cells):
    """Meshes large enough that most column-sweep strips are interior (their window away from
    the mesh edge and from coded-out cells): those strips run the interior kernel, the others
    the general one, and every field stays bit for bit the oracle's."""
    nx, ny = 231, 170
    z, h, u, v = wet_dry_state(nx, ny, 2.0, seed=variant + 31 * nan_cells, nan_cells=nan_cells)
    g, o = pair(nx, ny, 2.0, cn_target=0.5, step_duration=4.0, rain_mode="physical")
    g.set_kernel_variant(variant)
    for b in (g, o):
        setup(b, z, h, u, v, n=(0.03, 0.06, 0.1, 0.3))
        b.set_forcing(forcing((2e-5, 1e-5), head=(0.01, 0.0), edges=EDGE_XMIN | EDGE_YMAX))
    rg, ro = g.do_timestep(0.5, 0.02), o.do_timestep(0.5, 0.02)
    for f in range(3):
        assert_same(g.get_field(100 + 12 + f), o.get_field(100 + 12 + f), f"U_[N] field {f}")
    if nan_cells:
        return  # NaN beds make the step itself non-finite in the reference arithmetic
    assert rg == ro, (rg, ro)
    sg, so = g.advance(), o.advance()
    assert sg["accepted"] == so["accepted"] and sg["repeated"] == so["repeated"]
    for f in ("H", "U", "V"):
        assert_same(g.get_field(f), o.get_field(f), f)


@pytest.mark.parametrize("precision", ["f32", "f32_datum64"])
@pytest.mark.parametrize("variant", [4, 5, 9, 12, 13, 14, 15])
def test_fp32_interior_strips_close_to_fp64(precision, variant):
    """The FP32 interior kernel (no tangential finiteness tests) against the FP64 oracle."""
    nx, ny, dx = 200, 180, 5.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=4)
    h = np.full((ny, nx), 1e-3)
    g = SaintVenantSolver(nx, ny, dx, precision=precision, cn_target=0.5, rain_mode="physical", step_duration=60.0)
    g.set_kernel_variant(variant)
    o = OracleSolver(nx, ny, dx, cn_target=0.5, rain_mode="physical", step_duration=60.0)
    for b in (g, o):
        setup(b, z, h, np.zeros_like(h), np.zeros_like(h))
    rain = rain_series(50.0 * synth.MM_PER_H, stop=600.0)
    solve(g, 0.0, 120.0, rain=rain, head=0.0, head_edges=synth.lowest_edge(z))
    solve(o, 0.0, 120.0, rain=rain, head=0.0, head_edges=synth.lowest_edge(z))
    assert np.max(np.abs(g.get_field("H") - o.get_field("H"))) <= 1e-3
    sg, so = g.stats(), o.stats()
    # the FP32 run's own mass balance (initial + rain - outflow + wall flow) closes to 1e-6; its
    # volume differs from FP64's by what the slightly different flow let out through the outflow
    # strip, a few parts in a million after 120 s here
    v0 = float(h.sum()) * dx * dx
    closure = sg["volume"] - (v0 + sg["rain_in"] - sg["outflow"] + sg["wall_in"])
    assert abs(closure) <= 1e-6 * sg["volume"], (closure, sg)
    assert abs(sg["volume"] - so["volume"]) <= 1e-5 * so["volume"], (sg["volume"], so["volume"])


@pytest.mark.parametrize("variant", range(12))
@pytest.mark.parametrize("shape", [(61, 45), (29, 70), (3, 5)])
def test_every_kernel_variant(variant, shape):
    """All stage-kernel variants (tiled, column sweep at every tile height, and the split
    slopes-then-stage schedule) give the same bits as the oracle, including grids narrower than
    one warp strip."""
    nx, ny = shape
    z, h, u, v = wet_dry_state(nx, ny, 2.0, seed=nx + 7 * ny, nan_cells=3 if nx * ny > 50 else 0)
    g, o = pair(nx, ny, 2.0, cn_target=0.5, step_duration=5.0, rain_mode="physical")
    g.set_kernel_variant(variant)
    for b in (g, o):
        setup(b, z, h, u, v, n=(0.03, 0.06, 0.1, 0.3))
        b.set_forcing(forcing((2e-5, 1e-5), head=(0.01, 0.0), edges=EDGE_XMIN | EDGE_YMAX))
    rg, ro = g.do_timestep(0.5, 0.02), o.do_timestep(0.5, 0.02)
    assert (rg[0] == ro[0] or (rg[0] != rg[0] and ro[0] != ro[0])) and rg[1:] == ro[1:] or rg[2] != rg[2], (rg, ro)
    for f in range(3):
        assert_same(g.get_field(100 + 12 + f), o.get_field(100 + 12 + f), f"U_[N] field {f}")
    if nx * ny > 50:
        return  # NaN beds make the step itself non-finite in the reference arithmetic
    sg, so = g.advance(), o.advance()
    assert sg["accepted"] == so["accepted"] and sg["repeated"] == so["repeated"]
    for f in ("H", "U", "V"):
        assert_same(g.get_field(f), o.get_field(f), f)


@pytest.mark.parametrize("variant", [0, 4, 5, 6])
def test_variant_steps_no_nan(variant):
    nx, ny, dx = 70, 41, 3.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=9)
    h = np.full((ny, nx), 2e-3)
    g, o = pair(nx, ny, dx, cn_target=0.5, step_duration=15.0, rain_mode="physical")
    g.set_kernel_variant(variant)
    for b in (g, o):
        setup(b, z, h, np.zeros_like(h), np.zeros_like(h))
    rain = rain_series(80.0 * synth.MM_PER_H, stop=30.0)
    sg = solve(g, 0.0, 45.0, rain=rain, head=0.0, head_edges=EDGE_XMAX | EDGE_YMIN)
    so = solve(o, 0.0, 45.0, rain=rain, head=0.0, head_edges=EDGE_XMAX | EDGE_YMIN)
    for a, b in zip(sg, so):
        assert a["accepted"] == b["accepted"] and a["repeated"] == b["repeated"]
    for f in ("H", "U", "V"):
        assert_same(g.get_field(f), o.get_field(f), f)


def test_autotune_keeps_state_and_bits():
    nx, ny, dx = 300, 200, 2.0
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=21)
    g, o = pair(nx, ny, dx, cn_target=0.5, step_duration=2.0, rain_mode="physical")
    for b in (g, o):
        setup(b, z, h, u, v)
    before = g.get_field("H")
    best = g.autotune()
    assert 0 <= best < 12  # FP64 solvers never take the FP32-only variants 12-13
    assert same(before, g.get_field("H"))
    g.advance(); o.advance()
    for f in ("H", "U", "V"):
        assert_same(g.get_field(f), o.get_field(f), f)


@pytest.mark.parametrize("precision,tol", [("f64", 1e-12), ("f32", 1e-6), ("f32_datum64", 1e-6)])
def test_mass_balance_closure_and_tallies(precision, tol):
    """The FP64 tallies (rain in, outflow, flow through the walls) close the volume balance
    to rounding in every precision, and in FP64 match the oracle's."""
    nx, ny, dx = 45, 30, 4.0
    z = synth.plane_with_gaussians(nx, ny, dx, seed=3)
    res = []
    for cls in (SaintVenantSolver, OracleSolver):
        b = cls(nx, ny, dx, cn_target=0.5, step_duration=20.0, rain_mode="physical",
                **({"precision": precision} if cls is SaintVenantSolver else {}))
        setup(b, z, np.full((ny, nx), 1e-3), np.zeros((ny, nx)), np.zeros((ny, nx)))
        v0 = b.stats()["volume"]
        solve(b, 0.0, 60.0, rain=rain_series(50 * synth.MM_PER_H, stop=1e4), head=0.0, head_edges=EDGE_XMAX)
        s = b.stats()
        res.append((s, v0))
        if cls is SaintVenantSolver and precision != "f64":
            break
    s, v0 = res[0]
    closure = s["volume"] - (v0 + s["rain_in"] - s["outflow"] + s["wall_in"])
    assert abs(closure) <= tol * s["volume"], closure
    if precision == "f64":
        so = res[1][0]
        for k in ("rain_in", "outflow", "wall_in"):
            assert abs(s[k] - so[k]) <= 1e-12 * max(abs(so[k]), 1e-300), (k, s[k], so[k])


@pytest.mark.parametrize("precision", ["f32", "f32_datum64"])
@pytest.mark.parametrize("shape", [(232, 170), (231, 170), (290, 97), (58, 40)])
@pytest.mark.parametrize("eddy,nan_cells", [(False, 0), (True, 0), (False, 5)])
def test_fp32_two_cells_per_lane_matches_one_cell_sweep(precision, shape, eddy, nan_cells):
    """Variants 12-13 sweep pairs of interior strips with two cells per lane and 8-byte loads;
    the arithmetic per face and cell is the one-cell interior sweep's (variant 7: the same strip
    height and variant 12's register cap), so the fields after a timestep agree to FP32 rounding.
    Odd row lengths and meshes too narrow for a pair have no pairs, and variant 12 then gives
    variant 7's results bit for bit. Coded-out cells move strips out of pairs. The pairs' reductions (CFL, volume,
    tallies) are checked through the controller and the mass balance of a whole step."""
    nx, ny = shape
    z, h, u, v = wet_dry_state(nx, ny, 2.0, seed=nx + ny + nan_cells, nan_cells=nan_cells)
    out = {}
    for variant in (7, 12, 13, 14, 15):
        g = SaintVenantSolver(nx, ny, 2.0, precision=precision, cn_target=0.5, step_duration=3.0,
                              rain_mode="physical")
        g.set_kernel_variant(variant)
        setup(g, z, h, u, v, n=(0.03, 0.06, 0.1, 0.3))
        if eddy:
            g.set_eddy_viscosity("smagorinsky", mu=1.0, mu_const=0.05, mu_smag=0.5)
        g.set_forcing(forcing((2e-5, 1e-5), head=(0.01, 0.0), edges=EDGE_XMIN | EDGE_YMAX))
        v0 = g.stats()["volume"]
        cn, rep, nd = g.do_timestep(0.5, 0.02)
        fields = [g.get_field(100 + 12 + f) for f in range(3)]
        st = None
        if not nan_cells:  # coded-out beds make the step non-finite in the reference arithmetic
            g.accept()
            g.advance()
            st = g.stats()
        out[variant] = (cn, fields, st, v0)
        g.close()
    no_pairs = nx % 2 == 1 or nx < 2 * 28 + 32
    # variant 12 has variant 7's register cap, so without pairs it runs variant 7's kernels
    for single, pair_v in ((7, 12), (7, 13), (7, 14), (7, 15)):
        cn1, f1, s1, v0 = out[single]
        cn2, f2, s2, _ = out[pair_v]
        for a, b in zip(f1, f2):
            if no_pairs and pair_v == 12:
                assert np.array_equal(a, b, equal_nan=True)
            else:
                fin = np.isfinite(a)
                assert np.array_equal(fin, np.isfinite(b))
                np.testing.assert_allclose(b[fin], a[fin], rtol=2e-6, atol=2e-7)
        if nan_cells:
            continue
        assert abs(cn2 - cn1) <= 1e-5 * abs(cn1)
        # the pair kernel's tallies close its mass balance like the one-cell sweep's
        for st in (s1, s2):
            closure = st["volume"] - (v0 + st["rain_in"] - st["outflow"] + st["wall_in"])
            assert abs(closure) <= 1e-5 * abs(st["volume"]), (closure, st)


def test_fp32_only_variants_refused_by_fp64_solvers():
    g = SaintVenantSolver(64, 40, 2.0)
    for variant in (12, 13, 14, 15):
        with pytest.raises(Exception):
            g.set_kernel_variant(variant)
    g.close()
