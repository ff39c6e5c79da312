"""Fields cross the interface in FP64 and are converted on the device: an FP32 solver returns
each value rounded once to FP32, NaN, infinities and signed zeros included, and the FP32
solver with tile datums stores its bed as FP32 offsets from per-32x8-tile FP64 datums (the
tile's lowest valid bed, rounded down to a multiple of 2^-10 m; 0 for a tile without one)."""
import numpy as np
import pytest

from mfcm_b200 import SaintVenantSolver

pytestmark = pytest.mark.gpu


def _special(shape, seed):
    rng = np.random.default_rng(seed)
    a = rng.normal(0.0, 100.0, shape) * 10.0 ** rng.integers(-40, 38, shape)
    flat = a.reshape(-1)
    flat[:8] = [np.nan, np.inf, -np.inf, -0.0, 0.0, 1e-45, 3.4028235e38, 1.0 + 2.0 ** -30]
    return a


def _bits_equal(a, b):
    a = np.asarray(a, np.float64).view(np.uint64)
    b = np.asarray(b, np.float64).view(np.uint64)
    nan = np.isnan(np.asarray(a).view(np.float64))
    return np.array_equal(nan, np.isnan(b.view(np.float64))) and np.array_equal(a[~nan], b[~nan])


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_field_round_trip(precision):
    nx, ny = 37, 23
    x = _special((ny, nx), 1)
    s = SaintVenantSolver(nx, ny, 1.0, precision=precision)
    for f in ("H", "U", "N_SHALLOW", "RAIN_PATTERN"):
        s.set_field(f, x)
        with np.errstate(over="ignore"):   # values beyond FP32 become infinities
            expect = x if precision == "f64" else x.astype(np.float32).astype(np.float64)
        assert _bits_equal(s.get_field(f), expect), f
    out = np.empty(nx * ny)
    s.get_field("H", out=out)
    with np.errstate(over="ignore"):
        assert _bits_equal(out.reshape(ny, nx), x if precision == "f64" else x.astype(np.float32))
    with pytest.raises(ValueError):
        s.get_field("H", out=np.empty(nx * ny, dtype=np.float32))
    s.close()


def _datum_restatement(z):
    ny, nx = z.shape
    tx, ty = (nx + 31) // 32, (ny + 7) // 8
    dat = np.zeros((ty, tx))
    for j in range(ty):
        for i in range(tx):
            t = z[j * 8:(j + 1) * 8, i * 32:(i + 1) * 32].ravel()
            t = t[~np.isnan(t)]
            dat[j, i] = np.floor(t.min() * 1024.0) / 1024.0 if t.size else 0.0
    full = np.repeat(np.repeat(dat, 8, axis=0), 32, axis=1)[:ny, :nx]
    off = (z - full).astype(np.float32)
    return full, off.astype(np.float64) + full


def test_datum_bed_on_a_ragged_mesh():
    nx, ny = 70, 21                       # partial datum tiles on the right and the top
    rng = np.random.default_rng(4)
    z = 350.0 + np.cumsum(rng.normal(0.0, 0.05, (ny, nx)), axis=1)
    z[3, 5] = np.nan                      # a coded-out cell
    z[8:16, 32:64] = np.nan               # a tile without a valid bed: datum 0
    z[0:8, 64:70] = 0.0                   # a tile whose minimum is a tie of -0.0 and 0.0
    z[2, 66] = -0.0
    s = SaintVenantSolver(nx, ny, 1.0, precision="f32_datum64")
    s.set_field("Z", z)
    got = s.get_field("Z")
    _, expect = _datum_restatement(z)
    assert _bits_equal(got, expect)
    assert np.max(np.abs(got[~np.isnan(z)] - z[~np.isnan(z)])) < 2.0 ** -16 * 400   # FP32 offsets
    s.close()


@pytest.mark.parametrize("precision", ["f64", "f32"])
def test_n_deep_shares_n_shallow_only_while_equal(precision):
    """A deep-water roughness field equal to the shallow one is read from one array; setting
    either field later leaves the other with its own values."""
    nx, ny = 40, 30
    rng = np.random.default_rng(8)
    a, b = rng.uniform(0.02, 0.06, (ny, nx)), rng.uniform(0.02, 0.06, (ny, nx))
    cast = (lambda x: x) if precision == "f64" else (lambda x: x.astype(np.float32).astype(np.float64))
    s = SaintVenantSolver(nx, ny, 1.0, precision=precision)
    s.set_field("N_SHALLOW", a)
    s.set_field("N_DEEP", a)                  # shared
    s.set_field("N_SHALLOW", b)               # n_deep keeps a
    assert _bits_equal(s.get_field("N_DEEP"), cast(a)) and _bits_equal(s.get_field("N_SHALLOW"), cast(b))
    s.set_field("N_DEEP", b)                  # shared again
    s.set_field("N_DEEP", a)                  # an array of its own
    assert _bits_equal(s.get_field("N_DEEP"), cast(a)) and _bits_equal(s.get_field("N_SHALLOW"), cast(b))
    s.close()
