"""Seeded scenarios shared by the parity tests: each builds the same problem on any backend
(the CUDA solver or the CPU oracle) through the common method set."""
import numpy as np

from mfcm_b200 import synth, Forcing, TimeSeries, RAIN_UNIFORM, RAIN_FIELDS, RAIN_PATTERN, HEAD_EDGES, HEAD_FIELDS


def wet_dry_state(nx, ny, dx, seed=0, nan_cells=0, film=0.0):
    """Bumpy bed with a partly wet surface (wet/dry fronts on every row), random velocities."""
    rng = np.random.default_rng(seed)
    z = synth.plane_with_gaussians(nx, ny, dx, slope=0.02, n_bumps=4, amp=(0.2, 1.5),
                                   sigma=(2 * dx, 5 * dx), seed=seed + 100)
    z = z + rng.normal(0, 0.02, size=z.shape)
    level = np.percentile(z, 55)
    h = np.maximum(level - z, 0.0) + film
    h = h * (rng.uniform(size=h.shape) > 0.1)
    u = rng.normal(0, 0.3, size=h.shape) * (h > 0)
    v = rng.normal(0, 0.3, size=h.shape) * (h > 0)
    if nan_cells:
        idx = rng.choice(nx * ny, nan_cells, replace=False)
        z.ravel()[idx] = np.nan
    return z, h, u, v


def setup(backend, z, h, u, v, n=(0.03, 0.03, 0.1, 0.3), n_field=None):
    backend.set_field("Z", z)
    backend.set_field("H", h)
    backend.set_field("U", u)
    backend.set_field("V", v)
    backend.set_manning(*n)
    if n_field is not None:
        backend.set_field("N_SHALLOW", n_field)
        backend.set_field("N_DEEP", n_field)


def rain_series(rate, stop=600.0, end=1e6):
    return TimeSeries([0.0, stop, stop + 1e-3, end], [rate, rate, 0.0, 0.0])


def forcing(rain_q=(0.0, 0.0), rain_kind=RAIN_UNIFORM, head=None, edges=0):
    f = Forcing()
    if rain_q != (0.0, 0.0) or rain_kind != RAIN_UNIFORM:
        f.rain_kind, f.rain_q0, f.rain_q1 = rain_kind, rain_q[0], rain_q[1]
    if head is not None:
        f.head_kind, f.head_edges, f.head_h0, f.head_h1 = HEAD_EDGES, edges, head[0], head[1]
    return f


def same(a, b):
    """Bit-for-bit equality up to the sign of zero, NaN where NaN."""
    a = np.asarray(a)
    b = np.asarray(b)
    return a.shape == b.shape and bool(np.array_equal(a, b, equal_nan=True))


def first_diff(a, b):
    a = np.asarray(a).ravel()
    b = np.asarray(b).ravel()
    bad = ~((a == b) | (np.isnan(a) & np.isnan(b)))
    if not bad.any():
        return None
    i = int(np.argmax(bad))
    return i, a[i], b[i], int(bad.sum())
