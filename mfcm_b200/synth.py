"""Seeded synthetic catchments (no public dataset is used or needed).

Each generator returns float64 numpy arrays shaped (ny, nx), row-major with x fastest
(cell i = y*nx + x, src/Mesh/Cartesian2DMesh.hpp:143-145).
"""
import numpy as np

MM_PER_H = 1.0 / 3.6e6  # 1 mm/h in m/s


def plane_with_gaussians(nx, ny, dx, slope=0.01, n_bumps=8, amp=(0.0, 2.0), sigma=(20.0, 60.0), seed=1):
    """Tilted plane descending toward +x with `slope`, plus Gaussian bumps of amplitude
    U(amp) m, width U(sigma) m and centres uniform in the domain."""
    rng = np.random.default_rng(seed)
    x = (np.arange(nx) + 0.5) * dx
    y = (np.arange(ny) + 0.5) * dx
    X, Y = np.meshgrid(x, y)
    z = slope * (nx * dx - X)
    for _ in range(n_bumps):
        a = rng.uniform(*amp)
        s = rng.uniform(*sigma)
        cx, cy = rng.uniform(0, nx * dx), rng.uniform(0, ny * dx)
        z = z + a * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2.0 * s * s))
    return z


def diamond_square(nx, ny, hurst=0.8, relief=100.0, seed=2):
    """Diamond-square fractal surface with Hurst exponent `hurst`, rescaled to `relief` m
    (max - min), cropped from the smallest 2^k+1 square covering nx x ny."""
    rng = np.random.default_rng(seed)
    k = int(np.ceil(np.log2(max(nx, ny, 2) - 1))) if max(nx, ny) > 2 else 1
    n = 2 ** k + 1
    a = np.zeros((n, n))
    a[0, 0], a[0, -1], a[-1, 0], a[-1, -1] = rng.normal(size=4)
    step = n - 1
    scale = 1.0
    while step > 1:
        h = step // 2
        # diamond: centres of squares
        c = (a[0:-1:step, 0:-1:step] + a[0:-1:step, step::step] + a[step::step, 0:-1:step] + a[step::step, step::step]) / 4.0
        a[h:-1:step, h:-1:step] = c + scale * rng.normal(size=c.shape)
        # square: edge midpoints (average of up to 4 neighbours)
        for (oy, ox) in ((0, h), (h, 0)):
            ys = np.arange(oy, n, step)
            xs = np.arange(ox, n, step)
            Yi, Xi = np.meshgrid(ys, xs, indexing="ij")
            acc = np.zeros(Yi.shape)
            cnt = np.zeros(Yi.shape)
            for dy_, dx_ in ((-h, 0), (h, 0), (0, -h), (0, h)):
                yy, xx = Yi + dy_, Xi + dx_
                ok = (yy >= 0) & (yy < n) & (xx >= 0) & (xx < n)
                acc[ok] += a[yy[ok], xx[ok]]
                cnt[ok] += 1
            a[Yi, Xi] = acc / cnt + scale * rng.normal(size=Yi.shape)
        step = h
        scale *= 0.5 ** hurst
    z = a[:ny, :nx]
    z = z - z.min()
    span = z.max()
    return z * (relief / span if span > 0 else 0.0)


def gaussian_smooth(field, sigma_cells):
    """Periodic Gaussian smoothing by FFT (sigma in cells)."""
    ny, nx = field.shape
    ky = np.fft.fftfreq(ny)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    g = np.exp(-2.0 * (np.pi ** 2) * (sigma_cells ** 2) * (kx ** 2 + ky ** 2))
    return np.fft.irfft2(np.fft.rfft2(field) * g, s=field.shape)


def lognormal_rain(nx, ny, dx, mean_mm_h=30.0, sigma_log=0.5, smooth_m=200.0, seed=3):
    """Spatial rain-rate field (m/s): lognormal with the given mean, Gaussian-smoothed over
    `smooth_m` metres, rescaled back to the requested mean."""
    rng = np.random.default_rng(seed)
    mu = np.log(mean_mm_h) - 0.5 * sigma_log ** 2
    f = rng.lognormal(mu, sigma_log, size=(ny, nx))
    f = gaussian_smooth(f, smooth_m / dx)
    f = np.maximum(f, 0.0)
    f *= mean_mm_h / f.mean()
    return f * MM_PER_H


def voronoi_classes(nx, ny, values=(0.02, 0.035, 0.05, 0.1), n_sites=256, seed=4):
    """Piecewise-constant field: each cell takes the value of its nearest of `n_sites`
    random sites, each site holding one of `values`."""
    rng = np.random.default_rng(seed)
    sx = rng.uniform(0, nx, n_sites)
    sy = rng.uniform(0, ny, n_sites)
    cls = rng.integers(0, len(values), n_sites)
    try:
        from scipy.spatial import cKDTree
        t = cKDTree(np.stack([sx, sy], 1))
        X, Y = np.meshgrid(np.arange(nx) + 0.5, np.arange(ny) + 0.5)
        _, idx = t.query(np.stack([X.ravel(), Y.ravel()], 1))
        idx = idx.reshape(ny, nx)
    except ImportError:  # pragma: no cover
        X, Y = np.meshgrid(np.arange(nx) + 0.5, np.arange(ny) + 0.5)
        d = (X[..., None] - sx) ** 2 + (Y[..., None] - sy) ** 2
        idx = d.argmin(-1)
    return np.asarray(values)[cls[idx]]


def regional_slope(nx, ny, dx, slope=0.005):
    x = (np.arange(nx) + 0.5) * dx
    return np.broadcast_to(slope * (nx * dx - x), (ny, nx)).copy()


def dam_break(nx, ny, z0=350.0, h_up=1.0):
    """Flat bed at z0 with h = h_up for x below the centre, dry downstream."""
    z = np.full((ny, nx), z0)
    h = np.zeros((ny, nx))
    h[:, : nx // 2] = h_up
    return z, h


def lowest_edge(z):
    """Edge (SV_EDGE_* bit) with the lowest mean bed elevation."""
    means = {1: z[:, 0].mean(), 2: z[:, -1].mean(), 4: z[0, :].mean(), 8: z[-1, :].mean()}
    return min(means, key=means.get)


def config1(seed=1):
    """256 x 256, dx = 5 m: plane slope 0.01 along +x plus 8 Gaussian bumps; rain 50 mm/h
    for 600 s; n = 0.03; walls plus outflow on the lowest edge."""
    nx = ny = 256
    dx = 5.0
    z = plane_with_gaussians(nx, ny, dx, seed=seed)
    return dict(nx=nx, ny=ny, dx=dx, z=z, rain_rate=50.0 * MM_PER_H, n=0.03, edges=lowest_edge(z))


def config2(nx=4096, ny=4096, dx=2.0, seed=2):
    """4096 x 4096, dx = 2 m: diamond-square (H 0.8, 100 m relief) + 0.005 slope; lognormal
    rain field (mean 30 mm/h, sigma_log 0.5, smoothed 200 m) for 1800 s; Voronoi Manning n
    classes; outflow on all edges."""
    z = diamond_square(nx, ny, 0.8, 100.0, seed=seed) + regional_slope(nx, ny, dx, 0.005)
    rain = lognormal_rain(nx, ny, dx, 30.0, 0.5, 200.0, seed=seed + 1)
    n = voronoi_classes(nx, ny, seed=seed + 2)
    return dict(nx=nx, ny=ny, dx=dx, z=z, rain=rain, n=n, edges=15)
