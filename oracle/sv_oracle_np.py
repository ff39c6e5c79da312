"""TEST INFRASTRUCTURE, NOT PRODUCT CODE: an independent numpy restatement (FP64) of the
reference's stage derivative (SaintVenantSolver::update_dUdt) and of one Runge-Kutta timestep
built on it (stages, stage combination, control number, dt controller).

It restates the reference's lines a second time, vectorised over cells and faces, so that the
C++ oracle (oracle/sv_oracle.hpp) can be checked bit for bit against a restatement that shares
no code with it. Every operation keeps the reference's evaluation order, and numpy's float64
arithmetic and square root are IEEE-754 round-to-nearest like the C++ build
(-ffp-contract=off). Only the tests may import it.

Reference lines followed:
  Minmod3                       src/SpatialDerivative/Minmod3.hpp:34-82
  neighbours / faces            src/Mesh/Cartesian2DMesh.hpp:379-519
  spatial derivatives           src/SaintVenant/State.cpp:176-193, SpatialDerivative.hpp:104-121
  bed slopes                    src/SaintVenant/Constants.cpp:25-44
  face flux                     src/SaintVenant/FluxKernel.cpp:48-60 (zero_flux), 62-295
  temporal derivative           src/SaintVenant/TemporalDerivativeKernel.cpp:43-99
  Manning roughness             src/SaintVenant/SourceTerms/ManningRoughnessSourceTerm.cpp:44-88
  discharge (rain) boundary     src/SaintVenant/Boundaries/DischargeBoundarySourceTerm.cpp:39-69
  head (outflow) boundary       src/SaintVenant/Boundaries/HeadBoundarySourceTerm.cpp:39-67
  stage boundary                src/SaintVenant/Boundaries/StageBoundarySourceTerm.cpp:39-69
  energy loss                   src/SaintVenant/SourceTerms/EnergyLossSourceTerm.cpp:56-88
  infiltration                  src/SaintVenant/SourceTerms/InfiltrationSourceTerm.cpp:38-64
  update_dUdt order             src/SaintVenant/Solver.cpp:73-114
  tableaux                      src/TemporalScheme/RungeKutta.cpp:83-115
  timestep and controller       src/TemporalScheme/RungeKutta.cpp:141-167
  stage combination             src/TemporalScheme/RungeKutta.hpp:371-405
  control number                src/SaintVenant/State.cpp:195-230

sycl::pow(x, 4/3) is the division-free pow43 routine shared by both sides (cubic seed for
w^(-1/3), three Newton steps, one cube-root correction), restated here in numpy.
"""
import numpy as np

G = 9.81
NAN = np.float64("nan")
_POW43_SEED = (-0.019273, 0.18161161, -0.63413856, 1.48409885)


def sign(x):
    """sycl::sign: 1 for x > 0, -1 for x < 0, x itself for +-0, 0 for NaN."""
    x = np.asarray(x, dtype=np.float64)
    out = np.where(x > 0, 1.0, np.where(x < 0, -1.0, x))
    return np.where(np.isnan(x), 0.0, out)


def smin(x, y):
    """sycl::min (SYCL 2020): y if y < x, otherwise x."""
    return np.where(y < x, y, x)


def pow43(x):
    """x^(4/3) with IEEE + - * only: x = m 2^e, w = m 2^(e mod 3) in [0.5, 4), seed
    y ~ w^(-1/3) by a cubic, three Newton steps y += y (1 - w y^3) / 3, cube root
    cb = w y^2 with one correction, result x * cb * 2^(e div 3)."""
    x = np.asarray(x, dtype=np.float64)
    with np.errstate(all="ignore"):
        m, e = np.frexp(x)
        q = np.floor_divide(e, 3)
        w = np.ldexp(m, e - 3 * q)
        c0, c1, c2, c3 = _POW43_SEED
        third = 1.0 / 3.0
        y = ((c0 * w + c1) * w + c2) * w + c3
        for _ in range(3):
            y3 = (y * y) * y
            y = y + (y * (1.0 - w * y3)) * third
        cb = (w * y) * y
        cb = cb - ((cb * cb) * cb - w) * ((y * y) * third)
        r = x * np.ldexp(cb, q)
    r = np.where(x == 0.0, x, r)
    r = np.where(np.isinf(x) & (x > 0), np.inf, r)
    return np.where(np.isnan(x), NAN, r)


def minmod3(ul, dxl, uc, dxr, ur):
    """Minmod3 with theta = 2 (Minmod3.hpp:34-82), elementwise."""
    with np.errstate(all="ignore"):
        lhs = np.where(dxl > 0.01 * dxr, (2.0 * (uc - ul)) / np.where(dxl > 0, dxl, 1.0), NAN)
        rhs = np.where(dxr > 0.01 * dxl, (2.0 * (ur - uc)) / np.where(dxr > 0, dxr, 1.0), NAN)
        tot = dxl + dxr
        central = np.where(tot > 1e-6, (ur - ul) / np.where(tot > 0, tot, 1.0), 0.0)
        both = (0.5 * (sign(lhs) + sign(rhs))) * smin(np.abs(lhs), np.abs(rhs))
        outer = np.where(np.isnan(lhs), rhs, np.where(np.isnan(rhs), lhs, both))
        mm = (0.5 * (sign(outer) + sign(central))) * smin(np.abs(outer), np.abs(central))
        return np.where(np.isnan(outer), central, mm)


def slope_x(f, dx):
    """Minmod3 along x: west neighbour left, east neighbour right; a missing neighbour is
    the cell itself at distance 0 (Cartesian2DMesh.hpp:470-490)."""
    ny, nx = f.shape
    x = np.arange(nx)[None, :]
    left = np.concatenate([f[:, :1], f[:, :-1]], axis=1)
    right = np.concatenate([f[:, 1:], f[:, -1:]], axis=1)
    dxl = np.broadcast_to(np.where(x > 0, dx, 0.0), f.shape)
    dxr = np.broadcast_to(np.where(x < nx - 1, dx, 0.0), f.shape)
    return minmod3(left, dxl, f, dxr, right)


def slope_y(f, dy):
    """Minmod3 along y with the reference's orientation: the NORTH neighbour (row + 1) is
    the left operand and the SOUTH neighbour (row - 1) the right (Cartesian2DMesh.hpp:492-519,
    SpatialDerivative.hpp:113-118)."""
    ny, nx = f.shape
    y = np.arange(ny)[:, None]
    north = np.concatenate([f[1:, :], f[-1:, :]], axis=0)
    south = np.concatenate([f[:1, :], f[:-1, :]], axis=0)
    dl = np.broadcast_to(np.where(y < ny - 1, dy, 0.0), f.shape)
    dr = np.broadcast_to(np.where(y > 0, dy, 0.0), f.shape)
    return minmod3(north, dl, f, dr, south)


def face_geometry(nx, ny, dx, dy):
    """Per face: lhs cell, rhs cell, edge flag, direction and spacing
    (Cartesian2DMesh.hpp:379-435). Faces: the vertical block first, row by row."""
    nv = (nx + 1) * ny
    fid = np.arange(nv)
    fx, fy = fid % (nx + 1), fid // (nx + 1)
    rhs_v = np.where(fx < nx, fy * nx + np.minimum(fx, nx - 1), fy * nx + fx - 1)
    lhs_v = np.where(fx == 0, rhs_v, fy * nx + fx - 1)
    edge_v = np.where(fx == 0, -1, np.where(fx == nx, 1, 0))
    f2 = np.arange(nx * (ny + 1))
    gx, gy = f2 % nx, f2 // nx
    rhs_h = np.where(gy < ny, np.minimum(gy, ny - 1) * nx + gx, (gy - 1) * nx + gx)
    lhs_h = np.where(gy == 0, rhs_h, (gy - 1) * nx + gx)
    edge_h = np.where(gy == 0, -1, np.where(gy == ny, 1, 0))
    lhs = np.concatenate([lhs_v, lhs_h])
    rhs = np.concatenate([rhs_v, rhs_h])
    edge = np.concatenate([edge_v, edge_h])
    d = np.concatenate([np.zeros(nv, dtype=int), np.ones(f2.size, dtype=int)])
    spacing = np.where(d == 0, dx, dy).astype(np.float64)
    return lhs, rhs, edge, d, spacing


def face_fluxes(h, u, v, z, sl, nx, ny, dx, dy):
    """SaintVenantFluxKernel::operator() (FluxKernel.cpp:62-295) for every face. `sl` holds
    the cell slopes dhdx, dudx, dvdx, dhdy, dudy, dvdy, dzdx, dzdy. Returns the h, u, v, z
    fluxes and the branch code."""
    H, U, V, Z = (a.ravel() for a in (h, u, v, z))
    S = {k: a.ravel() for k, a in sl.items()}
    lhs, rhs, edge, d, fdx = face_geometry(nx, ny, dx, dy)
    xdir = 1.0 - d.astype(np.float64)
    ydir = d.astype(np.float64)
    zero = np.zeros(lhs.size, dtype=bool)
    # coded-out (NaN bed) cells, FluxKernel.cpp:85-108
    zl_nan = np.isnan(Z[lhs])
    zero |= zl_nan & (edge == 1)
    lhs = np.where(zl_nan, rhs, lhs)
    edge = np.where(zl_nan & (edge != 1), -1, edge)
    zr_nan = np.isnan(Z[rhs])
    zero |= zr_nan & (edge == -1)
    rhs = np.where(zr_nan & (edge != -1), lhs, rhs)
    edge = np.where(zr_nan & (edge != -1), 1, edge)
    zb_L, zb_R = Z[lhs], Z[rhs]
    mL = np.where(edge < 0, 0.0, 1.0)
    mR = np.where(edge > 0, 0.0, 1.0)
    muL = np.where((edge < 0) & (xdir == 1), 0.0, 1.0)
    muR = np.where((edge > 0) & (xdir == 1), 0.0, 1.0)
    mvL = np.where((edge < 0) & (ydir == 1), 0.0, 1.0)
    mvR = np.where((edge > 0) & (ydir == 1), 0.0, 1.0)
    with np.errstate(all="ignore"):
        h_L, h_R = H[lhs] * mL, H[rhs] * mR
        u_L, u_R = U[lhs] * muL, U[rhs] * muR
        v_L, v_R = V[lhs] * mvL, V[rhs] * mvR
        dhdx_L, dhdx_R = S["dhdx"][lhs] * mL, S["dhdx"][rhs] * mR
        dhdy_L, dhdy_R = S["dhdy"][lhs] * mL, S["dhdy"][rhs] * mR
        dudx_L, dudx_R = S["dudx"][lhs] * muL, S["dudx"][rhs] * muR
        dudy_L, dudy_R = S["dudy"][lhs] * muL, S["dudy"][rhs] * muR
        dvdx_L, dvdx_R = S["dvdx"][lhs] * mvL, S["dvdx"][rhs] * mvR
        dvdy_L, dvdy_R = S["dvdy"][lhs] * mvL, S["dvdy"][rhs] * mvR
        dzdx_L, dzdx_R = S["dzdx"][lhs] * mL, S["dzdx"][rhs] * mR
        dzdy_L, dzdy_R = S["dzdy"][lhs] * mL, S["dzdy"][rhs] * mR
        zb_L = np.where(edge < 0, zb_R + h_R * 2.0, zb_L)
        zb_R = np.where(edge > 0, zb_L + h_L * 2.0, zb_R)

        def proj(c, sx, sy, k):
            return (c + ((k * fdx) * sx) * xdir) + ((k * fdx) * sy) * ydir

        zb_m, h_m = proj(zb_L, dzdx_L, dzdy_L, 0.5), proj(h_L, dhdx_L, dhdy_L, 0.5)
        u_m, v_m = proj(u_L, dudx_L, dudy_L, 0.5), proj(v_L, dvdx_L, dvdy_L, 0.5)
        zb_p, h_p = proj(zb_R, dzdx_R, dzdy_R, -0.5), proj(h_R, dhdx_R, dhdy_R, -0.5)
        u_p, v_p = proj(u_R, dudx_R, dudy_R, -0.5), proj(v_R, dvdx_R, dvdy_R, -0.5)
        zb_f = np.fmax(zb_m, zb_p)
        y_m, y_p = zb_m + h_m, zb_p + h_p
        h_m, h_p = np.fmax(h_m, 0.0), np.fmax(h_p, 0.0)
        c_m, c_p = np.sqrt(G * h_m), np.sqrt(G * h_p)
        kx, ky = 1.0 - 0.5 * xdir, 1.0 - 0.5 * ydir
        spd_m = u_m * xdir + v_m * ydir
        spd_p = u_p * xdir + v_p * ydir
        hf_m, hf_p = h_m * spd_m, h_p * spd_p
        uf_m_plus = u_m * (kx * spd_m) + (G * h_m) * xdir
        vf_m_plus = v_m * (ky * spd_m) + (G * h_m) * ydir
        uf_p_minus = u_p * (kx * spd_p) - (G * h_p) * xdir
        vf_p_minus = v_p * (ky * spd_p) - (G * h_p) * ydir
        uf_p_plus = u_p * (kx * spd_p) + (G * h_p) * xdir
        vf_p_plus = v_p * (ky * spd_p) + (G * h_p) * ydir
        a_m = np.abs(spd_m + sign(spd_m) * c_m)
        a_p = np.abs(spd_p + sign(spd_p) * c_p)
        # branch 1: both water levels above the face bed
        a1 = np.fmax(a_p, a_m)
        b1 = ((0.5 * (hf_p + hf_m)) - (0.5 * a1) * (h_p - h_m),
              (0.5 * (uf_p_minus + uf_m_plus)) - (0.5 * a1) * (u_p - u_m),
              (0.5 * (vf_p_minus + vf_m_plus)) - (0.5 * a1) * (v_p - v_m),
              (zb_m - zb_p) * G)
        # branch 2: both below; the lower side pushes on the step
        up = zb_p > zb_m
        b2 = (np.zeros_like(h_m),
              np.where(up, 0.5 * ((G * h_m) * xdir), -0.5 * ((G * h_p) * xdir)),
              np.where(up, 0.5 * ((G * h_m) * ydir), -0.5 * ((G * h_p) * ydir)),
              np.where(up, ((-h_m) * 0.5) * G, (h_p * 0.5) * G))
        # branch 3: only the left side above the face bed
        b3 = ((0.5 * hf_m) - (0.5 * a_m) * (-h_m), (0.5 * uf_m_plus) - (0.5 * a_m) * (-u_m),
              (0.5 * vf_m_plus) - (0.5 * a_m) * (-v_m), h_p / fdx)
        # branch 4: only the right side above (pressure term added, as in the reference)
        b4 = ((0.5 * hf_p) - (0.5 * a_p) * h_p, (0.5 * uf_p_plus) - (0.5 * a_p) * u_p,
              (0.5 * vf_p_plus) - (0.5 * a_p) * v_p, h_m / fdx)
    c1 = (y_m > zb_f) & (y_p > zb_f)
    c2 = ~c1 & (y_m <= zb_f) & (y_p <= zb_f)
    c3 = ~c1 & ~c2 & (y_m > zb_f)
    out = []
    for k in range(4):
        f = np.where(c1, b1[k], np.where(c2, b2[k], np.where(c3, b3[k], b4[k])))
        out.append(np.where(zero, 0.0, f))
    branch = np.where(c1, 1.0, np.where(c2, np.where(up, 2.25, 2.75), np.where(c3, 3.0, 4.0)))
    out.append(np.where(zero, 0.0, branch))
    return out


def update_dudt(h, u, v, z, dx, dy, *, manning=None, qbdy=None, hbdy=None, time_now=0.0, timestep=1.0,
                step_length=60.0, rain_mode="reference", head_first=False, eloss=None, eloss_first=False,
                infil=None, stage=False, eddy=None, order=None):
    """dU/dt of one state (SaintVenantSolver::update_dUdt, Solver.cpp:73-114). Arrays are
    (ny, nx). manning = (n_shallow, n_deep, d_shallow, d_deep) per-cell arrays or None (no
    roughness term); eloss = (fx, fy) energy-loss coefficients or None; infil = (rate,
    capacity) or None; qbdy = (q0, q1) and hbdy = (h0, h1) per-cell boundary values or None,
    hbdy holding water levels when `stage` (a stage boundary). eddy = ("constant", mu) with mu
    a scalar or per-cell array, or ("smagorinsky", mu_const, mu_smag), or None; order lists the
    momentum terms ("manning", "energy loss", "eddy viscosity") in configuration order
    (default: per eloss_first, then eddy viscosity). Returns a dict of slopes, face
    fields, dhdt/dudt/dvdt and, with infiltration, the capacity left ("infil_cap")."""
    ny, nx = h.shape
    sl = {"dhdx": slope_x(h, dx), "dudx": slope_x(u, dx), "dvdx": slope_x(v, dx),
          "dhdy": slope_y(h, dy), "dudy": slope_y(u, dy), "dvdy": slope_y(v, dy),
          "dzdx": slope_x(z, dx), "dzdy": slope_y(z, dy)}
    fh, fu, fv, fz, fb = face_fluxes(h, u, v, z, sl, nx, ny, dx, dy)
    cx = np.arange(nx)[None, :]
    cy = np.arange(ny)[:, None]
    w = cy * (nx + 1) + cx
    e = w + 1
    s = (nx + 1) * ny + cy * nx + cx
    n = s + nx
    with np.errstate(all="ignore"):
        dhdt = (fh[w] - fh[e]) / dx + (fh[s] - fh[n]) / dy
        dudt = (fu[w] - fu[e]) / dx + (fu[s] - fu[n]) / dy
        dvdt = (fv[w] - fv[e]) / dx + (fv[s] - fv[n]) / dy
        dudt = dudt + sl["dhdx"] * -G
        dvdt = dvdt + sl["dhdy"] * -G
        zx, zy = sl["dzdx"], sl["dzdy"]
        zx = np.where(np.abs(zx) > h / dx, (sign(zx) * h) / dx, zx)
        zy = np.where(np.abs(zy) > h / dy, (sign(zy) * h) / dy, zy)
        dudt = dudt + (fz[w] - fz[e]) / dx
        dvdt = dvdt + (fz[s] - fz[n]) / dy
        dudt = dudt + (-G) * zx
        dvdt = dvdt + (-G) * zy
        def roughness(dudt, dvdt):
            if manning is None:
                return dudt, dvdt
            ns, nd, ds, dd = manning
            t = np.fmin(np.fmax((h - ds) / (dd - ds), 0.0), 1.0)
            nman = ns + (nd - ns) * ((t * t) * (3.0 - 2.0 * t))
            wet = h > 1e-6
            inv_h = h / (h * h + 1e-3)
            sf = ((nman * nman) * np.sqrt(u * u + v * v)) * pow43(inv_h)
            fu_ = ((-G) * sf) * u
            fv_ = ((-G) * sf) * v
            capu = (np.abs(fu_ * timestep) > np.abs(u)) & (sign(fu_ * timestep) != sign(u))
            capv = (np.abs(fv_ * timestep) > np.abs(v)) & (sign(fv_ * timestep) != sign(v))
            fu_ = np.where(capu, -u / timestep, fu_)
            fv_ = np.where(capv, -v / timestep, fv_)
            return np.where(wet, dudt + fu_, dudt), np.where(wet, dvdt + fv_, dvdt)

        def energy_loss(dudt, dvdt):
            # EnergyLossSourceKernel::operator() (EnergyLossSourceTerm.cpp:64-87)
            if eloss is None:
                return dudt, dvdt
            fx, fy = eloss
            wet = h > 1e-6
            hyp = np.sqrt(u * u + v * v)
            eu = (((-0.5) * u) * fx) * hyp
            ev = (((-0.5) * v) * fy) * hyp
            capu = (np.abs(eu * timestep) > np.abs(u)) & (sign(eu * timestep) != sign(u))
            capv = (np.abs(ev * timestep) > np.abs(v)) & (sign(ev * timestep) != sign(v))
            eu = np.where(capu, -u / timestep, eu)
            ev = np.where(capv, -v / timestep, ev)
            return np.where(wet, dudt + eu, dudt), np.where(wet, dvdt + ev, dvdt)

        def eddy_viscosity(dudt, dvdt):
            # SmagorinskyCoefficientKernel and EddyViscositySourceKernel
            # (EddyViscositySourceTerm.cpp:46-110); second derivatives are Minmod3 slopes of
            # the slopes along the same axis (EddyViscositySourceTerm.hpp:222-228)
            if eddy is None:
                return dudt, dvdt
            uxx, uyy = slope_x(sl["dudx"], dx), slope_y(sl["dudy"], dy)
            vxx, vyy = slope_x(sl["dvdx"], dx), slope_y(sl["dvdy"], dy)
            if eddy[0] == "smagorinsky":
                a = np.abs(sl["dudy"]) + np.abs(sl["dvdx"])
                strain = np.sqrt((sl["dudx"] * sl["dudx"] + sl["dvdy"] * sl["dvdy"]) + 0.5 * (a * a))
                mu = eddy[1] + (eddy[2] * (dx * dy)) * strain
            else:
                mu = np.broadcast_to(np.asarray(eddy[1], dtype=np.float64), h.shape)
            wet = h > 1e-6
            eu = (-mu) * (uxx + uyy)
            ev = (-mu) * (vxx + vyy)
            capu = (np.abs(eu * timestep) > np.abs(u)) & (sign(eu * timestep) != sign(u))
            capv = (np.abs(ev * timestep) > np.abs(v)) & (sign(ev * timestep) != sign(v))
            eu = np.where(capu, -u / timestep, eu)
            ev = np.where(capv, -v / timestep, ev)
            return np.where(wet, dudt + eu, dudt), np.where(wet, dvdt + ev, dvdt)

        terms = {"manning": roughness, "energy loss": energy_loss, "eddy viscosity": eddy_viscosity}
        if order is None:
            order = ["energy loss", "manning"] if eloss_first else ["manning", "energy loss"]
        order = list(order) + [t for t in ("manning", "energy loss", "eddy viscosity") if t not in order]
        for t in order:
            dudt, dvdt = terms[t](dudt, dvdt)
        cap_left = None
        if infil is not None:
            # InfiltrationSourceKernel::operator() (InfiltrationSourceTerm.cpp:43-62)
            rate, cap = infil
            dh = rate * timestep
            dh = np.where(dh > h, h, dh)
            dh = np.where(dh > cap, cap, dh)
            dhdt = dhdt - dh / timestep
            cap_left = cap - dh

        def discharge(dh):
            if qbdy is None:
                return dh
            q0, q1 = qbdy
            on = (q0 != 0.0) | (q1 != 0.0)
            dqdt = (q1 - q0) / step_length
            qnow = q0 + time_now * dqdt
            qnext = qnow + timestep * dqdt
            r = 0.5 * (qnow + qnext)
            if rain_mode == "reference":
                r = np.where(h - r * timestep <= 0.0, -h / timestep, r)
            else:
                r = np.where(h + r * timestep <= 0.0, -h / timestep, r)
            return np.where(on, dh + r, dh)

        def head(dh):
            if hbdy is None:
                return dh
            h0, h1 = hbdy
            if stage:  # StageBoundarySourceKernel (StageBoundarySourceTerm.cpp:48-52)
                h0, h1 = h0 - z, h1 - z
            on = ~np.isnan(h0) & ~np.isnan(h1)
            slope = (h1 - h0) / step_length
            now = h0 + time_now * slope
            nxt = now + timestep * slope
            target = 0.5 * (now + nxt)
            target = np.where(target <= 0.0, 0.0, target)
            return np.where(on, (target - h) / timestep, dh)

        dhdt = discharge(head(dhdt)) if head_first else head(discharge(dhdt))
    out = dict(sl)
    out.update({"flux_h": fh, "flux_u": fu, "flux_v": fv, "flux_z": fz, "flux_branch": fb,
                "dhdt": dhdt, "dudt": dudt, "dvdt": dvdt, "infil_cap": cap_left})
    return out


def edge_strips(nx, ny, edges, v0, v1):
    """Head-boundary fields for a target on whole mesh edges (bit 1 x-min column, 2 x-max
    column, 4 y-min row, 8 y-max row); NaN elsewhere, as the reference's NaN-initialised
    head fields."""
    h0 = np.full((ny, nx), NAN)
    h1 = np.full((ny, nx), NAN)
    for bit, sl in ((1, (slice(None), 0)), (2, (slice(None), nx - 1)), (4, (0, slice(None))),
                    (8, (ny - 1, slice(None)))):
        if edges & bit:
            h0[sl] = v0
            h1[sl] = v1
    return h0, h1


# Butcher rows as the reference stores them (RungeKutta.cpp:83-115): row i holds c_i followed
# by a(i, 1..i-1); the last row holds 0 followed by the weights b.
TABLEAUX = {
    "classic": [[0.0], [0.5, 0.5], [0.5, 0.0, 0.5], [1.0, 0.0, 0.0, 1.0],
                [0.0, 1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0]],
    "ralston4": [[0.0], [0.4, 0.4], [0.45573725, 0.29697761, 0.15875964],
                 [1.0, 0.21810040, -3.05096516, 3.83286476],
                 [0.0, 0.17476028, -0.55148066, 1.20553560, 0.17118478]],
    "3/8rule": [[0.0], [1.0 / 3.0, 1.0 / 3.0], [2.0 / 3.0, -1.0 / 3.0, 1.0], [1.0, 1.0, -1.0, 1.0],
                [0.0, 1.0 / 8.0, 3.0 / 8.0, 3.0 / 8.0, 1.0 / 8.0]],
}


def control_number(h, u, v, dx, dy, timestep):
    """SaintVenantState::max_control_number (State.cpp:195-230); NaN propagates."""
    with np.errstate(all="ignore"):
        c = np.sqrt(G * np.fmax(h, 0.0))
        cn = timestep * (((np.abs(u) + c) / dx) + ((np.abs(v) + c) / dy))
    return float(np.max(cn))


def do_timestep(h, u, v, z, dx, dy, local_time, dt, method="classic", cn_target=1.0, terms_out=None, **terms):
    """RungeKuttaTemporalScheme::do_timestep (RungeKutta.cpp:141-167) with the stage
    combination of RungeKuttaSolver::update_y (RungeKutta.hpp:371-405): stage s evaluates
    dU/dt of state s-1 at local_time + c_s dt, then state s = U0 + sum_j k_j (a(s+1, j) dt),
    added left to right. Returns (state N, control number, repeat, new dt); the controller
    takes the target as a parameter (1.0 in the reference)."""
    rows = TABLEAUX[method]
    N = len(rows) - 1
    states = [(h, u, v)]
    ks = []
    terms = dict(terms)
    for s in range(1, N + 1):
        t_sub = local_time + rows[s - 1][0] * dt
        y = states[s - 1]
        r = update_dudt(y[0], y[1], y[2], z, dx, dy, time_now=t_sub, timestep=dt, **terms)
        if r["infil_cap"] is not None:  # the capacity is consumed by every stage evaluation
            terms["infil"] = (terms["infil"][0], r["infil_cap"])
        ks.append((r["dhdt"], r["dudt"], r["dvdt"]))
        acc = [a.copy() for a in states[0]]
        with np.errstate(all="ignore"):
            for col in range(s):
                coef = rows[s][col + 1] * dt
                acc = [acc[k] + ks[col][k] * coef for k in range(3)]
        states.append(tuple(acc))
    if terms_out is not None:
        terms_out.update(terms)
    hN, uN, vN = states[N]
    cn = control_number(hN, uN, vN, dx, dy, dt)
    if cn > cn_target:
        rep, nd = True, (dt / 5.0 if cn > 5.0 * cn_target else (dt * cn_target) / (cn * 1.1))
    elif cn > 0.9 * cn_target:
        rep, nd = False, dt
    else:
        rep, nd = False, (dt * cn_target) / cn if cn != 0.0 else float("inf")
    return states[N], cn, rep, nd
