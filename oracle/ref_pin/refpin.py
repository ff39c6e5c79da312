"""TEST INFRASTRUCTURE: ctypes binding of oracle/_ref/libsv_refpin.so (the reference's own
hot-path kernels, built by oracle/ref_pin/build.py). Only tests/ and tests/golden/ use it.

Every function takes and returns numpy arrays shaped (ny, nx) for cell fields and flat arrays
of (nx+1)*ny + (ny+1)*nx values for face fields, in the value type of the precision asked for.
"""
import ctypes as C
import importlib.util
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_lib = None


def _build_module():
    spec = importlib.util.spec_from_file_location("sv_refpin_build", os.path.join(_HERE, "build.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    return m


def available():
    return _build_module().available()


def load():
    global _lib
    if _lib is None:
        _lib = C.CDLL(_build_module().build())
        for t, ct in (("f64", C.c_double), ("f32", C.c_float)):
            P = C.POINTER(ct)
            f = getattr(_lib, f"refpin_dudt_{t}")
            f.restype = C.c_int
            f.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double] + [P] * 12 + \
                         [C.c_int, C.c_double, C.c_double, C.c_double, P]
            f = getattr(_lib, f"refpin_control_number_{t}")
            f.restype = C.c_int
            f.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double, P, P, P, C.c_double, P]
            f = getattr(_lib, f"refpin_solve_{t}")
            f.restype = C.c_int
            D = C.POINTER(C.c_double)
            f.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double, P, P, P, P, D, D, D, C.c_int, C.c_uint,
                          C.c_double, C.c_int, C.c_char_p, C.c_double, C.c_double, C.c_double, C.c_double, P,
                          C.POINTER(C.c_uint64)]
            f = getattr(_lib, f"refpin_dudt_terms_{t}")
            f.restype = C.c_int
            f.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double] + [P] * 4 + \
                         [C.POINTER(P), P, C.POINTER(C.c_int), C.POINTER(C.c_double), P]
            f = getattr(_lib, f"refpin_write_fields_{t}")
            f.restype = C.c_int
            f.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                          C.POINTER(C.c_char_p), C.POINTER(P), C.c_char_p, C.c_int, C.c_char_p]
            f = getattr(_lib, f"refpin_write_series_{t}")
            f.restype = C.c_int
            f.argtypes = [C.c_uint64, C.POINTER(C.c_double), P, C.c_char_p, C.c_char_p]
            f = getattr(_lib, f"refpin_update_y_{t}")
            f.restype = C.c_int
            f.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double, P, P, C.c_int,
                          C.POINTER(C.c_double), C.c_double, P]
    if not getattr(_lib, "_nearest_set", False):
        f = _lib.refpin_nearest_cells
        f.restype = C.c_int
        D = C.POINTER(C.c_double)
        f.argtypes = [C.c_uint64, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_double, C.c_uint64, D,
                      C.POINTER(C.c_uint64), D]
        f = _lib.refpin_num_steps
        f.restype = C.c_int
        f.argtypes = [C.c_double, C.c_double, C.c_double, C.POINTER(C.c_uint64)]
        _lib._nearest_set = True
    return _lib


def num_steps(start, end, step):
    """TimeParameters::num_steps of the reference (TimeType double)."""
    n = C.c_uint64()
    if load().refpin_num_steps(start, end, step, C.byref(n)) != 0:
        raise RuntimeError("reference time parameters failed")
    return n.value


def nearest_cells(nx, ny, dx, dy, origin, x, y):
    """Cartesian2DMesh::get_nearest_object_index<Cell> of the locations (x, y) (nx * ny when
    outside the mesh) and get_object_location<Cell> of every cell, as (index array, (cx, cy))."""
    lib = load()
    xy = np.ascontiguousarray(np.stack([np.ravel(x), np.ravel(y)], axis=1), dtype=np.float64)
    n = xy.shape[0]
    out = np.empty(n, dtype=np.uint64)
    loc = np.empty(2 * nx * ny, dtype=np.float64)
    r = lib.refpin_nearest_cells(nx, ny, dx, dy, origin[0], origin[1], n, _ptr(xy, C.c_double),
                                 out.ctypes.data_as(C.POINTER(C.c_uint64)), _ptr(loc, C.c_double))
    if r != 0:
        raise RuntimeError("reference mesh failed")
    return out.astype(np.int64), (loc[0::2], loc[1::2])


def _np(precision):
    return (np.float64, C.c_double) if precision == "f64" else (np.float32, C.c_float)


def _ptr(a, ct):
    return None if a is None else a.ctypes.data_as(C.POINTER(ct))


SLOPES = ["DZDX", "DZDY", "DHDX", "DUDX", "DVDX", "DHDY", "DUDY", "DVDY"]
FACES = ["FLUX_H", "FLUX_U", "FLUX_V", "FLUX_Z", "FLUX_BRANCH"]
KS = ["DHDT", "DUDT", "DVDT"]


def dudt(z, h, u, v, dx, dy=None, manning=None, q=None, head=None, head_first=False, time_now=0.0, timestep=1.0,
         step_length=60.0, precision="f64"):
    """One SaintVenantSolver::update_dUdt through the reference's kernels. manning = (ns, nd, ds,
    dd) cell arrays, q = (q0, q1) discharge boundary values, head = (h0, h1) head boundary
    values (NaN = not selected). Returns a dict of the slope, face and derivative fields."""
    lib = load()
    dt_, ct = _np(precision)
    dy = dx if dy is None else dy
    ny, nx = h.shape
    nc, nf = nx * ny, (nx + 1) * ny + (ny + 1) * nx
    arr = lambda a: None if a is None else np.ascontiguousarray(a, dtype=dt_)
    m = [arr(a) for a in (manning or (None,) * 4)]
    qq = [arr(a) for a in (q or (None, None))]
    hh = [arr(a) for a in (head or (None, None))]
    ins = [arr(a) for a in (z, h, u, v)]
    out = np.empty(8 * nc + 5 * nf + 3 * nc, dtype=dt_)
    f = getattr(lib, f"refpin_dudt_{precision}")
    r = f(nx, ny, dx, dy, *[_ptr(a, ct) for a in ins + m + qq + hh], 1 if head_first else 0, time_now, timestep,
          step_length, _ptr(out, ct))
    if r != 0:
        raise RuntimeError("reference kernels failed")
    res = {}
    o = 0
    for name in SLOPES:
        res[name] = out[o:o + nc].reshape(ny, nx)
        o += nc
    for name in FACES:
        res[name] = out[o:o + nf]
        o += nf
    for name in KS:
        res[name] = out[o:o + nc].reshape(ny, nx)
        o += nc
    return res


def dudt_terms(z, h, u, v, dx, dy=None, manning=None, eloss=None, infil=None, eddy=None, q=None, stage=None,
               stage_first=False, order=(1, 2, 3), time_now=0.0, timestep=1.0, step_length=60.0, precision="f64"):
    """One update_dUdt with the further source and boundary terms through the reference's
    kernels: manning = (ns, nd, ds, dd) cell arrays, eloss = (fx, fy), infil = (rate, capacity),
    eddy = ("field", mu) or ("smagorinsky", mu_const, mu_smag), q = (q0, q1) discharge values,
    stage = (l0, l1) water levels (NaN = not selected); `order` the configured order of the
    momentum terms (1 roughness, 2 energy loss, 3 eddy viscosity). Returns dh/dt, du/dt, dv/dt
    and the infiltration capacity after the evaluation (None without infiltration)."""
    lib = load()
    dt_, ct = _np(precision)
    dy = dx if dy is None else dy
    ny, nx = h.shape
    nc = nx * ny
    arr = lambda a: None if a is None else np.ascontiguousarray(a, dtype=dt_)
    keep = []
    slots = [None] * 12

    def put(i, a):
        a = arr(a)
        keep.append(a)
        slots[i] = a

    for i, a in enumerate(manning or ()):
        put(i, a)
    if eloss:
        put(4, eloss[0]); put(5, eloss[1])
    cap = None
    if infil:
        put(6, infil[0])
        cap = arr(infil[1]).copy()
    mode, mu_c, mu_s = 0, 0.0, 0.0
    if eddy:
        if eddy[0] == "field":
            mode = 1
            put(7, eddy[1])
        else:
            mode, mu_c, mu_s = 2, float(eddy[1]), float(eddy[2])
    if q:
        put(8, q[0]); put(9, q[1])
    if stage:
        put(10, stage[0]); put(11, stage[1])
    F = (C.POINTER(ct) * 12)(*[_ptr(a, ct) if a is not None else None for a in slots])
    iopt = (C.c_int * 5)(mode, 1 if stage_first else 0, *list(order))
    dopt = (C.c_double * 5)(mu_c, mu_s, time_now, timestep, step_length)
    ins = [arr(a) for a in (z, h, u, v)]
    out = np.empty(3 * nc, dtype=dt_)
    r = getattr(lib, f"refpin_dudt_terms_{precision}")(nx, ny, dx, dy, *[_ptr(a, ct) for a in ins], F, _ptr(cap, ct),
                                                       iopt, dopt, _ptr(out, ct))
    if r != 0:
        raise RuntimeError("reference kernels failed")
    res = {name: out[i * nc:(i + 1) * nc].reshape(ny, nx) for i, name in enumerate(KS)}
    res["INFIL_CAP"] = None if cap is None else cap.reshape(ny, nx)
    return res


def write_fields(path, nx, ny, dx, dy, origin, names, values, delimiter=", ", binary=False, precision="f64"):
    """Write cell fields (arrays of nx * ny values, names as str) the way the reference's
    MultiFieldOutputFile does: CSVOutput (or RawBinaryOutput) over a FieldOutputFunction on a
    mesh with the given cell size and origin."""
    lib = load()
    dt_, ct = _np(precision)
    vals = [np.ascontiguousarray(np.asarray(v).ravel(), dtype=dt_) for v in values]
    nm = (C.c_char_p * len(names))(*[n.encode() for n in names])
    vp = (C.POINTER(ct) * len(vals))(*[_ptr(v, ct) for v in vals])
    r = getattr(lib, f"refpin_write_fields_{precision}")(nx, ny, dx, dy, origin[0], origin[1], len(vals), nm, vp,
                                                         delimiter.encode(), 1 if binary else 0,
                                                         os.fsencode(path))
    if r != 0:
        raise RuntimeError("reference output failed")


def write_series(path, times, values, name, precision="f64"):
    """Write a measure's points the way the reference's Measure::output does."""
    lib = load()
    dt_, ct = _np(precision)
    t = np.ascontiguousarray(times, dtype=np.float64)
    v = np.ascontiguousarray(values, dtype=dt_)
    r = getattr(lib, f"refpin_write_series_{precision}")(len(t), t.ctypes.data_as(C.POINTER(C.c_double)),
                                                         _ptr(v, ct), name.encode(), os.fsencode(path))
    if r != 0:
        raise RuntimeError("reference output failed")


def control_number(h, u, v, dx, dy=None, timestep=1.0, precision="f64"):
    """SaintVenantState::max_control_number through the reference's reduction kernel."""
    lib = load()
    dt_, ct = _np(precision)
    dy = dx if dy is None else dy
    ny, nx = h.shape
    a = [np.ascontiguousarray(x, dtype=dt_) for x in (h, u, v)]
    cn = (ct * 1)()
    r = getattr(lib, f"refpin_control_number_{precision}")(nx, ny, dx, dy, *[_ptr(x, ct) for x in a], timestep, cn)
    if r != 0:
        raise RuntimeError("reference kernels failed")
    return cn[0]


def update_y(u0, ks, a, timestep, dx=1.0, dy=None, precision="f64"):
    """RungeKuttaSolver::update_y through the SaintVenantState operators: u0 is (3, ny, nx), ks a
    list of (3, ny, nx) stage derivatives, a their coefficients a(s+1, col+1)."""
    lib = load()
    dt_, ct = _np(precision)
    dy = dx if dy is None else dy
    _, ny, nx = u0.shape
    U0 = np.ascontiguousarray(u0, dtype=dt_)
    K = np.ascontiguousarray(np.stack(ks) if len(ks) else np.zeros((0, 3, ny, nx)), dtype=dt_)
    A = (C.c_double * max(1, len(a)))(*a)
    y = np.empty_like(U0)
    r = getattr(lib, f"refpin_update_y_{precision}")(nx, ny, dx, dy, _ptr(U0, ct), _ptr(K, ct), len(ks), A, timestep,
                                                    _ptr(y, ct))
    if r != 0:
        raise RuntimeError("reference kernels failed")
    return y


def solve(z, h, u, v, dx, dy=None, manning=None, rain=None, head_edges=0, head_value=0.0, head_first=False,
          rk_method="classic", start=0.0, end=60.0, step_length=60.0, initial_dt=1.0, precision="f64"):
    """RungeKuttaSolver::solve of the reference (control-number target 1.0, as it hard-codes)
    over [start, end]: manning = (n_shallow, n_deep, d_shallow, d_deep) uniform values, rain =
    (times, values) of a rain time series in m/s applied everywhere, head_edges the SV_EDGE_*
    strips held at head_value. Returns (h, u, v, number of timesteps taken)."""
    lib = load()
    dt_, ct = _np(precision)
    dy = dx if dy is None else dy
    ny, nx = h.shape
    ins = [np.ascontiguousarray(a, dtype=dt_) for a in (z, h, u, v)]
    man = None if manning is None else (C.c_double * 4)(*manning)
    rt, rv, nr = None, None, 0
    if rain is not None:
        nr = len(rain[0])
        rt = (C.c_double * nr)(*rain[0])
        rv = (C.c_double * nr)(*rain[1])
    out = np.empty((3, ny, nx), dtype=dt_)
    n = C.c_uint64()
    r = getattr(lib, f"refpin_solve_{precision}")(nx, ny, dx, dy, *[_ptr(a, ct) for a in ins], man, rt, rv, nr,
                                                  int(head_edges), float(head_value), 1 if head_first else 0,
                                                  rk_method.encode(), start, end, step_length, initial_dt,
                                                  _ptr(out, ct), C.byref(n))
    if r != 0:
        raise RuntimeError("reference solve failed")
    return out[0], out[1], out[2], n.value


class RefReaderError(RuntimeError):
    """The reference's reader threw; the message is its exception's."""


_nimrod = None


def _load_nimrod():
    global _nimrod
    if _nimrod is None:
        _nimrod = C.CDLL(_build_module().build_nimrod())
        f = _nimrod.refpin_nimrod_read
        f.restype = C.c_int
        D = C.POINTER(C.c_double)
        f.argtypes = [C.c_char_p, D, C.POINTER(C.c_int16), C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_char_p,
                      C.POINTER(C.c_int16), C.POINTER(C.c_uint64), D, D, D, D, C.c_uint64, D, C.c_uint64, C.c_char_p,
                      C.c_uint64]
    return _nimrod


def nimrod_read(path, bbox=None):
    """The reference's NIMRODRasterFormat<double> on the file at `path` (bbox = xmin, ymin, xmax,
    ymax or None). Returns a dict: h1..h5 (header arrays), nxpx, nypx, ulc (x, y) and lrc (x, y)
    pixel corners, ncols, nrows (of the crop), buffer (the whole grid, nypx x nxpx, file order,
    north row first), values (values_, flat, the crop row by row from the north), geo (the
    geotransform), llc (the reader's llc()) and nodata. Raises RefReaderError when the reader
    throws."""
    lib = _load_nimrod()
    bb = None if bbox is None else (C.c_double * 4)(*[float(b) for b in bbox])
    err = C.create_string_buffer(512)
    dims = (C.c_uint64 * 9)()
    h1, h5 = (C.c_int16 * 31)(), (C.c_int16 * 51)()
    h2, h3 = (C.c_float * 28)(), (C.c_float * 45)()
    h4 = C.create_string_buffer(56)
    geo, llc, nod = (C.c_double * 6)(), (C.c_double * 2)(), (C.c_double * 1)()
    r = lib.refpin_nimrod_read(os.fsencode(path), bb, h1, h2, h3, h4, h5, dims, geo, llc, nod, None, 0, None, 0,
                               err, len(err))
    if r == 1:
        raise RefReaderError(err.value.decode(errors="replace"))
    nxpx, nypx, nval = int(dims[0]), int(dims[1]), int(dims[8])
    buf = np.empty(nxpx * nypx, dtype=np.float64)
    val = np.empty(max(1, nval), dtype=np.float64)
    r = lib.refpin_nimrod_read(os.fsencode(path), bb, None, None, None, None, None, None, None, None, None,
                               _ptr(buf, C.c_double), buf.size, _ptr(val, C.c_double), val.size, err, len(err))
    if r != 0:
        raise RefReaderError(f"second read failed ({r}): {err.value.decode(errors='replace')}")
    return {"h1": list(h1), "h2": list(h2), "h3": list(h3), "h4": h4.raw, "h5": list(h5), "nxpx": nxpx, "nypx": nypx,
            "ulc": (int(dims[2]), int(dims[3])), "lrc": (int(dims[4]), int(dims[5])), "ncols": int(dims[6]),
            "nrows": int(dims[7]), "buffer": buf.reshape(nypx, nxpx), "values": val[:nval], "geo": list(geo),
            "llc": (llc[0], llc[1]), "nodata": nod[0]}


_ts = None


def _load_ts():
    global _ts
    if _ts is None:
        _ts = C.CDLL(_build_module().build_ts())
        S = C.POINTER(C.c_char_p)
        D = C.POINTER(C.c_double)
        f = _ts.refpin_ts_load
        f.restype = C.c_int
        f.argtypes = [S, S, C.c_int, S, S, C.c_int, S, S, C.c_int, D, D, C.c_uint64, C.POINTER(C.c_uint64),
                      C.c_char_p, C.c_uint64]
        f = _ts.refpin_ts_at
        f.restype = C.c_int
        f.argtypes = [D, D, C.c_uint64, D, C.c_uint64, D]
    return _ts


def _strings(items):
    items = list(items)
    return (C.c_char_p * max(1, len(items)))(*[str(x).encode() for x in items]), len(items)


def ts_load(section, data=None, transform=None):
    """TimeSeries<double, double>::load of the reference on a "time series" section given as
    key -> value strings (`source`, `filename`, `separator`, `headers`, ...), the inline data
    as (time string, value string) pairs, and the transform section's keys. Returns (times,
    values); raises RefReaderError when the reader throws."""
    lib = _load_ts()
    k, nk = _strings(section.keys())
    v, _ = _strings(section.values())
    data = list(data or [])
    dk, nd = _strings(d[0] for d in data)
    dv, _ = _strings(d[1] for d in data)
    transform = dict(transform or {})
    tk, nt = _strings(transform.keys())
    tv, _ = _strings(transform.values())
    err = C.create_string_buffer(512)
    n = C.c_uint64()
    cap = 1 << 16
    t = np.empty(cap)
    x = np.empty(cap)
    r = lib.refpin_ts_load(k, v, nk, dk, dv, nd, tk, tv, nt, _ptr(t, C.c_double), _ptr(x, C.c_double), cap,
                           C.byref(n), err, len(err))
    if r != 0:
        raise RefReaderError(err.value.decode(errors="replace"))
    m = min(n.value, cap)
    return t[:m].copy(), x[:m].copy()


def ts_at(times, values, queries):
    """TimeSeries<double, double>::at (ts_linterp) of the reference at each query time (each
    below the last knot)."""
    lib = _load_ts()
    t = np.ascontiguousarray(times, dtype=np.float64)
    v = np.ascontiguousarray(values, dtype=np.float64)
    q = np.ascontiguousarray(queries, dtype=np.float64)
    out = np.empty_like(q)
    if lib.refpin_ts_at(_ptr(t, C.c_double), _ptr(v, C.c_double), len(t), _ptr(q, C.c_double), len(q),
                        _ptr(out, C.c_double)) != 0:
        raise RuntimeError("reference time series failed")
    return out
