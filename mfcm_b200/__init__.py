"""mfcm_b200: B200-native 2-D Saint-Venant explicit Runge-Kutta time step.

Python host mirror of the reference's solver interface (oojimaflib/mfcm):
  SaintVenantSolver   SaintVenantSolver<TT,T,Cartesian2DMesh> + RungeKuttaSolver
                      (src/SaintVenant/Solver.hpp:30-172, src/TemporalScheme/RungeKutta.hpp:268-463)
  solve()             TypedTemporalScheme::solve (src/TemporalScheme/TemporalScheme.hpp:244-276)
  TimeSeries          TimeSeries::at / ts_linterp (src/Input/TimeSeries.cpp:26-47, :107-115)
  num_steps()         TimeParameters::num_steps (src/Config/TimeParameters.cpp:40-58)

All numerical work runs in libsv_b200.so (CUDA, sm_100a) through the C-ABI of include/sv.h;
importing this package without the built library raises instead of falling back to the CPU.
"""
import ctypes as C
import os

import numpy as np

from . import _abi
from ._abi import (FIELD, FACE_FIELDS, RK_METHODS, RK_STAGES, Forcing, MeshDesc, Params, Stats,
                   RAIN_NONE, RAIN_UNIFORM, RAIN_FIELDS, RAIN_PATTERN, HEAD_NONE, HEAD_EDGES,
                   HEAD_FIELDS, STAGE_EDGES, STAGE_FIELDS, EDGE_XMIN, EDGE_XMAX, EDGE_YMIN, EDGE_YMAX,
                   SV_F32, SV_F64, SV_F32_DATUM64)

__all__ = ["SaintVenantSolver", "SvError", "TimeSeries", "solve", "num_steps", "load_library",
           "FIELD", "Forcing", "RK_METHODS", "RAIN_NONE", "RAIN_UNIFORM", "RAIN_FIELDS",
           "RAIN_PATTERN", "HEAD_NONE", "HEAD_EDGES", "HEAD_FIELDS", "STAGE_EDGES", "STAGE_FIELDS",
           "EDGE_XMIN", "EDGE_XMAX", "EDGE_YMIN", "EDGE_YMAX"]

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib", "libsv_b200.so")
_lib = None


class SvError(RuntimeError):
    """A non-zero status from the C-ABI (the reference raises std::runtime_error)."""

    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


def load_library(path=None):
    """Load libsv_b200.so (built in-tree by mfcm_b200/build.py)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: build it with `python mfcm_b200/build.py`")
    lib = C.CDLL(p)
    _abi.declare(lib, "sv_")
    lib.sv_create.restype = C.c_int
    lib.sv_create.argtypes = [C.POINTER(MeshDesc), C.POINTER(Params), C.c_int, C.POINTER(C.c_void_p)]
    lib.sv_destroy.restype = None
    lib.sv_destroy.argtypes = [C.c_void_p]
    lib.sv_last_error.restype = C.c_char_p
    lib.sv_last_error.argtypes = [C.c_void_p]
    lib.sv_last_advance_ms.restype = C.c_int
    lib.sv_last_advance_ms.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
    lib.sv_set_kernel_variant.restype = C.c_int
    lib.sv_set_kernel_variant.argtypes = [C.c_void_p, C.c_int]
    for name in ("sv_get_kernel_variant", "sv_autotune"):
        getattr(lib, name).restype = C.c_int
        getattr(lib, name).argtypes = [C.c_void_p, C.POINTER(C.c_int)]
    lib.sv_get_autotune_ms.restype = C.c_int
    lib.sv_get_autotune_ms.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.c_int]
    lib.sv_run_timesteps.restype = C.c_int
    lib.sv_run_timesteps.argtypes = [C.c_void_p, C.c_uint64, C.c_int, C.POINTER(Stats), C.POINTER(C.c_int),
                                     C.POINTER(_abi.Timing)]
    if path is None:
        _lib = lib
    return lib


def _field_id(f):
    return FIELD[f.upper()] if isinstance(f, str) else int(f)


class _Backend:
    """Methods shared by the CUDA solver and the CPU oracle (same C-ABI shape)."""
    _prefix = "sv_"

    def _call(self, name, *args):
        r = getattr(self._lib, self._prefix + name)(self._h, *args)
        if r != 0:
            raise SvError(r, self.last_error())
        return r

    def field_size(self, fid):
        return self.nfaces if fid in FACE_FIELDS else self.ncells

    def set_field(self, field, values):
        fid = _field_id(field)
        a = np.ascontiguousarray(np.asarray(values, dtype=np.float64).reshape(-1))
        self._call("set_field", fid, a.ctypes.data_as(C.POINTER(C.c_double)), a.size)

    def get_field(self, field, out=None):
        """A field as FP64. `out`, a C-contiguous float64 array of the field's size (pinned
        host memory, for one DMA copy), receives it in place of a new array."""
        fid = _field_id(field)
        n = self.field_size(fid)
        if out is None:
            a = np.empty(n, dtype=np.float64)
        else:
            if out.dtype != np.float64 or out.size != n or not out.flags["C_CONTIGUOUS"]:
                raise ValueError(f"out must be a C-contiguous float64 array of {n} values")
            a = out.reshape(-1)
        self._call("get_field", fid, a.ctypes.data_as(C.POINTER(C.c_double)), n)
        return a if fid in FACE_FIELDS else a.reshape(self.ny, self.nx)

    def set_manning(self, n_shallow=0.03, n_deep=0.3, d_shallow=0.1, d_deep=0.3):
        """ManningRoughnessSourceTerm defaults (ManningRoughnessSourceTerm.cpp:99-102)."""
        self._call("set_manning", float(n_shallow), float(n_deep), float(d_shallow), float(d_deep))

    def set_eddy_viscosity(self, mode="constant", mu=1.0, mu_const=0.05, mu_smag=0.5):
        """EddyViscositySourceTerm (EddyViscositySourceTerm.cpp:112-137): mode "off",
        "constant" (the EDDY_MU field when set, else `mu`, "default mu") or "smagorinsky"
        (mu_const + mu_smag * cell area * |strain|, "constant coefficient" and "dynamic
        coefficient"); defaults are the reference's."""
        if mode not in _abi.EDDY_MODES:
            raise ValueError(f"unknown eddy viscosity mode {mode!r}")
        self._call("set_eddy_viscosity", _abi.EDDY_MODES[mode], float(mu), float(mu_const), float(mu_smag))

    def set_source_order(self, terms):
        """Configuration order of the momentum source terms, names from "manning", "energy
        loss" and "eddy viscosity" (each adds to du/dt, so the order sets the rounding)."""
        codes = [_abi.TERMS[t] for t in terms]
        arr = (C.c_int * max(1, len(codes)))(*codes)
        self._call("set_source_order", arr, len(codes))

    def set_forcing(self, forcing):
        self._call("set_forcing", C.byref(forcing))

    def set_dt(self, dt):
        self._call("set_dt", float(dt))

    def get_dt(self):
        v = C.c_double()
        self._call("get_dt", C.byref(v))
        return v.value

    def eval_dudt(self, state_no, t_sub, dt):
        self._call("eval_dudt", int(state_no), float(t_sub), float(dt))

    def do_timestep(self, t_local, dt):
        cn, rep, nd = C.c_double(), C.c_int(), C.c_double()
        self._call("do_timestep", float(t_local), float(dt), C.byref(cn), C.byref(rep), C.byref(nd))
        return cn.value, bool(rep.value), nd.value

    def accept(self):
        self._call("accept")

    def advance(self):
        s = Stats()
        self._call("advance", C.byref(s))
        return s.as_dict()

    def stats(self):
        s = Stats()
        self._call("get_stats", C.byref(s))
        return s.as_dict()

    def set_stats(self, st):
        """Restore the running counters and tallies (a checkpoint's); volume is recomputed."""
        s = Stats(int(st["accepted"]), int(st["repeated"]), 0.0, float(st["rain_in"]), float(st["outflow"]),
                  float(st.get("wall_in", 0.0)))
        self._call("set_stats", C.byref(s))


class SaintVenantSolver(_Backend):
    """One catchment on one GPU: SaintVenantSolver + RungeKuttaSolver behind the C-ABI.

    precision: "f64" (bit-for-bit the reference arithmetic at T = double) or "f32".
    rain_mode: "reference" keeps the discharge boundary's clamp exactly as written
    (DischargeBoundarySourceTerm.cpp:62-64); "physical" applies it only when the rate would
    make the depth negative.
    """

    def __init__(self, nx, ny, dx, dy=None, precision="f64", rk_method="classic", cn_target=1.0,
                 step_duration=60.0, initial_dt=1.0, max_dt=0.0, rain_mode="reference", manning=True,
                 head_first=False, tallies=True, device=0, eloss_first=False):
        self._lib = load_library()
        self.nx, self.ny = int(nx), int(ny)
        self.dx = float(dx)
        self.dy = float(dx if dy is None else dy)
        self.ncells = self.nx * self.ny
        self.nfaces = (self.nx + 1) * self.ny + (self.ny + 1) * self.nx
        self.step_duration = float(step_duration)
        self.precision = precision
        self.depth_compensation = precision != "f64"  # FP32 depth updates carry a compensation
        self.rk_method = rk_method
        self.nstages = RK_STAGES[RK_METHODS.index(rk_method)]
        m = MeshDesc(self.nx, self.ny, self.dx, self.dy, 0.0, 0.0)
        p = Params(_precision_code(precision), RK_METHODS.index(rk_method), float(cn_target),
                   self.step_duration, float(initial_dt), float(max_dt),
                   0 if rain_mode == "reference" else 1, 1 if manning else 0, 1 if head_first else 0,
                   _flags(tallies, eloss_first))
        h = C.c_void_p()
        r = self._lib.sv_create(C.byref(m), C.byref(p), int(device), C.byref(h))
        if r != 0:
            raise SvError(r, self._lib.sv_last_error(None).decode())
        self._h = h

    def last_error(self):
        return self._lib.sv_last_error(self._h).decode()

    def run_timesteps(self, max_timesteps, begin=False, timing=False):
        """Up to `max_timesteps` device-controlled timesteps of the current step (part of
        TypedTemporalScheme::step); returns (running stats, step finished?, timing or None)."""
        s = Stats()
        done = C.c_int()
        t = _abi.Timing() if timing else None
        r = self._lib.sv_run_timesteps(self._h, int(max_timesteps), 1 if begin else 0, C.byref(s), C.byref(done),
                                       C.byref(t) if t is not None else None)
        if r != 0:
            raise SvError(r, self.last_error())
        return s.as_dict(), bool(done.value), (t.as_dict() if t is not None else None)

    def set_kernel_variant(self, variant):
        r = self._lib.sv_set_kernel_variant(self._h, int(variant))
        if r != 0:
            raise SvError(r, self.last_error())

    def kernel_variant(self):
        v = C.c_int()
        self._lib.sv_get_kernel_variant(self._h, C.byref(v))
        return v.value

    def autotune(self):
        """Time every stage-kernel variant on the current state; keep the fastest."""
        v = C.c_int()
        r = self._lib.sv_autotune(self._h, C.byref(v))
        if r != 0:
            raise SvError(r, self.last_error())
        return v.value

    def autotune_ms(self, n=16):
        """Per-variant stage-kernel times (ms) measured by the last autotune (0 = untimed)."""
        a = (C.c_float * n)()
        self._lib.sv_get_autotune_ms(self._h, a, n)
        return {v: float(a[v]) for v in range(n) if a[v] > 0}

    def last_advance_ms(self):
        v = C.c_double()
        self._lib.sv_last_advance_ms(self._h, C.byref(v))
        return v.value

    def close(self):
        if getattr(self, "_h", None):
            self._lib.sv_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _precision_code(p):
    return {"f64": SV_F64, "f32": SV_F32, "f32_datum64": SV_F32_DATUM64}[p]


class TimeSeries:
    """TimeSeries<double,double>::at with ts_linterp (src/Input/TimeSeries.cpp:26-47).

    At or beyond the last knot the reference reads past the end of its arrays; here the last
    segment is extrapolated (the same choice as the oracle)."""

    def __init__(self, times, values):
        self.t = [float(x) for x in times]
        self.v = [float(x) for x in values]
        if len(self.t) < 2 or len(self.t) != len(self.v):
            raise ValueError("a time series needs at least two (time, value) knots")

    def at(self, time):
        i1 = 1
        while i1 < len(self.t):
            if self.t[i1] > time:
                break
            i1 += 1
        if i1 >= len(self.t):
            i1 = len(self.t) - 1
        i0 = i1 - 1
        t0, t1, v0, v1 = self.t[i0], self.t[i1], self.v[i0], self.v[i1]
        dvdt = (v1 - v0) / (t1 - t0)
        return v0 + dvdt * (time - t0)


def num_steps(start_time, end_time, step_duration):
    """TimeParameters::num_steps (src/Config/TimeParameters.cpp:40-58)."""
    eps = 1e-6
    sim = end_time - start_time
    n = int(sim / step_duration)
    if step_duration * n >= sim - eps and step_duration * n <= sim + eps:
        return n
    return n + 1


def _flags(tallies=True, eloss_first=False):
    return (0 if tallies else _abi.SV_FLAG_NO_TALLIES) | (_abi.SV_FLAG_ELOSS_FIRST if eloss_first else 0)


def start_new_step_forcing(t, L, rain=None, rain_kind=RAIN_UNIFORM, head=None, head_edges=0,
                           head_kind=HEAD_EDGES):
    """Boundary values for [t, t + L] (DischargeBoundarySourceTerm.hpp:114-146,
    HeadBoundarySourceTerm.hpp:114-146): rain / head are TimeSeries, constants or None;
    head_kind STAGE_EDGES reads `head` as water levels (a stage boundary)."""
    f = Forcing()
    if rain is not None:
        q0, q1 = (rain.at(t), rain.at(t + L)) if isinstance(rain, TimeSeries) else (float(rain), float(rain))
        f.rain_kind, f.rain_q0, f.rain_q1 = rain_kind, q0, q1
    if head is not None:
        h0, h1 = (head.at(t), head.at(t + L)) if isinstance(head, TimeSeries) else (float(head), float(head))
        f.head_kind, f.head_edges, f.head_h0, f.head_h1 = head_kind, head_edges, h0, h1
    return f


def solve(solver, start_time, end_time, rain=None, rain_kind=RAIN_UNIFORM, head=None, head_edges=0,
          on_step=None):
    """TypedTemporalScheme::solve: for each step of length L, outputs at its start
    (end_of_step + do_outputs via on_step), start_new_step, then the adaptive-dt inner loop."""
    L = solver.step_duration
    n = num_steps(start_time, end_time, L)
    per_step = []
    for i in range(n):
        t = start_time + i * L
        if on_step:
            on_step(t, solver)
        solver.set_forcing(start_new_step_forcing(t, L, rain, rain_kind, head, head_edges))
        per_step.append(solver.advance())
    if on_step:
        on_step(start_time + n * L, solver)
    return per_step
