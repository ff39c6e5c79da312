"""TEST INFRASTRUCTURE: Python binding of the CPU oracle (oracle/_build/libsv_oracle*.so).

Only tests/, the smoke check and bench.py's CPU-baseline leg may import this module. The
class exposes the same methods as mfcm_b200.SaintVenantSolver so one scenario script can run
against both.
"""
import ctypes as C
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(_HERE))

from mfcm_b200 import _abi  # noqa: E402
from mfcm_b200 import _Backend, RK_METHODS, RK_STAGES, _precision_code  # noqa: E402

_libs = {}


def load(openmp=False):
    key = "omp" if openmp else "serial"
    if key in _libs:
        return _libs[key]
    import importlib.util
    spec = importlib.util.spec_from_file_location("sv_oracle_build", os.path.join(_HERE, "build.py"))
    _b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(_b)
    paths = _b.build()
    lib = C.CDLL(paths[key])
    _abi.declare(lib, "svo_")
    lib.svo_create.restype = C.c_int
    lib.svo_create.argtypes = [C.POINTER(_abi.MeshDesc), C.POINTER(_abi.Params), C.POINTER(C.c_void_p)]
    lib.svo_destroy.restype = None
    lib.svo_destroy.argtypes = [C.c_void_p]
    lib.svo_last_error.restype = C.c_char_p
    lib.svo_last_error.argtypes = []
    lib.svo_set_threads.restype = C.c_int
    lib.svo_set_threads.argtypes = [C.c_int]
    lib.svo_pow43.restype = C.c_double
    lib.svo_pow43.argtypes = [C.c_double]
    lib.svo_minmod3.restype = C.c_double
    lib.svo_minmod3.argtypes = [C.c_double] * 5
    lib.svo_minmod3f.restype = C.c_float
    lib.svo_minmod3f.argtypes = [C.c_float, C.c_double, C.c_float, C.c_double, C.c_float]
    _libs[key] = lib
    return lib


class OracleSolver(_Backend):
    """CPU restatement of SaintVenantSolver + RungeKuttaSolver (precision f64 or f32)."""
    _prefix = "svo_"

    def __init__(self, nx, ny, dx, dy=None, precision="f64", rk_method="classic", cn_target=1.0,
                 step_duration=60.0, initial_dt=1.0, max_dt=0.0, rain_mode="reference", manning=True,
                 head_first=False, tallies=True, openmp=False, threads=0, eloss_first=False):
        self._lib = load(openmp)
        if openmp and threads:
            self._lib.svo_set_threads(int(threads))
        self.nx, self.ny = int(nx), int(ny)
        self.dx = float(dx)
        self.dy = float(dx if dy is None else dy)
        self.ncells = self.nx * self.ny
        self.precision = precision
        self.nfaces = (self.nx + 1) * self.ny + (self.ny + 1) * self.nx
        self.step_duration = float(step_duration)
        self.nstages = RK_STAGES[RK_METHODS.index(rk_method)]
        m = _abi.MeshDesc(self.nx, self.ny, self.dx, self.dy, 0.0, 0.0)
        p = _abi.Params(_precision_code(precision), RK_METHODS.index(rk_method), float(cn_target),
                        self.step_duration, float(initial_dt), float(max_dt),
                        0 if rain_mode == "reference" else 1, 1 if manning else 0, 1 if head_first else 0,
                        (0 if tallies else _abi.SV_FLAG_NO_TALLIES) |
                        (_abi.SV_FLAG_ELOSS_FIRST if eloss_first else 0))
        h = C.c_void_p()
        r = self._lib.svo_create(C.byref(m), C.byref(p), C.byref(h))
        if r != 0:
            raise RuntimeError(self._lib.svo_last_error().decode())
        self._h = h

    def last_error(self):
        return self._lib.svo_last_error().decode()

    def close(self):
        if getattr(self, "_h", None):
            self._lib.svo_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pow43(x):
    return load().svo_pow43(float(x))


def minmod3(ul, dxl, uc, dxr, ur, precision="f64"):
    lib = load()
    if precision == "f64":
        return lib.svo_minmod3(ul, dxl, uc, dxr, ur)
    return lib.svo_minmod3f(ul, dxl, uc, dxr, ur)


def threads_available(openmp=True):
    return load(openmp).svo_set_threads(0)
