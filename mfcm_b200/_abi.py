"""ctypes mirror of include/sv.h (structs, constants and prototypes)."""
import ctypes as C

SV_OK = 0
SV_E_ARG = -1
SV_E_CUDA = -2
SV_E_NOMEM = -3
SV_E_STATE = -4
SV_E_NONFINITE = -5
SV_E_TIMEOUT = -6
SV_E_LIMIT = -7

SV_F32 = 1
SV_F64 = 2
SV_F32_DATUM64 = 3

SV_FLAG_NO_TALLIES = 1
SV_FLAG_ELOSS_FIRST = 2

RK_METHODS = ["euler", "midpoint", "heun2", "ralston2", "kutta3", "heun3", "wray3", "ralston3",
              "ssprk3", "classic", "ralston4", "3/8rule"]
RK_STAGES = [1, 2, 2, 2, 3, 3, 3, 3, 3, 4, 4, 4]

FIELD = dict(
    Z=0, H=1, U=2, V=3, N_SHALLOW=4, N_DEEP=5, D_SHALLOW=6, D_DEEP=7, QBDY0=8, QBDY1=9,
    HBDY0=10, HBDY1=11, RAIN_PATTERN=12, INFIL_RATE=13, INFIL_CAP=14, ELOSS_FX=15, ELOSS_FY=16, H_COMP=17, EDDY_MU=18, DHDT=20, DUDT=21, DVDT=22, DHDX=23, DUDX=24, DVDX=25,
    DHDY=26, DUDY=27, DVDY=28, DZDX=29, DZDY=30, FLUX_H=40, FLUX_U=41, FLUX_V=42, FLUX_Z=43,
    FLUX_BRANCH=44, STATE_BASE=100, K_BASE=200,
)
FACE_FIELDS = {40, 41, 42, 43, 44}

RAIN_NONE, RAIN_UNIFORM, RAIN_FIELDS, RAIN_PATTERN = 0, 1, 2, 3
HEAD_NONE, HEAD_EDGES, HEAD_FIELDS, STAGE_EDGES, STAGE_FIELDS = 0, 1, 2, 3, 4
EDGE_XMIN, EDGE_XMAX, EDGE_YMIN, EDGE_YMAX = 1, 2, 4, 8
EDDY_MODES = {"off": 0, "constant": 1, "smagorinsky": 2}
TERMS = {"manning": 1, "energy loss": 2, "eddy viscosity": 3}


class MeshDesc(C.Structure):
    _fields_ = [("nx", C.c_uint64), ("ny", C.c_uint64), ("dx", C.c_double), ("dy", C.c_double),
                ("origin_x", C.c_double), ("origin_y", C.c_double)]


class Params(C.Structure):
    _fields_ = [("precision", C.c_int), ("rk_method", C.c_int), ("cn_target", C.c_double),
                ("step_duration", C.c_double), ("initial_dt", C.c_double), ("max_dt", C.c_double),
                ("rain_mode", C.c_int), ("manning", C.c_int), ("head_first", C.c_int), ("flags", C.c_int)]


class Forcing(C.Structure):
    _fields_ = [("rain_kind", C.c_int), ("rain_q0", C.c_double), ("rain_q1", C.c_double),
                ("head_kind", C.c_int), ("head_edges", C.c_uint), ("head_h0", C.c_double),
                ("head_h1", C.c_double)]


class Stats(C.Structure):
    _fields_ = [("accepted", C.c_uint64), ("repeated", C.c_uint64), ("volume", C.c_double),
                ("rain_in", C.c_double), ("outflow", C.c_double), ("wall_in", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Timing(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("stage_ms", C.c_double), ("finalize_ms", C.c_double),
                ("stage_launches", C.c_uint64), ("finalize_launches", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def declare(lib, prefix, ctx_type=C.c_void_p):
    """Declare the sv_* (or svo_*) prototypes on a loaded library."""
    P = C.POINTER
    d = C.c_double
    sig = {
        "set_field": (C.c_int, [ctx_type, C.c_int, P(d), C.c_uint64]),
        "get_field": (C.c_int, [ctx_type, C.c_int, P(d), C.c_uint64]),
        "set_manning": (C.c_int, [ctx_type, d, d, d, d]),
        "set_forcing": (C.c_int, [ctx_type, P(Forcing)]),
        "set_dt": (C.c_int, [ctx_type, d]),
        "get_dt": (C.c_int, [ctx_type, P(d)]),
        "eval_dudt": (C.c_int, [ctx_type, C.c_int, d, d]),
        "do_timestep": (C.c_int, [ctx_type, d, d, P(d), P(C.c_int), P(d)]),
        "accept": (C.c_int, [ctx_type]),
        "advance": (C.c_int, [ctx_type, P(Stats)]),
        "get_stats": (C.c_int, [ctx_type, P(Stats)]),
        "set_stats": (C.c_int, [ctx_type, P(Stats)]),
        "set_eddy_viscosity": (C.c_int, [ctx_type, C.c_int, d, d, d]),
        "set_source_order": (C.c_int, [ctx_type, P(C.c_int), C.c_int]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, prefix + name)
        f.restype = res
        f.argtypes = args
