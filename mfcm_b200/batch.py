"""Batches of independent catchments advanced in shared launches (sv_batch_* in include/sv.h).

The reference runs one catchment per process; here many uneven catchments advance together:
per timestep one batched launch per RK stage covers every member's tiles and one batched
launch runs every member's reductions and dt controller. Each member keeps its own dt, step
clock and tallies, so its results are bit-identical to running it alone.
"""
import ctypes as C

from . import _abi, load_library, SvError, _Backend, _precision_code, _flags, RK_METHODS, RK_STAGES
from ._abi import MeshDesc, Params, Stats


def _declare(lib):
    if getattr(lib, "_batch_declared", False):
        return
    P = C.POINTER
    lib.sv_batch_create.restype = C.c_int
    lib.sv_batch_create.argtypes = [C.c_int, C.c_int, C.c_int, P(C.c_void_p)]
    lib.sv_batch_destroy.restype = None
    lib.sv_batch_destroy.argtypes = [C.c_void_p]
    lib.sv_batch_add.restype = C.c_int
    lib.sv_batch_add.argtypes = [C.c_void_p, P(MeshDesc), P(Params), P(C.c_int)]
    lib.sv_batch_adopt.restype = C.c_int
    lib.sv_batch_adopt.argtypes = [C.c_void_p, C.c_void_p, P(C.c_int)]
    lib.sv_batch_remove.restype = C.c_int
    lib.sv_batch_remove.argtypes = [C.c_void_p, C.c_int]
    lib.sv_batch_member.restype = C.c_void_p
    lib.sv_batch_member.argtypes = [C.c_void_p, C.c_int]
    lib.sv_batch_advance.restype = C.c_int
    lib.sv_batch_advance.argtypes = [C.c_void_p, P(Stats), C.c_int]
    lib.sv_batch_set_step_limit.restype = C.c_int
    lib.sv_batch_set_step_limit.argtypes = [C.c_void_p, C.c_longlong]
    lib.sv_batch_advance_steps.restype = C.c_int
    lib.sv_batch_advance_steps.argtypes = [C.c_void_p, C.c_int, P(C.c_int), P(_abi.Forcing), P(Stats), C.c_int]
    lib.sv_batch_kernel_variant.restype = C.c_int
    lib.sv_batch_kernel_variant.argtypes = [C.c_void_p, P(C.c_int)]
    lib.sv_batch_status.restype = C.c_int
    lib.sv_batch_status.argtypes = [C.c_void_p, P(C.c_int), C.c_int]
    lib.sv_batch_set_persistent.restype = C.c_int
    lib.sv_batch_set_persistent.argtypes = [C.c_void_p, C.c_int, C.c_uint64, C.c_double]
    lib.sv_batch_size.restype = C.c_int
    lib.sv_batch_size.argtypes = [C.c_void_p, P(C.c_int), P(C.c_uint64)]
    lib._batch_declared = True


class BatchMember(_Backend):
    """One catchment of a batch: the usual field / forcing / stats calls on its context."""

    def __init__(self, batch, slot, nx, ny, dx, dy, step_duration, nstages):
        self._lib = batch._lib
        self._batch = batch
        self.slot = slot
        self._h = C.c_void_p(batch._lib.sv_batch_member(batch._b, slot))
        self.nx, self.ny, self.dx, self.dy = nx, ny, dx, dy
        self.ncells = nx * ny
        self.nfaces = (nx + 1) * ny + (ny + 1) * nx
        self.step_duration = step_duration
        self.nstages = nstages

    def last_error(self):
        return self._lib.sv_last_error(self._h).decode()


MAX_STEPS = 16  # SV_BATCH_MAX_STEPS


class SaintVenantBatch:
    def __init__(self, precision="f64", rk_method="classic", device=0):
        self._lib = load_library()
        _declare(self._lib)
        self.precision = precision
        self.rk_method = rk_method
        h = C.c_void_p()
        r = self._lib.sv_batch_create(_precision_code(precision), RK_METHODS.index(rk_method), int(device), C.byref(h))
        if r != 0:
            raise SvError(r, self._lib.sv_last_error(None).decode())
        self._b = h
        self.members = {}

    def add(self, nx, ny, dx, dy=None, cn_target=1.0, step_duration=60.0, initial_dt=1.0, max_dt=0.0,
            rain_mode="reference", manning=True, head_first=False, tallies=True, eloss_first=False):
        dy = float(dx if dy is None else dy)
        m = MeshDesc(int(nx), int(ny), float(dx), dy, 0.0, 0.0)
        p = Params(_precision_code(self.precision), RK_METHODS.index(self.rk_method), float(cn_target),
                   float(step_duration), float(initial_dt), float(max_dt), 0 if rain_mode == "reference" else 1,
                   1 if manning else 0, 1 if head_first else 0, _flags(tallies, eloss_first))
        slot = C.c_int()
        r = self._lib.sv_batch_add(self._b, C.byref(m), C.byref(p), C.byref(slot))
        if r != 0:
            raise SvError(r, self._lib.sv_last_error(None).decode())
        mem = BatchMember(self, slot.value, int(nx), int(ny), float(dx), dy, float(step_duration),
                          RK_STAGES[RK_METHODS.index(self.rk_method)])
        self.members[slot.value] = mem
        return mem

    def adopt(self, solver):
        """A SaintVenantSolver of this batch's precision, tableau and device, created and
        filled on its own (its uploads run on its own stream, so this can happen while the
        batch advances on another thread), joins the batch. The batch takes the solver's
        context over: `solver` is closed (its handle cleared) and the returned member is the
        catchment from now on. Not to be called while an advance of this batch runs."""
        if solver.precision != self.precision:
            raise ValueError(f"solver precision {solver.precision} differs from the batch's {self.precision}")
        slot = C.c_int()
        r = self._lib.sv_batch_adopt(self._b, solver._h, C.byref(slot))
        if r != 0:
            raise SvError(r, self._lib.sv_last_error(None).decode())
        solver._h = None  # owned by the batch now
        mem = BatchMember(self, slot.value, solver.nx, solver.ny, solver.dx, solver.dy, solver.step_duration,
                          solver.nstages)
        self.members[slot.value] = mem
        return mem

    def remove(self, member):
        r = self._lib.sv_batch_remove(self._b, member.slot)
        if r != 0:
            raise SvError(r, self._lib.sv_last_error(None).decode())
        self.members.pop(member.slot, None)
        member._h = None

    def set_step_limit(self, max_timesteps):
        """Cap the timesteps one member may take within one step (0: no cap). A member that
        reaches it leaves the step part-way with status SV_E_LIMIT; the others go on."""
        r = self._lib.sv_batch_set_step_limit(self._b, int(max_timesteps))
        if r != 0:
            raise SvError(r, self._lib.sv_last_error(None).decode())

    def set_persistent(self, on=True, spin_limit=0, max_seconds=0.0):
        """Run each advance as one persistent cooperative launch (every member at its own dt;
        idle warps take work from any member). The launch gives up with SV_E_TIMEOUT after
        spin_limit polls of a waiting warp with no work item completed anywhere, or after
        max_seconds of wall clock (0: the library's defaults)."""
        r = self._lib.sv_batch_set_persistent(self._b, 1 if on else 0, int(spin_limit), float(max_seconds))
        if r != 0:
            raise SvError(r, self._lib.sv_last_error(None).decode())

    def advance(self, raise_on_error=True):
        """One step (of each member's own step length) for every member; returns
        {slot: stats} with the step's counts, each member's running tallies and its
        "status" (0, SV_E_NONFINITE or SV_E_LIMIT). A failing member does not stop the
        others; with raise_on_error (the default) its failure still raises SvError after
        the step, otherwise it is only reported in its status."""
        n = max(self.members) + 1 if self.members else 0
        out = (Stats * max(n, 1))()
        r = self._lib.sv_batch_advance(self._b, out, n)
        if r != 0 and (raise_on_error or r not in (_abi.SV_E_NONFINITE, _abi.SV_E_LIMIT)):
            raise SvError(r, self._lib.sv_last_error(None).decode())
        status = (C.c_int * max(n, 1))()
        self._lib.sv_batch_status(self._b, status, n)
        res = {}
        for k in self.members:
            d = out[k].as_dict()
            d["status"] = status[k]
            res[k] = d
        return res

    def advance_steps(self, forcings, raise_on_error=True):
        """Several steps per call. `forcings` maps a member (or its slot) to the list of its
        steps' boundary values (Forcing, at most MAX_STEPS); members not listed sit the call
        out. Each member runs its steps back to back at its own pace, bit-identical to one
        advance() per step. Returns {slot: {"steps": [stats per step run], "status": s}}
        where a failed member's last entry is the step it failed in."""
        slots = {}
        for key, fl in forcings.items():
            slot = key.slot if isinstance(key, BatchMember) else int(key)
            if slot not in self.members:
                raise SvError(_abi.SV_E_ARG, f"no batch member in slot {slot}")
            slots[slot] = list(fl)
        n = max(self.members) + 1 if self.members else 0
        ms = max([len(v) for v in slots.values()] + [1])
        if ms > MAX_STEPS:
            raise SvError(_abi.SV_E_LIMIT, f"at most {MAX_STEPS} steps per batched advance")
        counts = (C.c_int * max(n, 1))()
        fa = (_abi.Forcing * (max(n, 1) * ms))()
        for slot, fl in slots.items():
            counts[slot] = len(fl)
            for k, f in enumerate(fl):
                fa[slot * ms + k] = f
        out = (Stats * (max(n, 1) * ms))()
        r = self._lib.sv_batch_advance_steps(self._b, ms, counts, fa, out, n)
        if r != 0 and (raise_on_error or r not in (_abi.SV_E_NONFINITE, _abi.SV_E_LIMIT)):
            raise SvError(r, self._lib.sv_last_error(None).decode())
        status = (C.c_int * max(n, 1))()
        self._lib.sv_batch_status(self._b, status, n)
        res = {}
        for slot in self.members:
            k = counts[slot] if slot < n else 0
            steps = [out[slot * ms + j].as_dict() for j in range(k)]
            if status[slot] != 0:  # the steps run, the last being the one it failed in
                while steps and steps[-1]["accepted"] == 0 and steps[-1]["repeated"] == 0:
                    steps.pop()
            res[slot] = {"steps": steps, "status": status[slot]}
        return res

    def kernel_variant(self):
        """The stage-kernel variant every member runs; a solo SaintVenantSolver with this
        variant reproduces a member's FP32 bits."""
        v = C.c_int()
        self._lib.sv_batch_kernel_variant(self._b, C.byref(v))
        return v.value

    def size(self):
        n, b = C.c_int(), C.c_uint64()
        self._lib.sv_batch_size(self._b, C.byref(n), C.byref(b))
        return n.value, b.value

    def close(self):
        if getattr(self, "_b", None):
            for m in self.members.values():
                m._h = None
            self._lib.sv_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
