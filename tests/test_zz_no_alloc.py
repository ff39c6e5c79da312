"""sv_timestep_noalloc: one timestep on caller-owned device buffers, with no device allocation.

This entry point serves callers that cannot allocate device memory once they are running --
a host framework that owns all device memory through its own pool, or a real-time loop in
which a cudaMalloc would synchronise the device. Its working memory is a fixed array inside
the library. The test checks it against the allocating solver (sv_create + sv_do_timestep),
bit for bit in FP64 like the other parity tests, on two calls in a row: the second call
starts from the first call's outputs and overwrites the array the first call left behind.
This file is named so that pytest collects it after every other test file.
"""
import ctypes as C

import numpy as np
import pytest

from mfcm_b200 import SaintVenantSolver, load_library, Forcing, MeshDesc, Params, EDGE_XMIN, EDGE_YMAX
from mfcm_b200._abi import SV_F64, SV_E_LIMIT, SV_E_ARG
from mfcm_b200._abi import RK_STAGES, RK_METHODS
from tests.scenarios import wet_dry_state, setup, same

MANNING = (0.03, 0.05, 0.1, 0.3)


def _bind():
    lib = load_library()
    f = lib.sv_timestep_noalloc
    f.restype = C.c_int
    P = C.POINTER
    f.argtypes = [P(MeshDesc), P(Params), P(C.c_double), P(Forcing)] + [C.c_void_p] * 7 + \
                 [C.c_double, C.c_double, C.c_void_p, C.c_void_p]
    return lib, f


def _params(rk=9, cn_target=0.5, step_duration=30.0):
    return Params(SV_F64, rk, cn_target, step_duration, 0.5, 0.0, 1, 1, 0, 0)


def _forcing():
    f = Forcing()
    f.rain_kind, f.rain_q0, f.rain_q1 = 1, 2e-5, 1e-5
    f.head_kind, f.head_edges, f.head_h0, f.head_h1 = 1, EDGE_XMIN | EDGE_YMAX, 0.01, 0.0
    return f


def _call(f, mesh, params, ptrs, result=5):
    man = (C.c_double * 4)(*MANNING)
    return f(C.byref(mesh), C.byref(params), man, C.byref(_forcing()), *[C.c_void_p(p) for p in ptrs],
             0.0, 0.1, C.c_void_p(result), None)


def test_noalloc_rejects_meshes_beyond_the_working_array():
    """No GPU needed: the size check comes before any CUDA call."""
    lib, f = _bind()
    r = _call(f, MeshDesc(257, 256, 1.0, 1.0, 0.0, 0.0), _params(), [16, 16, 16, 16, 1 << 40, 2 << 40, 3 << 40])
    assert r == SV_E_LIMIT
    assert "65536" in lib.sv_last_error(None).decode()


def test_noalloc_rejects_overlapping_outputs():
    """No GPU needed: outputs that overlap an input or each other by part of a field are refused
    before any CUDA call (fake, never dereferenced addresses)."""
    lib, f = _bind()
    mesh = MeshDesc(16, 16, 1.0, 1.0, 0.0, 0.0)
    nb = 16 * 16 * 8
    ins = [1 << 32, 2 << 32, 3 << 32, 4 << 32]
    outs = [5 << 32, 6 << 32, 7 << 32]
    assert _call(f, mesh, _params(), ins + [ins[1] + nb - 8, outs[1], outs[2]]) == SV_E_ARG
    assert "inputs" in lib.sv_last_error(None).decode()
    assert _call(f, mesh, _params(), ins + [outs[0], outs[0] + 8, outs[2]]) == SV_E_ARG
    assert "each other" in lib.sv_last_error(None).decode()
    assert _call(f, mesh, _params(rk=4), ins + outs) == SV_E_ARG  # kutta3 stores its k's


def _pair(nx, ny, dx, rk, seed):
    """Two timesteps in a row through sv_timestep_noalloc against the allocating solver (sv_create
    + sv_do_timestep + sv_accept), bit for bit; the second call starts from the first call's
    outputs and overwrites what the first call left in the working array."""
    import torch

    lib, f = _bind()
    z, h, u, v = wet_dry_state(nx, ny, dx, seed=seed)
    forcing = _forcing()

    g = SaintVenantSolver(nx, ny, dx, rk_method=RK_METHODS[rk], cn_target=0.5, step_duration=30.0, initial_dt=0.5,
                          rain_mode="physical")
    setup(g, z, h, u, v, n=MANNING)
    g.set_forcing(forcing)
    N = RK_STAGES[rk]
    t1, dt1, t2, dt2 = 2.0, 0.04, 2.04, 0.03
    r1 = g.do_timestep(t1, dt1)
    s1 = [g.get_field(100 + 3 * N + k) for k in range(3)]
    g.accept()
    r2 = g.do_timestep(t2, dt2)
    s2 = [g.get_field(100 + 3 * N + k) for k in range(3)]
    g.close()

    dev = torch.device("cuda:0")
    tz, th, tu, tv = (torch.tensor(a, dtype=torch.float64, device=dev).contiguous() for a in (z, h, u, v))
    out1 = [torch.empty_like(th) for _ in range(3)]
    out2 = [torch.empty_like(th) for _ in range(3)]
    res = torch.zeros(3, dtype=torch.float64, device=dev)
    mesh = MeshDesc(nx, ny, dx, dx, 0.0, 0.0)
    man = (C.c_double * 4)(*MANNING)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    p = lambda t: C.c_void_p(t.data_ptr())

    rc = f(C.byref(mesh), C.byref(_params(rk)), man, C.byref(forcing), p(tz), p(th), p(tu), p(tv),
           p(out1[0]), p(out1[1]), p(out1[2]), t1, dt1, p(res), stream)
    assert rc == 0, lib.sv_last_error(None).decode()
    torch.cuda.synchronize(dev)
    for k in range(3):
        assert same(out1[k].cpu().numpy().reshape(ny, nx), s1[k]), f"first call, field {k}"
    cn, nd, rep = res.cpu().tolist()
    assert (cn, nd, bool(rep)) == (r1[0], r1[2], r1[1])

    rc = f(C.byref(mesh), C.byref(_params(rk)), man, C.byref(forcing), p(tz), p(out1[0]), p(out1[1]), p(out1[2]),
           p(out2[0]), p(out2[1]), p(out2[2]), t2, dt2, p(res), stream)
    assert rc == 0, lib.sv_last_error(None).decode()
    torch.cuda.synchronize(dev)
    for k in range(3):
        assert same(out2[k].cpu().numpy().reshape(ny, nx), s2[k]), f"second call, field {k}"
    cn, nd, rep = res.cpu().tolist()
    assert (cn, nd, bool(rep)) == (r2[0], r2[2], r2[1])


@pytest.mark.gpu
@pytest.mark.parametrize("rk", [0, 1, 2, 3, 5, 7, 9])
def test_noalloc_timestep_matches_allocating_solver_twice(rk):
    _pair(70, 41, 2.5, rk, seed=77 + rk)


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny", [(256, 256), (1, 65536)])
def test_noalloc_at_the_working_array_limits(nx, ny):
    """The full 65536-cell mesh, and the 1-cell-wide strip that needs every one of the 8192
    partial-sum slots of the working array."""
    _pair(nx, ny, 2.0, 9, seed=5)
