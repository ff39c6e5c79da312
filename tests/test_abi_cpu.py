"""The C-ABI library: it loads without a GPU, exports every entry point include/sv.h declares,
and fails cleanly (status code and message, no crash) when no device is present."""
import ctypes as C
import os
import re

import pytest

import mfcm_b200
from mfcm_b200 import MeshDesc, Params
from mfcm_b200._abi import SV_F64, SV_E_ARG

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_entry_points():
    text = open(os.path.join(ROOT, "include", "sv.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|const char\*)\s+(sv_\w+)\s*\(", text, flags=re.M)))


def test_library_exports_every_declared_entry_point():
    lib = mfcm_b200.load_library()
    names = declared_entry_points()
    assert len(names) >= 20
    for n in names:
        assert hasattr(lib, n), f"{n} declared in include/sv.h but not exported"


def test_create_rejects_bad_arguments_before_touching_the_device():
    lib = mfcm_b200.load_library()
    h = C.c_void_p()
    bad_mesh = MeshDesc(0, 10, 1.0, 1.0, 0.0, 0.0)
    p = Params(SV_F64, 9, 1.0, 60.0, 1.0, 0.0, 0, 1, 0, 0)
    assert lib.sv_create(C.byref(bad_mesh), C.byref(p), 0, C.byref(h)) == SV_E_ARG
    assert lib.sv_last_error(None).decode() == "empty mesh"
    bad_rk = Params(SV_F64, 42, 1.0, 60.0, 1.0, 0.0, 0, 1, 0, 0)
    assert lib.sv_create(C.byref(MeshDesc(4, 4, 1.0, 1.0, 0, 0)), C.byref(bad_rk), 0, C.byref(h)) == SV_E_ARG
    assert "Runge Kutta" in lib.sv_last_error(None).decode()


def test_null_context_is_an_argument_error():
    lib = mfcm_b200.load_library()
    assert lib.sv_accept(None) == SV_E_ARG
    assert lib.sv_set_dt(None, 1.0) == SV_E_ARG


def test_create_without_a_device_fails_cleanly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    with pytest.raises(mfcm_b200.SvError) as e:
        mfcm_b200.SaintVenantSolver(8, 8, 1.0)
    assert e.value.code == -2  # SV_E_CUDA
