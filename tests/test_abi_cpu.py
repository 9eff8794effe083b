"""The C ABI library builds for sm_100a, loads, and exports every entry point
that include/isf.h declares (no compute calls: this runs without a GPU)."""
import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "isf.h")).read()
    return sorted(set(re.findall(r"^ISF_API\s+[\w\s\*]+?\b(isf_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_the_operator_set():
    names = declared_symbols()
    for must in ("isf_create", "isf_destroy", "isf_schroedinger_flow", "isf_normalize_psi", "isf_pressure_project",
                 "isf_velocity_one_form", "isf_staggered_sharp", "isf_restrict_velocity", "isf_add_particles",
                 "isf_staggered_advect", "isf_step", "isf_isjet", "isf_sync", "isf_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(libisf_path):
    lib = C.CDLL(libisf_path)
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_python_binding_covers_the_header(isfpkg):
    import importlib
    _lib = importlib.import_module(isfpkg.__name__ + "._lib")
    assert sorted(_lib.EXPORTS) == declared_symbols()


def test_create_without_gpu_fails_cleanly(isfpkg):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import importlib
    _lib = importlib.import_module(isfpkg.__name__ + "._lib")
    L = _lib.load()
    p = _lib.IsfParams()
    p.grid_res[:] = [16, 8, 8]
    p.physical_size[:] = [1, 1, 1]
    p.hbar, p.dt = 0.1, 0.02
    h = C.c_void_p()
    rc = L.isf_create(C.byref(p), C.byref(h))
    assert rc != 0 and not h.value
    assert L.isf_last_error(None)
    with pytest.raises(isfpkg.ISFError):
        isfpkg.ISF((1, 1, 1), (16, 8, 8), 0.1, 0.02)


def test_invalid_sizes_rejected_before_touching_cuda(isfpkg):
    import importlib
    _lib = importlib.import_module(isfpkg.__name__ + "._lib")
    L = _lib.load()
    for dims in ((22, 8, 8), (14, 8, 8), (16, 8, 6), (16, 9, 8), (1024, 8, 8)):
        p = _lib.IsfParams()
        p.grid_res[:] = list(dims)
        p.physical_size[:] = [1, 1, 1]
        p.hbar, p.dt = 0.1, 0.02
        h = C.c_void_p()
        assert L.isf_create(C.byref(p), C.byref(h)) == _lib.ISF_ERR_INVALID
        assert b"grid_res" in L.isf_last_error(None)
