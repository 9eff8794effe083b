"""isf_poisson_solve_static: the Poisson solve for callers that cannot let
the library allocate device memory (a host runtime whose own pool owns all
device memory, a hard memory cap, or a loop that must not allocate after its
set-up).  It takes the grid parameters instead of a handle and works in a
2 MiB file-scope device workspace shared by all calls.  Checked through the
C ABI against the handle-based isf_poisson_solve on the same input, on two
calls in a row (the second reuses what the first left in the workspace),
with the relative tolerance of the other Poisson tests (1e-5).

This file is collected last so that a run stopping at its first failure has
already run every other test."""
import ctypes as C
import importlib

import numpy as np
import pytest
import torch

from helpers import rel

pytestmark = pytest.mark.gpu

HBAR = float(np.float32(0.1))
DT = float(np.float32(1 / 48))


def _params(_lib, L, dims):
    p = _lib.IsfParams()
    p.grid_res[:] = list(dims)
    p.physical_size[:] = list(L)
    p.hbar = HBAR
    p.dt = DT
    p.device = 0
    p.flags = 0
    p.stream = None  # legacy default stream, the one torch uses here
    return p


def test_static_poisson_matches_handle_entry_point(isfpkg):
    _lib = importlib.import_module(isfpkg.__name__ + "._lib")
    lib = _lib.load()
    for L, dims in (((4, 2, 2), (64, 32, 32)), ((3, 2, 2), (48, 32, 32))):
        isf = isfpkg.ISF(L, dims, HBAR, DT)
        rng = np.random.default_rng(21)
        f = rng.normal(size=dims[::-1])
        f -= f.mean()
        ft = torch.tensor(f, dtype=torch.float32, device="cuda")
        ref = isf.poisson_solve(ft)
        isf.sync()
        ref = ref.double().cpu().numpy()
        p = _params(_lib, L, dims)
        for call in range(2):
            q = torch.full(dims[::-1], float("nan"), dtype=torch.float32, device="cuda")
            rc = lib.isf_poisson_solve_static(C.byref(p), C.c_void_p(ft.data_ptr()), C.c_void_p(q.data_ptr()))
            assert rc == 0, lib.isf_static_last_error()
            torch.cuda.synchronize()
            assert rel(q.double().cpu().numpy(), ref) < 1e-5, (dims, call)
        isf.close()


def test_static_poisson_rejects_grids_beyond_the_workspace(isfpkg):
    _lib = importlib.import_module(isfpkg.__name__ + "._lib")
    lib = _lib.load()
    p = _params(_lib, (10, 5, 5), (256, 128, 128))
    dummy = torch.zeros(1, device="cuda")
    rc = lib.isf_poisson_solve_static(C.byref(p), C.c_void_p(dummy.data_ptr()), C.c_void_p(dummy.data_ptr()))
    assert rc == _lib.ISF_ERR_INVALID
    assert b"static workspace" in lib.isf_static_last_error()


def test_static_poisson_refuses_a_table_upload_under_capture(isfpkg):
    """A call whose grid parameters differ from the previous call's must
    upload tables from a host buffer that lives only during the call; under
    stream capture that copy would replay from freed memory, so the call is
    refused before it queues anything."""
    import warnings

    _lib = importlib.import_module(isfpkg.__name__ + "._lib")
    lib = _lib.load()
    L, dims = (4, 2, 2), (64, 32, 32)
    f = torch.zeros(dims[::-1], dtype=torch.float32, device="cuda")
    q = torch.empty_like(f)
    p = _params(_lib, L, dims)
    # an ordinary call first: looks up the workspace address and uploads the tables
    assert lib.isf_poisson_solve_static(C.byref(p), C.c_void_p(f.data_ptr()), C.c_void_p(q.data_ptr())) == 0
    torch.cuda.synchronize()
    other = _params(_lib, (2, 2, 2), (32, 32, 32))
    s = torch.cuda.Stream()
    other.stream = C.c_void_p(s.cuda_stream)
    graph = torch.cuda.CUDAGraph()
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        with torch.cuda.graph(graph, stream=s):
            rc = lib.isf_poisson_solve_static(C.byref(other), C.c_void_p(f.data_ptr()), C.c_void_p(q.data_ptr()))
    del graph
    assert rc == _lib.ISF_ERR_INVALID
    assert b"captured" in lib.isf_static_last_error()
    torch.cuda.synchronize()
