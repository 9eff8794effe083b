"""ctypes binding of libisf.so (the C ABI declared in include/isf.h).

The library is the product: if it is missing, or no CUDA device is usable,
loading fails loudly -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libisf.so")

ISF_OK, ISF_ERR_INVALID, ISF_ERR_CUDA, ISF_ERR_NOMEM, ISF_ERR_NAN, ISF_ERR_TIMEOUT = 0, 1, 2, 3, 4, 5
PERSIST_ON, PERSIST_STALL = 1, 2
FLAG_NORMALIZED_WEIGHTS, FLAG_CHECK_NAN, FLAG_TMA_Z_PASS, FLAG_TMA_Z_STALL = 1, 2, 4, 8
PHASE_REFERENCE_SUM, PHASE_DOT = 0, 1
EMIT_RING, EMIT_DISC, EMIT_CYLINDER, EMIT_RING_PLANE = 0, 1, 2, 3

# every exported entry point of include/isf.h
EXPORTS = (
    "isf_create", "isf_destroy", "isf_last_error", "isf_get_stream", "isf_sync", "isf_join", "isf_malloc", "isf_free",
    "isf_memcpy_h2d", "isf_memcpy_d2h", "isf_grid_info", "isf_schroedinger_flow", "isf_normalize_psi",
    "isf_pressure_project", "isf_velocity_one_form", "isf_staggered_sharp", "isf_get_velocity",
    "isf_set_velocity", "isf_isjet", "isf_restrict_velocity", "isf_init_jet", "isf_add_particles", "isf_staggered_advect",
    "isf_step", "isf_div", "isf_poisson_solve", "isf_fft3", "isf_counters", "isf_counters_async", "isf_profile_start",
    "isf_profile_stop", "isf_profile_sites", "isf_profile_get", "isf_launch_count", "isf_poisson_solve_static",
    "isf_static_last_error", "isf_batch_create", "isf_batch_destroy", "isf_batch_last_error",
    "isf_batch_set_psi", "isf_batch_get_psi", "isf_batch_set_particles", "isf_batch_get_particles",
    "isf_batch_state", "isf_batch_init_jet", "isf_batch_step", "isf_batch_set_step", "isf_batch_get_stream",
    "isf_batch_sync", "isf_batch_info", "isf_batch_tiles", "isf_batch_counters",
    "isf_adj_schroedinger_flow", "isf_adj_normalize_psi", "isf_adj_pressure_project", "isf_adj_restrict_velocity",
    "isf_adj_velocity_one_form", "isf_adj_staggered_advect", "isf_adj_get_velocity_bar", "isf_adj_set_velocity_bar",
    "isf_adj_step", "isf_adj_loss", "isf_adj_gradient",
    "isf_psi_from_f64", "isf_psi_to_f64", "isf_velocity_from_f64", "isf_velocity_to_f64", "isf_real_from_f64",
    "isf_real_to_f64", "isf_complex_to_f64", "isf_gauge_transform", "isf_add_particles_soa",
    "isf_staggered_velocity", "isf_advect_active", "isf_keep_inside", "isf_gather_particles",
    "isf_set_particle_order", "isf_sort_particles", "isf_get_particle_order", "isf_batch_set_persistent",
)
TILE_KINDS = ("x_psi", "x_real", "y_psi", "z_psi", "y_half", "z_half")


class ISFError(RuntimeError):
    """A libisf call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"libisf error {code}: {msg}")
        self.code = code


class IsfParams(C.Structure):
    _fields_ = [
        ("grid_res", C.c_int32 * 3),
        ("physical_size", C.c_int32 * 3),
        ("hbar", C.c_float),
        ("dt", C.c_float),
        ("device", C.c_int32),
        ("flags", C.c_int32),
        ("stream", C.c_void_p),
    ]


class IsfStepArgs(C.Structure):
    _fields_ = [
        ("jet", C.c_int32),
        ("phase_mode", C.c_int32),
        ("kvec", C.c_float * 3),
        ("omega_t", C.c_float),
        ("nozzle_cen", C.c_float * 3),
        ("nozzle_len", C.c_float),
        ("nozzle_rad", C.c_float),
        ("emit_mode", C.c_int32),
        ("jetmask", C.c_void_p),
        ("emit_start", C.c_int64),
        ("emit_count", C.c_int64),
        ("seed", C.c_uint64),
        ("counter", C.c_uint64),
    ]


class IsfSimDesc(C.Structure):
    _fields_ = [
        ("grid_res", C.c_int32 * 3),
        ("physical_size", C.c_int32 * 3),
        ("hbar", C.c_float),
        ("dt", C.c_float),
        ("nslots", C.c_int64),
        ("jet", C.c_int32),
        ("phase_mode", C.c_int32),
        ("kvec", C.c_float * 3),
        ("omega", C.c_float),
        ("nozzle_cen", C.c_float * 3),
        ("nozzle_len", C.c_float),
        ("nozzle_rad", C.c_float),
        ("emit_mode", C.c_int32),
        ("emit_per_step", C.c_int64),
        ("seed", C.c_uint64),
    ]


class IsfAdjProblem(C.Structure):
    _fields_ = [
        ("nsteps", C.c_int32),
        ("checkpoint_every", C.c_int32),
        ("init_iters", C.c_int32),
        ("phase_mode", C.c_int32),
        ("kvec", C.c_float * 3),
        ("omega", C.c_float),
        ("nozzle_cen", C.c_float * 3),
        ("nozzle_len", C.c_float),
        ("nozzle_rad", C.c_float),
    ]


_lib = None


def load(path: str | None = None):
    """Load libisf.so (or the library named by $ISF_LIBRARY, e.g. the
    bounds-checking libisf_check.so) and declare its signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or os.environ.get("ISF_LIBRARY") or LIB_PATH
    if not os.path.exists(p):
        raise ImportError(f"libisf.so not built ({p}); run schroedingerssmoke.jl_b200/build.py")
    L = C.CDLL(p)
    vp, i32, i64, u64, f32, sz = C.c_void_p, C.c_int32, C.c_int64, C.c_uint64, C.c_float, C.c_size_t
    fp = C.POINTER(C.c_float)
    dp = C.POINTER(C.c_double)
    sig = {
        "isf_create": [C.POINTER(IsfParams), C.POINTER(vp)],
        "isf_destroy": [vp],
        "isf_get_stream": [vp, C.POINTER(vp)],
        "isf_join": [vp],
        "isf_sync": [vp],
        "isf_malloc": [vp, C.POINTER(vp), sz],
        "isf_free": [vp, vp],
        "isf_memcpy_h2d": [vp, vp, vp, sz],
        "isf_memcpy_d2h": [vp, vp, vp, sz],
        "isf_grid_info": [vp, C.POINTER(C.c_int32), fp],
        "isf_schroedinger_flow": [vp, vp],
        "isf_normalize_psi": [vp, vp],
        "isf_pressure_project": [vp, vp],
        "isf_velocity_one_form": [vp, vp, f32],
        "isf_staggered_sharp": [vp],
        "isf_get_velocity": [vp, vp],
        "isf_set_velocity": [vp, vp],
        "isf_isjet": [vp, vp, fp, f32, f32],
        "isf_restrict_velocity": [vp, vp, fp, vp, fp, f32, f32, f32, i32],
        "isf_init_jet": [vp, vp, i32, fp, vp, fp, f32, f32, i32],
        "isf_add_particles": [vp, vp, i64, i64, i64, fp, f32, f32, u64, u64, i32],
        "isf_staggered_advect": [vp, vp, i64],
        "isf_step": [vp, vp, vp, i64, C.POINTER(IsfStepArgs)],
        "isf_set_particle_order": [vp, i32],
        "isf_batch_set_persistent": [vp, i32, i64],
        "isf_sort_particles": [vp, vp, i64],
        "isf_get_particle_order": [vp, vp, i64, C.POINTER(i64)],
        "isf_div": [vp, vp],
        "isf_poisson_solve": [vp, vp, vp],
        "isf_fft3": [vp, vp, i32],
        "isf_counters": [vp, C.POINTER(C.c_uint64), i32, i32],
        "isf_counters_async": [vp, vp, i32, i32],
        "isf_profile_start": [vp],
        "isf_profile_stop": [vp],
        "isf_profile_sites": [vp, C.POINTER(C.c_int32)],
        "isf_profile_get": [vp, i32, C.c_char_p, sz, C.POINTER(C.c_double), C.POINTER(C.c_int64)],
        "isf_launch_count": [vp, C.POINTER(C.c_uint64)],
        "isf_poisson_solve_static": [C.POINTER(IsfParams), vp, vp],
        "isf_batch_create": [C.POINTER(IsfSimDesc), i32, i32, i32, C.POINTER(vp)],
        "isf_batch_destroy": [vp],
        "isf_batch_set_psi": [vp, i32, vp],
        "isf_batch_get_psi": [vp, i32, vp],
        "isf_batch_set_particles": [vp, i32, vp],
        "isf_batch_get_particles": [vp, i32, vp],
        "isf_batch_state": [vp, i32, C.POINTER(vp), C.POINTER(vp)],
        "isf_batch_init_jet": [vp, i32],
        "isf_batch_step": [vp, i32],
        "isf_batch_set_step": [vp, i64],
        "isf_batch_get_stream": [vp, C.POINTER(vp)],
        "isf_batch_sync": [vp],
        "isf_batch_info": [vp, C.POINTER(C.c_int32), C.POINTER(C.c_int32)],
        "isf_batch_tiles": [vp, i32, C.POINTER(C.c_int32)],
        "isf_batch_counters": [vp, i32, C.POINTER(C.c_uint64), i32],
        "isf_adj_schroedinger_flow": [vp, vp],
        "isf_adj_normalize_psi": [vp, vp, vp],
        "isf_adj_pressure_project": [vp, vp, vp],
        "isf_adj_restrict_velocity": [vp, vp, vp, fp, vp, fp, f32, f32, f32, i32, dp],
        "isf_adj_velocity_one_form": [vp, vp, f32, i32, vp],
        "isf_adj_staggered_advect": [vp, vp, vp, i64],
        "isf_adj_get_velocity_bar": [vp, vp],
        "isf_adj_set_velocity_bar": [vp, vp],
        "isf_adj_step": [vp, vp, vp, i64, C.POINTER(IsfStepArgs), vp, vp, dp],
        "isf_adj_loss": [vp, C.POINTER(IsfAdjProblem), vp, vp, i64, vp, dp],
        "isf_adj_gradient": [vp, C.POINTER(IsfAdjProblem), vp, vp, i64, vp, dp, vp, vp, dp],
        "isf_psi_from_f64": [vp, vp, vp, vp],
        "isf_psi_to_f64": [vp, vp, vp, vp],
        "isf_velocity_from_f64": [vp, vp, vp, vp],
        "isf_velocity_to_f64": [vp, vp, vp, vp],
        "isf_real_from_f64": [vp, vp, i64, C.c_double, vp, i64],
        "isf_real_to_f64": [vp, vp, vp, i64],
        "isf_complex_to_f64": [vp, vp, vp, vp, i64],
        "isf_gauge_transform": [vp, vp, vp, vp],
        "isf_add_particles_soa": [vp, vp, vp, vp, i64, i64, i64, fp, f32, f32, u64, u64, i32],
        "isf_staggered_velocity": [vp, vp, vp, vp, i64, vp, vp, vp],
        "isf_advect_active": [vp, vp, vp, vp, i64, vp, i64, f32],
        "isf_keep_inside": [vp, vp, vp, vp, i64, vp, i64, vp, vp],
        "isf_gather_particles": [vp, vp, vp, vp, i64, vp, i64, vp, vp, vp],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = C.c_int
    L.isf_last_error.argtypes = [vp]
    L.isf_last_error.restype = C.c_char_p
    L.isf_static_last_error.argtypes = []
    L.isf_static_last_error.restype = C.c_char_p
    L.isf_batch_last_error.argtypes = [vp]
    L.isf_batch_last_error.restype = C.c_char_p
    if path is None:
        _lib = L
    return L


def check(rc: int, handle=None):
    if rc != ISF_OK:
        msg = load().isf_last_error(handle)
        raise ISFError(rc, msg.decode() if msg else "")
    return rc


def check_batch(rc: int, batch=None):
    if rc != ISF_OK:
        msg = load().isf_batch_last_error(batch)
        raise ISFError(rc, msg.decode() if msg else "")
    return rc


def f3(v):
    return (C.c_float * 3)(*[float(x) for x in v])
