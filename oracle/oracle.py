"""ORACLE -- test infrastructure only (tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py).  The product library never imports this.

ctypes front-end of oracle/isf_oracle.cpp, the CPU restatement of the ISF
time step of SchroedingersSmoke.jl (src/parallel.jl, src/particles.jl,
examples/benchmark.jl:46-65).  `Oracle(prec=64)` is the FP64 oracle the GPU
parity tests compare against; `Oracle(prec=32)` is the FP32 restatement timed
as the CPU baseline.

Parity status: UNPINNED against the reference's own outputs (Julia is absent
and the reference holds no golden vectors).  The oracle is pinned by
numpy.fft, by the independent MatlabPort restatement (oracle/matlabport.py)
and by analytic known answers; see tests/test_oracle_cpu.py.

Array conventions (0-based, x fastest, as the Julia arrays):
  psi        (nz, ny, nx, 4)  re1, im1, re2, im2
  velocity   (nz, ny, nx, 3)
  particles  (P, 3), dead slot = (-1, -1, -1)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
SOURCES = [os.path.join(HERE, "isf_oracle.cpp"), os.path.join(HERE, "philox.h")]

# emission modes (particles.jl:86-90 ring / nozzle disc / nozzle cylinder)
EMIT_RING, EMIT_DISC, EMIT_CYLINDER, EMIT_RING_PLANE = 0, 1, 2, 3
# jet phase modes: reference tuple_dot = sum(k .+ x) (particles.jl:1,15) / k.x
PHASE_REFERENCE_SUM, PHASE_DOT = 0, 1


def build(force: bool = False) -> str:
    """Compile liboracle.so with g++ (OpenMP).  Returns the library path."""
    if not force and os.path.exists(LIB_PATH):
        lib_m = os.path.getmtime(LIB_PATH)
        if all(os.path.getmtime(s) <= lib_m for s in SOURCES):
            return LIB_PATH
    cmd = ["g++", "-O3", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
           "-o", LIB_PATH + ".tmp", SOURCES[0]]
    subprocess.check_call(cmd, cwd=HERE)
    os.replace(LIB_PATH + ".tmp", LIB_PATH)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, i32, f32, f64, i64, u64 = C.c_void_p, C.c_int, C.c_float, C.c_double, C.c_long, C.c_uint64
        fp = C.POINTER(C.c_float)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i32, ip, ip, f32, f32]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_normalized_weights.argtypes = [vp, i32]
        L.orc_num_threads.restype = i32
        L.orc_set_num_threads.argtypes = [i32]
        for name in ["orc_fft3"]:
            getattr(L, name).argtypes = [vp, vp, i32]
        for name in ["orc_get_mask", "orc_get_fac", "orc_get_velocity", "orc_set_velocity", "orc_get_f",
                     "orc_set_f", "orc_get_q", "orc_schroedinger_flow", "orc_normalize", "orc_gauge",
                     "orc_pressure_project"]:
            getattr(L, name).argtypes = [vp, vp]
        for name in ["orc_div", "orc_poisson_solve", "orc_staggered_sharp"]:
            getattr(L, name).argtypes = [vp]
        L.orc_clamp_events.restype = i64
        L.orc_clamp_events.argtypes = [vp]
        L.orc_velocity_one_form.argtypes = [vp, vp, f64]
        L.orc_restrict_velocity.argtypes = [vp, vp, dp, vp, fp, f32, f32, f64, i32]
        L.orc_isjet.argtypes = [vp, vp, fp, f32, f32]
        L.orc_add_particles.argtypes = [vp, vp, i64, i64, i64, fp, f32, f32, u64, u64, i32]
        L.orc_staggered_advect.argtypes = [vp, vp, i64, vp]
        L.orc_philox.argtypes = [vp, vp, vp]
        L.orc_step.argtypes = [vp, vp, vp, i64, i32, dp, f64, fp, f32, f32, i64, i64, u64, u64, i32, i32, vp]
        _lib = L
    return _lib


def _f3(v):
    return (C.c_float * 3)(*[float(np.float32(x)) for x in v])


def _d3(v):
    return (C.c_double * 3)(*[float(x) for x in v])


def _ptr(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


class Oracle:
    """One ISF instance (parallel.jl:41) in FP64 (prec=64) or FP32 (prec=32).

    Parameters are passed as Float32 values, as the reference's callers pass
    `hbar = 0.1f0`, `dt = 1f0/48f0` (examples/benchmark.jl:6-7); the FP64
    oracle promotes those exact values.
    """

    def __init__(self, physical_size, dims, hbar, dt, prec: int = 64, normalized_weights: bool = False):
        self.L = lib()
        self.prec = prec
        self.dtype = np.float64 if prec == 64 else np.float32
        self.cdtype = np.complex128 if prec == 64 else np.complex64
        self.dims = tuple(int(x) for x in dims)
        self.physical_size = tuple(int(x) for x in physical_size)
        self.hbar = float(np.float32(hbar))
        self.dt = float(np.float32(dt))
        d = (C.c_int * 3)(*self.dims)
        s = (C.c_int * 3)(*self.physical_size)
        self.h = self.L.orc_create(prec, d, s, self.hbar, self.dt)
        if not self.h:
            raise ValueError(f"unsupported grid {self.dims} (sizes must be 2^a 3^b)")
        if normalized_weights:
            self.L.orc_set_normalized_weights(self.h, 1)
        self.nx, self.ny, self.nz = self.dims
        self.N = self.nx * self.ny * self.nz
        self.d = tuple(self.dtype(L) / self.dtype(n) for L, n in zip(self.physical_size, self.dims))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.orc_destroy(h)
            self.h = None

    # ---- helpers
    def _psi(self, psi):
        assert psi.dtype == self.dtype and psi.shape == (self.nz, self.ny, self.nx, 4), (psi.dtype, psi.shape)
        return _ptr(psi)

    def new_psi(self, psi1=1.0, psi2=0.01):
        p = np.zeros((self.nz, self.ny, self.nx, 4), self.dtype)
        a = np.broadcast_to(np.asarray(psi1, np.complex128), (self.nz, self.ny, self.nx))
        b = np.broadcast_to(np.asarray(psi2, np.complex128), (self.nz, self.ny, self.nx))
        p[..., 0], p[..., 1], p[..., 2], p[..., 3] = a.real, a.imag, b.real, b.imag
        return p

    # ---- tables
    def mask(self):
        out = np.zeros((self.nz, self.ny, self.nx), self.cdtype)
        self.L.orc_get_mask(self.h, _ptr(out))
        return out

    def fac(self):
        out = np.zeros((self.nz, self.ny, self.nx), self.cdtype)
        self.L.orc_get_fac(self.h, _ptr(out))
        return out

    def velocity(self):
        out = np.zeros((self.nz, self.ny, self.nx, 3), self.dtype)
        self.L.orc_get_velocity(self.h, _ptr(out))
        return out

    def set_velocity(self, v):
        v = np.ascontiguousarray(v, self.dtype)
        assert v.shape == (self.nz, self.ny, self.nx, 3)
        self.L.orc_set_velocity(self.h, _ptr(v))

    def f(self):
        out = np.zeros((self.nz, self.ny, self.nx), self.dtype)
        self.L.orc_get_f(self.h, _ptr(out))
        return out

    def set_f(self, f):
        f = np.ascontiguousarray(f, self.dtype)
        self.L.orc_set_f(self.h, _ptr(f))

    def q(self):
        out = np.zeros((self.nz, self.ny, self.nx), self.cdtype)
        self.L.orc_get_q(self.h, _ptr(out))
        return out

    def clamp_events(self):
        return int(self.L.orc_clamp_events(self.h))

    # ---- operators (reference names)
    def fft3(self, a, sign=-1):
        a = np.ascontiguousarray(a, self.cdtype).copy()
        self.L.orc_fft3(self.h, _ptr(a), int(sign))
        return a

    def schroedinger_flow(self, psi):
        self.L.orc_schroedinger_flow(self.h, self._psi(psi))
        return psi

    def normalize(self, psi):
        self.L.orc_normalize(self.h, self._psi(psi))
        return psi

    def velocity_one_form(self, psi, hbar=1.0):
        self.L.orc_velocity_one_form(self.h, self._psi(psi), float(np.float32(hbar)))
        return self.velocity()

    def div(self):
        self.L.orc_div(self.h)
        return self.f()

    def poisson_solve(self):
        self.L.orc_poisson_solve(self.h)
        return self.q()

    def gauge(self, psi):
        self.L.orc_gauge(self.h, self._psi(psi))
        return psi

    def pressure_project(self, psi):
        self.L.orc_pressure_project(self.h, self._psi(psi))
        return psi

    def staggered_sharp(self):
        self.L.orc_staggered_sharp(self.h)

    def isjet(self, cen, length, rad):
        out = np.zeros((self.nz, self.ny, self.nx), np.uint8)
        self.L.orc_isjet(self.h, _ptr(out), _f3(cen), float(length), float(rad))
        return out

    def restrict_velocity(self, psi, kvec, omgterm, cen, length, rad, phase_mode=PHASE_DOT, jetmask=None):
        mp = None if jetmask is None else _ptr(np.ascontiguousarray(jetmask, np.uint8))
        self.L.orc_restrict_velocity(self.h, self._psi(psi), _d3(kvec), mp, _f3(cen), float(length), float(rad),
                                     float(omgterm), int(phase_mode))
        return psi

    def add_particles(self, parts, start, count, cen, rad, seed, counter, mode=EMIT_RING, length=0.5):
        assert parts.dtype == self.dtype and parts.ndim == 2 and parts.shape[1] == 3
        self.L.orc_add_particles(self.h, _ptr(parts), parts.shape[0], int(start), int(count), _f3(cen),
                                 float(length), float(rad), int(seed), int(counter), int(mode))
        return parts

    def staggered_advect(self, parts, margin=False):
        assert parts.dtype == self.dtype and parts.ndim == 2 and parts.shape[1] == 3
        m = np.zeros(parts.shape[0], np.float64) if margin else None
        self.L.orc_staggered_advect(self.h, _ptr(parts), parts.shape[0], None if m is None else _ptr(m))
        return (parts, m) if margin else parts

    def step(self, psi, parts, jet=None, margin=None):
        """One simloop body (examples/benchmark.jl:46-65).

        jet: None for the no-nozzle step, else a dict with keys kvec,
        omega_t, cen, len, rad, emit_start, emit_count, seed, counter,
        emit_mode, phase_mode.
        """
        np_ = 0 if parts is None else parts.shape[0]
        pp = None if parts is None else _ptr(parts)
        mp = None if margin is None else _ptr(margin)
        if jet is None:
            self.L.orc_step(self.h, self._psi(psi), pp, np_, 0, _d3((0, 0, 0)), 0.0, _f3((0, 0, 0)), 0.0, 0.0,
                            0, 0, 0, 0, 0, 0, mp)
        else:
            self.L.orc_step(self.h, self._psi(psi), pp, np_, 1, _d3(jet["kvec"]), float(jet["omega_t"]),
                            _f3(jet["cen"]), float(jet["len"]), float(jet["rad"]), int(jet.get("emit_start", 0)),
                            int(jet.get("emit_count", 0)), int(jet.get("seed", 0)), int(jet.get("counter", 0)),
                            int(jet.get("emit_mode", EMIT_RING)), int(jet.get("phase_mode", PHASE_DOT)), mp)
        return psi


def philox(ctr, key):
    c = np.asarray(ctr, np.uint32)
    k = np.asarray(key, np.uint32)
    out = np.zeros(4, np.uint32)
    lib().orc_philox(_ptr(c), _ptr(k), _ptr(out))
    return [int(v) for v in out]


def num_threads() -> int:
    return int(lib().orc_num_threads())


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))
