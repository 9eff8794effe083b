"""B200 (sm_100a) incompressible Schroedinger flow -- host-side mirror of the
SchroedingersSmoke.jl API over the C ABI of libisf (include/isf.h).

Names follow the reference's exports (src/parallel.jl:264-266,
src/particles.jl:97); Julia's in-place `!` suffix is dropped.  Device arrays
are torch CUDA tensors with the reference's layouts:

    psi        float32 (nz, ny, nx, 4): re psi1, im psi1, re psi2, im psi2
    particles  float32 (P, 3); a dead slot is (-1, -1, -1)
    isjet mask uint8   (nz, ny, nx)

torch only supplies device memory and the stream for event timing; all
arithmetic runs in libisf's kernels.  Misuse raises ISFError (the reference
throws a Julia exception).
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _lib
from ._lib import (EMIT_CYLINDER, EMIT_DISC, EMIT_RING, EMIT_RING_PLANE, FLAG_CHECK_NAN, FLAG_NORMALIZED_WEIGHTS, FLAG_TMA_Z_PASS,
                   FLAG_TMA_Z_STALL, PHASE_DOT,
                   PHASE_REFERENCE_SUM, IsfParams, IsfStepArgs, ISFError, check, f3)

__all__ = [
    "ISF", "ISFBatch", "ISFError", "ParticleLoss", "schroedinger_flow", "normalize_psi", "pressure_project", "velocity_one_form",
    "staggered_sharp", "isjet", "restrict_velocity", "init_jet", "add_particles", "staggered_advect", "step", "new_psi",
    "PHASE_DOT", "PHASE_REFERENCE_SUM", "EMIT_RING", "EMIT_DISC", "EMIT_CYLINDER", "EMIT_RING_PLANE", "FLAG_NORMALIZED_WEIGHTS",
    "FLAG_CHECK_NAN", "STREAM_LEGACY",
]


# the CUDA runtime's handle of the legacy default stream (cudaStreamLegacy),
# the stream torch's default-stream work runs on
STREAM_LEGACY = 1


def _ptr(t: torch.Tensor | None):
    if t is None:
        return None
    if not t.is_cuda or not t.is_contiguous():
        raise ISFError(_lib.ISF_ERR_INVALID, "arrays must be contiguous CUDA tensors")
    return C.c_void_p(t.data_ptr())


class ISF:
    """ISF{B200Array, UInt32, Float32}(physical_size, dims, hbar, dt)
    (src/parallel.jl:41-98): grid, d, velocity and the spectral tables live on
    the device of `device`."""

    def __init__(self, physical_size, dims, hbar, dt, device: int = 0, flags: int = 0, stream=None):
        # stream: a torch.cuda.Stream for all the handle's work (then without
        # the separate particle stream), STREAM_LEGACY for the legacy default
        # stream, or None for a stream of its own
        if not torch.cuda.is_available():
            raise ISFError(_lib.ISF_ERR_CUDA, "no CUDA device: libisf has no CPU path")
        self.L = _lib.load()
        p = IsfParams()
        p.grid_res[:] = [int(x) for x in dims]
        p.physical_size[:] = [int(x) for x in physical_size]
        p.hbar = float(hbar)
        p.dt = float(dt)
        p.device = int(device)
        p.flags = int(flags)
        p.stream = None if stream is None else (stream if isinstance(stream, int) else stream.cuda_stream)
        h = C.c_void_p()
        check(self.L.isf_create(C.byref(p), C.byref(h)))
        self.h = h
        self.device = torch.device("cuda", int(device))
        self.grid_res = tuple(int(x) for x in dims)
        self.physical_size = tuple(int(x) for x in physical_size)
        d = (C.c_float * 3)()
        n = (C.c_int32 * 3)()
        check(self.L.isf_grid_info(h, n, d), h)
        self.d = tuple(float(x) for x in d)
        self.hbar = float(torch.tensor(hbar, dtype=torch.float32))
        self.dt = float(torch.tensor(dt, dtype=torch.float32))
        s = C.c_void_p()
        check(self.L.isf_get_stream(h, C.byref(s)), h)
        self.stream = (torch.cuda.default_stream(self.device) if s.value == STREAM_LEGACY
                       else torch.cuda.ExternalStream(s.value, device=self.device))
        nx, ny, nz = self.grid_res
        self.shape = (nz, ny, nx)
        self.ncells = nx * ny * nz

    def close(self):
        if getattr(self, "h", None):
            self.L.isf_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        """GPUArrays.synchronize (examples/benchmark.jl:66)."""
        check(self.L.isf_sync(self.h), self.h)

    def join(self):
        """Order `self.stream` after the particle work (emission, advection)
        that `step` leaves on the handle's particle stream; no host wait.
        Every other call on the handle does this first."""
        check(self.L.isf_join(self.h), self.h)

    @property
    def velocity(self) -> torch.Tensor:
        """isf.velocity as (nz, ny, nx, 3) float32 (src/parallel.jl:14)."""
        out = torch.empty(self.shape + (3,), dtype=torch.float32, device=self.device)
        check(self.L.isf_get_velocity(self.h, _ptr(out)), self.h)
        self.sync()
        return out

    @velocity.setter
    def velocity(self, v: torch.Tensor):
        v = v.to(self.device, torch.float32).contiguous()
        check(self.L.isf_set_velocity(self.h, _ptr(v)), self.h)
        self.sync()

    @property
    def positions(self) -> torch.Tensor:
        """isf.positions = (i .- 1) .* d as (nz, ny, nx, 3) (src/parallel.jl:75-77)."""
        nx, ny, nz = self.grid_res
        ax = [torch.arange(n, device=self.device, dtype=torch.float32) * torch.tensor(dd, dtype=torch.float32)
              for n, dd in zip((nx, ny, nz), self.d)]
        z, y, x = torch.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
        return torch.stack([x, y, z], dim=-1).contiguous()

    # ---- diagnostics
    def div(self) -> torch.Tensor:
        f = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        check(self.L.isf_div(self.h, _ptr(f)), self.h)
        return f

    def poisson_solve(self, f: torch.Tensor) -> torch.Tensor:
        f = f.contiguous()
        q = torch.empty(self.shape, dtype=torch.float32, device=self.device)
        check(self.L.isf_poisson_solve(self.h, _ptr(f), _ptr(q)), self.h)
        return q

    def fft3(self, a: torch.Tensor, sign: int = -1) -> torch.Tensor:
        """In-place 3D complex FFT of a complex64 (nz, ny, nx) tensor."""
        if a.dtype != torch.complex64:
            raise ISFError(_lib.ISF_ERR_INVALID, "fft3 wants complex64")
        check(self.L.isf_fft3(self.h, _ptr(a), int(sign)), self.h)
        return a

    def counters(self, reset: bool = False):
        """Advection counters since the last reset (see isf_counters)."""
        out = (C.c_uint64 * 16)()
        check(self.L.isf_counters(self.h, out, 16, int(reset)), self.h)
        return {"clamp_events": int(out[0]), "live": int(out[1]), "check_failures": int(out[2]),
                "first_bad_index": int(out[3]), "first_bad_context": [int(v) for v in out[4:12]],
                "wait_timeouts": int(out[14]), "nonfinite": int(out[15])}

    def counters_async(self, out: torch.Tensor, reset: bool = False):
        """Queue a copy of the advection counters [clamp events, live] into
        `out` (a pinned int64 CPU tensor of 2+ entries) on the handle's stream;
        valid after sync()."""
        if out.device.type != "cpu" or out.dtype != torch.int64 or out.numel() < 2:
            raise ISFError(_lib.ISF_ERR_INVALID, "counters_async needs an int64 CPU tensor of 2+ entries")
        check(self.L.isf_counters_async(self.h, C.c_void_p(out.data_ptr()), 2, int(reset)), self.h)

    def launch_count(self) -> int:
        out = C.c_uint64()
        check(self.L.isf_launch_count(self.h, C.byref(out)), self.h)
        return int(out.value)

    def set_particle_order(self, every: int):
        """isf_step advects through a cell-sorted permutation of the slots,
        rebuilt every `every` steps (0: storage order).  Positions are bitwise
        the same either way."""
        check(self.L.isf_set_particle_order(self.h, int(every)), self.h)

    def sort_particles(self, particles: torch.Tensor):
        ptr, P = self._parts(particles)
        check(self.L.isf_sort_particles(self.h, ptr, P), self.h)

    def particle_order(self) -> torch.Tensor | None:
        """The current permutation of the slots (int32, on the device), or None."""
        n = C.c_int64()
        check(self.L.isf_get_particle_order(self.h, None, 0, C.byref(n)), self.h)
        if n.value == 0:
            return None
        out = torch.empty(n.value, dtype=torch.int32, device=self.device)
        check(self.L.isf_get_particle_order(self.h, _ptr(out), n.value, C.byref(n)), self.h)
        self.sync()
        return out

    def profile_start(self):
        check(self.L.isf_profile_start(self.h), self.h)

    def profile_stop(self) -> dict:
        """Stop per-launch-site event timing; {site: (total_ms, launches)}."""
        check(self.L.isf_profile_stop(self.h), self.h)
        n = C.c_int32()
        check(self.L.isf_profile_sites(self.h, C.byref(n)), self.h)
        out = {}
        buf = C.create_string_buffer(64)
        for i in range(n.value):
            ms = C.c_double()
            cnt = C.c_int64()
            check(self.L.isf_profile_get(self.h, i, buf, 64, C.byref(ms), C.byref(cnt)), self.h)
            if cnt.value:
                out[buf.value.decode()] = (ms.value, cnt.value)
        return out

    def _psi(self, psi):
        if psi.dtype != torch.float32 or tuple(psi.shape) != self.shape + (4,):
            raise ISFError(_lib.ISF_ERR_INVALID, f"psi must be float32 {self.shape + (4,)}")
        return _ptr(psi)

    def _parts(self, parts):
        if parts is None:
            return None, 0
        if parts.dtype != torch.float32 or parts.dim() != 2 or parts.shape[1] != 3:
            raise ISFError(_lib.ISF_ERR_INVALID, "particles must be float32 (P, 3)")
        return _ptr(parts), int(parts.shape[0])


def new_psi(isf: ISF, psi1=1.0, psi2=0.01) -> torch.Tensor:
    """psi = [(psi1, psi2) for every cell] (examples/benchmark.jl:20)."""
    p = torch.empty(isf.shape + (4,), dtype=torch.float32, device=isf.device)
    p[..., 0] = complex(psi1).real
    p[..., 1] = complex(psi1).imag
    p[..., 2] = complex(psi2).real
    p[..., 3] = complex(psi2).imag
    return p


def schroedinger_flow(isf: ISF, psi: torch.Tensor) -> torch.Tensor:
    """schroedinger_flow!(isf, psi) (src/parallel.jl:176-187)."""
    check(isf.L.isf_schroedinger_flow(isf.h, isf._psi(psi)), isf.h)
    return psi


def normalize_psi(isf: ISF, psi: torch.Tensor) -> torch.Tensor:
    """psi .= normalize_psi.(psi) (src/parallel.jl:162-165)."""
    check(isf.L.isf_normalize_psi(isf.h, isf._psi(psi)), isf.h)
    return psi


def pressure_project(isf: ISF, psi: torch.Tensor) -> torch.Tensor:
    """pressure_project!(isf, psi) (src/parallel.jl:155-160)."""
    check(isf.L.isf_pressure_project(isf.h, isf._psi(psi)), isf.h)
    return psi


def velocity_one_form(isf: ISF, psi: torch.Tensor, hbar: float = 1.0) -> None:
    """velocity_one_form!(isf, psi, hbar = 1f0) (src/parallel.jl:115-122)."""
    check(isf.L.isf_velocity_one_form(isf.h, isf._psi(psi), float(hbar)), isf.h)


def staggered_sharp(isf: ISF) -> None:
    """isf.velocity .*= 1 ./ isf.d (examples/benchmark.jl:61-63)."""
    check(isf.L.isf_staggered_sharp(isf.h), isf.h)


def isjet(isf: ISF, nozzle_cen, nozzle_len, nozzle_rad) -> torch.Tensor:
    """isjet.(isf.positions, (cen,), (len,), (rad,)) (src/particles.jl:6-10)."""
    out = torch.empty(isf.shape, dtype=torch.uint8, device=isf.device)
    check(isf.L.isf_isjet(isf.h, _ptr(out), f3(nozzle_cen), float(nozzle_len), float(nozzle_rad)), isf.h)
    return out


def restrict_velocity(isf: ISF, psi: torch.Tensor, kvec, isjetarr=None, omgterm: float = 0.0, *,
                      nozzle=None, phase_mode: int = PHASE_REFERENCE_SUM) -> torch.Tensor:
    """restrict_velocity!(isf, psi, kvec, isjetarr, omgterm) (src/particles.jl:25-27).

    `isjetarr` is the uint8 isjet array, or None with `nozzle=(cen, len, rad)`
    to evaluate the nozzle per cell.  The default phase is the reference's
    tuple_dot (sum(kvec .+ pos)); PHASE_DOT gives k . x.
    """
    if isjetarr is None and nozzle is None:
        raise ISFError(_lib.ISF_ERR_INVALID, "restrict_velocity needs isjetarr or nozzle")
    cen, ln, rad = nozzle if nozzle is not None else ((0.0, 0.0, 0.0), 0.0, 0.0)
    check(isf.L.isf_restrict_velocity(isf.h, isf._psi(psi), f3(kvec), _ptr(isjetarr), f3(cen), float(ln),
                                      float(rad), float(omgterm), int(phase_mode)), isf.h)
    return psi


def init_jet(isf: ISF, psi: torch.Tensor, iters: int, kvec, isjetarr=None, *, nozzle=None,
             phase_mode: int = PHASE_REFERENCE_SUM) -> torch.Tensor:
    """The jet set-up loop of examples/benchmark.jl:28-31 in one library call:
    `iters` times restrict_velocity!(isf, psi, kvec, isjetarr, 0) followed by
    pressure_project!(isf, psi)."""
    if isjetarr is None and nozzle is None:
        raise ISFError(_lib.ISF_ERR_INVALID, "init_jet needs isjetarr or nozzle")
    cen, ln, rad = nozzle if nozzle is not None else ((0.0, 0.0, 0.0), 0.0, 0.0)
    check(isf.L.isf_init_jet(isf.h, isf._psi(psi), int(iters), f3(kvec), _ptr(isjetarr), f3(cen), float(ln),
                             float(rad), int(phase_mode)), isf.h)
    return psi


def add_particles(isf: ISF, particles: torch.Tensor, rng, nozzle_cen, nozzle_rad, *, seed: int = 0,
                  counter: int = 0, mode: int = EMIT_RING, nozzle_len: float = 0.5) -> None:
    """add_particles!(particles, range, nozzle_cen, nozzle_rad) (src/particles.jl:60-94).

    `rng` is a Python range of 0-based slots (wrapping modulo the slot count).
    """
    ptr, P = isf._parts(particles)
    start, count = int(rng.start), len(rng)
    check(isf.L.isf_add_particles(isf.h, ptr, P, start, count, f3(nozzle_cen), float(nozzle_len),
                                  float(nozzle_rad), int(seed), int(counter), int(mode)), isf.h)


def staggered_advect(particles: torch.Tensor, isf: ISF) -> torch.Tensor:
    """staggered_advect!(particles, isf) (src/parallel.jl:248-261)."""
    ptr, P = isf._parts(particles)
    check(isf.L.isf_staggered_advect(isf.h, ptr, P), isf.h)
    return particles


def step_args(jet: dict | None = None) -> IsfStepArgs:
    a = IsfStepArgs()
    if jet is None:
        a.jet = 0
        return a
    a.jet = 1
    a.phase_mode = int(jet.get("phase_mode", PHASE_DOT))
    a.kvec[:] = [float(x) for x in jet["kvec"]]
    a.omega_t = float(jet["omega_t"])
    a.nozzle_cen[:] = [float(x) for x in jet["cen"]]
    a.nozzle_len = float(jet["len"])
    a.nozzle_rad = float(jet["rad"])
    a.emit_mode = int(jet.get("emit_mode", EMIT_RING))
    m = jet.get("jetmask")
    a.jetmask = None if m is None else m.data_ptr()
    a.emit_start = int(jet.get("emit_start", 0))
    a.emit_count = int(jet.get("emit_count", 0))
    a.seed = int(jet.get("seed", 0))
    a.counter = int(jet.get("counter", 0))
    return a


def step(isf: ISF, psi: torch.Tensor, particles: torch.Tensor | None = None, jet: dict | None = None) -> None:
    """One simloop body (examples/benchmark.jl:46-65) as one fused sequence:
    schroedinger_flow! -> normalize -> pressure_project! -> [add_particles!,
    restrict_velocity!, pressure_project!] -> velocity_one_form!(hbar) ->
    staggered sharp -> staggered_advect!."""
    ptr, P = isf._parts(particles)
    a = step_args(jet)
    check(isf.L.isf_step(isf.h, isf._psi(psi), ptr, P, C.byref(a)), isf.h)


class ISFBatch:
    """Many independent simulations stepped together (isf_batch_*): each entry
    of `sims` is a dict with

        dims, physical_size, hbar, dt        the ISF constructor arguments
        nslots                               particle slots (default 0)
        jet                                  None, or a dict with kvec, omega,
                                             cen, len, rad, phase_mode,
                                             emit_mode, emit_per_step, seed

    Step k of simulation i equals `step(isf_i, psi_i, particles_i, jet_k)`
    with omega_t = float32(omega * float32(k * dt)), emit_start =
    (k-1) * emit_per_step mod nslots and counter = k.  The batch owns psi and
    the particles; copy them with set_psi / psi / set_particles / particles."""

    def __init__(self, sims, device: int = 0, tune: bool = True):
        if not torch.cuda.is_available():
            raise ISFError(_lib.ISF_ERR_CUDA, "no CUDA device: libisf has no CPU path")
        self.L = _lib.load()
        n = len(sims)
        arr = (_lib.IsfSimDesc * n)()
        self.shapes, self.nslots = [], []
        for i, s in enumerate(sims):
            d = arr[i]
            d.grid_res[:] = [int(x) for x in s["dims"]]
            d.physical_size[:] = [int(x) for x in s["physical_size"]]
            d.hbar = float(s["hbar"])
            d.dt = float(s["dt"])
            d.nslots = int(s.get("nslots", 0))
            j = s.get("jet")
            if j is not None:
                d.jet = 1
                d.phase_mode = int(j.get("phase_mode", PHASE_DOT))
                d.kvec[:] = [float(x) for x in j["kvec"]]
                d.omega = float(j["omega"])
                d.nozzle_cen[:] = [float(x) for x in j["cen"]]
                d.nozzle_len = float(j["len"])
                d.nozzle_rad = float(j["rad"])
                d.emit_mode = int(j.get("emit_mode", EMIT_RING))
                d.emit_per_step = int(j.get("emit_per_step", 0))
                d.seed = int(j.get("seed", 0))
            nx, ny, nz = (int(x) for x in s["dims"])
            self.shapes.append((nz, ny, nx, 4))
            self.nslots.append(int(d.nslots))
        b = C.c_void_p()
        _lib.check_batch(self.L.isf_batch_create(arr, n, int(device), 1 if tune else 0, C.byref(b)))
        self.b = b
        self.n = n
        self.device = torch.device("cuda", int(device))
        s = C.c_void_p()
        _lib.check_batch(self.L.isf_batch_get_stream(b, C.byref(s)), b)
        self.stream = torch.cuda.ExternalStream(s.value, device=self.device)

    def close(self):
        if getattr(self, "b", None):
            self.L.isf_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc):
        return _lib.check_batch(rc, self.b)

    def _src(self, t: torch.Tensor, shape):
        if tuple(t.shape) != tuple(shape) or t.dtype != torch.float32 or not t.is_contiguous():
            raise ISFError(_lib.ISF_ERR_INVALID, f"expected a contiguous float32 tensor of shape {shape}")
        if t.is_cuda:
            torch.cuda.current_stream(t.device).synchronize()
        return C.c_void_p(t.data_ptr())

    def set_psi(self, i: int, psi: torch.Tensor):
        self._chk(self.L.isf_batch_set_psi(self.b, int(i), self._src(psi, self.shapes[i])))

    def psi(self, i: int) -> torch.Tensor:
        out = torch.empty(self.shapes[i], dtype=torch.float32, device=self.device)
        self._chk(self.L.isf_batch_get_psi(self.b, int(i), C.c_void_p(out.data_ptr())))
        return out

    def set_particles(self, i: int, parts: torch.Tensor):
        self._chk(self.L.isf_batch_set_particles(self.b, int(i), self._src(parts, (self.nslots[i], 3))))

    def particles(self, i: int) -> torch.Tensor:
        out = torch.empty((self.nslots[i], 3), dtype=torch.float32, device=self.device)
        if self.nslots[i]:
            self._chk(self.L.isf_batch_get_particles(self.b, int(i), C.c_void_p(out.data_ptr())))
        return out

    def init_jet(self, iters: int = 10):
        """examples/benchmark.jl:28-31 for every jet simulation."""
        self._chk(self.L.isf_batch_init_jet(self.b, int(iters)))

    def step(self, nsteps: int = 1):
        self._chk(self.L.isf_batch_step(self.b, int(nsteps)))

    def set_step(self, k: int):
        self._chk(self.L.isf_batch_set_step(self.b, int(k)))

    def set_persistent(self, on: bool = True, spin_limit: int = 0, stall: bool = False):
        """Run each step(k) call as one launch of the persistent batch kernel
        (isf_batch_set_persistent); spin_limit bounds each device-side wait
        (<= 0: the default); stall makes the dependent passes wait on a flag
        nothing sets, so the launch times out (sync raises ISFError with
        ISF_ERR_TIMEOUT)."""
        mode = (_lib.PERSIST_ON if on else 0) | (_lib.PERSIST_STALL if stall else 0)
        self._chk(self.L.isf_batch_set_persistent(self.b, mode, int(spin_limit)))

    def sync(self):
        self._chk(self.L.isf_batch_sync(self.b))

    def classes(self):
        """(number of classes, class of every simulation)"""
        nc = C.c_int32()
        sc = (C.c_int32 * self.n)()
        self._chk(self.L.isf_batch_info(self.b, C.byref(nc), sc))
        return nc.value, list(sc)

    def tiles(self, cls: int) -> dict:
        t = (C.c_int32 * 6)()
        self._chk(self.L.isf_batch_tiles(self.b, int(cls), t))
        return dict(zip(_lib.TILE_KINDS, list(t)))

    def counters(self, i: int, reset: bool = False) -> dict:
        out = (C.c_uint64 * 2)()
        self._chk(self.L.isf_batch_counters(self.b, int(i), out, 1 if reset else 0))
        return {"clamps": int(out[0]), "live": int(out[1])}


# ---------------------------------------------------------------- adjoints
# The reference has no derivatives; these differentiate its operators
# (isf_adj_*).  Cotangents are float32 tensors shaped like their primal and
# are updated in place; psi's cotangent holds (dL/dRe, dL/dIm) per component.

def adj_schroedinger_flow(isf: ISF, psibar: torch.Tensor) -> torch.Tensor:
    check(isf.L.isf_adj_schroedinger_flow(isf.h, isf._psi(psibar)), isf.h)
    return psibar


def adj_normalize_psi(isf: ISF, psi_in: torch.Tensor, psibar: torch.Tensor) -> torch.Tensor:
    check(isf.L.isf_adj_normalize_psi(isf.h, isf._psi(psi_in), isf._psi(psibar)), isf.h)
    return psibar


def adj_pressure_project(isf: ISF, psi_in: torch.Tensor, psibar: torch.Tensor) -> torch.Tensor:
    check(isf.L.isf_adj_pressure_project(isf.h, isf._psi(psi_in), isf._psi(psibar)), isf.h)
    return psibar


def adj_restrict_velocity(isf: ISF, psi_in: torch.Tensor, psibar: torch.Tensor, kvec, omgterm: float = 0.0, *,
                          nozzle, isjetarr=None, phase_mode: int = PHASE_REFERENCE_SUM):
    """Returns the cotangents of (kvec[0], kvec[1], kvec[2], omgterm)."""
    cen, length, rad = nozzle
    out = (C.c_double * 4)()
    check(isf.L.isf_adj_restrict_velocity(isf.h, isf._psi(psi_in), isf._psi(psibar), f3(kvec), _ptr(isjetarr),
                                          f3(cen), float(length), float(rad), float(omgterm), int(phase_mode), out),
          isf.h)
    return [float(v) for v in out]


def adj_velocity_one_form(isf: ISF, psi: torch.Tensor, psibar: torch.Tensor, hbar: float = 1.0,
                          sharp: bool = False) -> torch.Tensor:
    """Consumes the handle's velocity cotangent (see velocity_bar)."""
    check(isf.L.isf_adj_velocity_one_form(isf.h, isf._psi(psi), float(hbar), 1 if sharp else 0, isf._psi(psibar)),
          isf.h)
    return psibar


def adj_staggered_advect(isf: ISF, particles: torch.Tensor, particles_bar: torch.Tensor) -> torch.Tensor:
    ptr, P = isf._parts(particles)
    bptr, Pb = isf._parts(particles_bar)
    if P != Pb:
        raise ISFError(_lib.ISF_ERR_INVALID, "particles and particles_bar differ in length")
    check(isf.L.isf_adj_staggered_advect(isf.h, ptr, bptr, P), isf.h)
    return particles_bar


def get_velocity_bar(isf: ISF) -> torch.Tensor:
    out = torch.empty(isf.shape + (3,), dtype=torch.float32, device=isf.device)
    check(isf.L.isf_adj_get_velocity_bar(isf.h, _ptr(out)), isf.h)
    return out


def set_velocity_bar(isf: ISF, vbar: torch.Tensor) -> None:
    if vbar.dtype != torch.float32 or tuple(vbar.shape) != isf.shape + (3,):
        raise ISFError(_lib.ISF_ERR_INVALID, f"velocity cotangent must be float32 {isf.shape + (3,)}")
    check(isf.L.isf_adj_set_velocity_bar(isf.h, _ptr(vbar)), isf.h)


def adj_step(isf: ISF, psi_in: torch.Tensor, particles_in, jet, psibar: torch.Tensor, particles_bar=None):
    """Reverse of step(isf, psi_in, particles_in, jet); returns the cotangents
    of (kvec[0..2], omega_t)."""
    ptr, P = isf._parts(particles_in)
    bptr, Pb = isf._parts(particles_bar)
    if P != Pb:
        raise ISFError(_lib.ISF_ERR_INVALID, "particles and particles_bar differ in length")
    a = step_args(jet)
    out = (C.c_double * 4)()
    check(isf.L.isf_adj_step(isf.h, isf._psi(psi_in), ptr, P, C.byref(a), isf._psi(psibar), bptr, out), isf.h)
    return [float(v) for v in out]


def adj_problem(nsteps, checkpoint_every, kvec, omega, nozzle, init_iters=10, phase_mode=PHASE_DOT):
    p = _lib.IsfAdjProblem()
    p.nsteps = int(nsteps)
    p.checkpoint_every = int(checkpoint_every)
    p.init_iters = int(init_iters)
    p.phase_mode = int(phase_mode)
    p.kvec[:] = [float(x) for x in kvec]
    p.omega = float(omega)
    cen, length, rad = nozzle
    p.nozzle_cen[:] = [float(x) for x in cen]
    p.nozzle_len = float(length)
    p.nozzle_rad = float(rad)
    return p


def adj_loss(isf: ISF, problem, psi0, particles0, targets) -> float:
    ptr, P = isf._parts(particles0)
    tptr, Pt = isf._parts(targets)
    if P != Pt:
        raise ISFError(_lib.ISF_ERR_INVALID, "targets differ in length from the particles")
    out = C.c_double()
    check(isf.L.isf_adj_loss(isf.h, C.byref(problem), isf._psi(psi0), ptr, P, tptr, C.byref(out)), isf.h)
    return float(out.value)


def adj_gradient(isf: ISF, problem, psi0, particles0, targets):
    """(L, dL/dpsi0, dL/dparticles0, dL/d(kvec[0], kvec[1], kvec[2], omega))."""
    ptr, P = isf._parts(particles0)
    tptr, Pt = isf._parts(targets)
    if P != Pt:
        raise ISFError(_lib.ISF_ERR_INVALID, "targets differ in length from the particles")
    gpsi = torch.empty_like(psi0)
    gparts = torch.empty_like(particles0)
    loss = C.c_double()
    jb = (C.c_double * 4)()
    check(isf.L.isf_adj_gradient(isf.h, C.byref(problem), isf._psi(psi0), ptr, P, tptr, C.byref(loss),
                                 isf._psi(gpsi), _ptr(gparts), jb), isf.h)
    return float(loss.value), gpsi, gparts, [float(v) for v in jb]


class ParticleLoss(torch.autograd.Function):
    """The jet run's particle loss as a differentiable function of (psi0,
    kvec, omega) -- the torch counterpart of a ChainRulesCore rrule over
    isf_adj_gradient.  The forward computes the loss and the gradient in one
    checkpointed pass; backward scales the stored gradient.

        L = ParticleLoss.apply(psi0, kvec, omega, isf, problem, particles0, targets)
    """

    @staticmethod
    def forward(ctx, psi0, kvec, omega, isf, problem, particles0, targets):
        kv = [float(x) for x in kvec.detach().cpu().tolist()]
        p = adj_problem(problem.nsteps, problem.checkpoint_every, kv, float(omega), (
            tuple(problem.nozzle_cen), problem.nozzle_len, problem.nozzle_rad), problem.init_iters, problem.phase_mode)
        loss, gpsi, _, jb = adj_gradient(isf, p, psi0.detach().contiguous(), particles0, targets)
        ctx.save_for_backward(gpsi)
        ctx.jb = jb
        return torch.tensor(loss, dtype=torch.float64, device=psi0.device)

    @staticmethod
    def backward(ctx, gout):
        (gpsi,) = ctx.saved_tensors
        g = gout.to(torch.float32)
        gk = torch.tensor(ctx.jb[:3], dtype=torch.float32, device=gpsi.device) * g
        gw = torch.tensor(ctx.jb[3], dtype=torch.float32, device=gpsi.device) * g
        return gpsi * g, gk, gw, None, None, None, None


from . import matlabport  # noqa: E402  (the FP64 structure-of-arrays front-end)
