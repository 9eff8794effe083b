"""MatlabPort -- the reference's FP64 structure-of-arrays formulation
(src/MatlabPort.jl) as a second front-end over libisf's kernels.

MatlabPort.jl restates the operators of src/parallel.jl with separate
Complex{Float64} arrays psi1, psi2, Float64 velocity components vx, vy, vz and
a `Particles` type holding Float32 x, y, z vectors with a list of active
slots; its driver is examples/matlabport/simple.jl.  The same names are kept
here.  Every function converts its FP64 arrays to the handle's FP32 layouts
with a libisf kernel, runs the libisf kernels of the operator, and converts
the result back (FP32 arithmetic inside, FP64 in and out).

Arrays are indexed [x, y, z] as in Julia: a field of an ISF with resolution
(nx, ny, nz) is a tensor of shape (nx, ny, nz) whose memory is column-major
(x fastest, strides (1, nx, nx*ny)).  CUDA tensors are used in place and the
results are CUDA tensors; numpy arrays are copied to the device and the
results come back as numpy arrays (the reference's Arrays live on the host).
Slot lists (`Particles.active`, `Keep` indices) are 0-based int64.

Every call runs on the legacy default stream, the one torch's default-stream
work uses, so the calls are ordered with each other (including the ones
without an ISF argument) and with the caller's torch operations.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _lib
from ._lib import EMIT_RING_PLANE, ISFError, check, f3

__all__ = [
    "ISF", "Particles", "land", "ndgrid", "SchroedingerFlow", "StaggeredSharp", "VelocityOneForm", "PoissonSolve",
    "GaugeTransform", "PressureProject", "Normalize", "Div", "append", "StaggeredAdvect", "Keep",
    "StaggeredVelocity", "remove_dead", "add_ring", "is_jet", "restrict",
]


def _vp(t: torch.Tensor | None):
    return None if t is None else C.c_void_p(t.data_ptr())


def land(a, b):
    """Elementwise logical and (MatlabPort.jl:4-8)."""
    if isinstance(a, np.ndarray) or isinstance(b, np.ndarray):
        return np.logical_and(np.asarray(a) != 0, np.asarray(b) != 0)
    return torch.logical_and(torch.as_tensor(a) != 0, torch.as_tensor(b) != 0)


def ndgrid(*vs):
    """MATLAB ndgrid (MatlabPort.jl:10-37): one array per argument, the k-th
    varying along dimension k."""
    arrs = np.meshgrid(*[np.asarray(v) for v in vs], indexing="ij")
    return arrs[0].copy() if len(vs) == 1 else tuple(a.copy() for a in arrs)


class _Grid:
    """The FP32 libisf handle behind one grid, and its conversion buffers."""

    def __init__(self, vol_size, vol_res, hbar, dt, device):
        from . import ISF as _ISF
        from . import STREAM_LEGACY
        self.isf = _ISF(vol_size, vol_res, hbar, dt, device=device, stream=STREAM_LEGACY)
        self.L = self.isf.L
        self.h = self.isf.h
        self.device = self.isf.device
        self.res = tuple(int(r) for r in vol_res)
        nx, ny, nz = self.res
        self.N = nx * ny * nz
        self.psi = torch.empty((self.N, 4), dtype=torch.float32, device=self.device)
        self.f = torch.empty(self.N, dtype=torch.float32, device=self.device)
        self.q = torch.empty(self.N, dtype=torch.float32, device=self.device)
        self.qi = torch.empty(self.N, dtype=torch.float32, device=self.device)

    def chk(self, rc):
        return check(rc, self.h)

    # ---- [x, y, z] column-major FP64 tensors
    def field(self, a, dtype=torch.float64):
        host = isinstance(a, np.ndarray)
        t = torch.from_numpy(np.asarray(a)) if host else torch.as_tensor(a)
        if tuple(t.shape) != self.res:
            raise ISFError(_lib.ISF_ERR_INVALID, f"array of shape {tuple(t.shape)}, the grid is {self.res}")
        t = t.to(device=self.device, dtype=dtype)
        nx, ny, _ = self.res
        if t.stride() != (1, nx, nx * ny) or t.data_ptr() % 16:
            t = t.permute(2, 1, 0).contiguous().permute(2, 1, 0)
        return t, host

    def new(self, dtype=torch.float64):
        nx, ny, nz = self.res
        return torch.empty((nz, ny, nx), dtype=dtype, device=self.device).permute(2, 1, 0)

    def psi_in(self, psi1, psi2):
        a, h1 = self.field(psi1, torch.complex128)
        b, h2 = self.field(psi2, torch.complex128)
        self.chk(self.L.isf_psi_from_f64(self.h, _vp(a), _vp(b), _vp(self.psi)))
        return h1 or h2

    def psi_out(self, host):
        a, b = self.new(torch.complex128), self.new(torch.complex128)
        self.chk(self.L.isf_psi_to_f64(self.h, _vp(self.psi), _vp(a), _vp(b)))
        return _out(a, host), _out(b, host)

    def vel_in(self, vx, vy, vz):
        (a, h1), (b, h2), (c, h3) = self.field(vx), self.field(vy), self.field(vz)
        self.chk(self.L.isf_velocity_from_f64(self.h, _vp(a), _vp(b), _vp(c)))
        return h1 or h2 or h3

    def vel_out(self, host):
        a, b, c = self.new(), self.new(), self.new()
        self.chk(self.L.isf_velocity_to_f64(self.h, _vp(a), _vp(b), _vp(c)))
        return _out(a, host), _out(b, host), _out(c, host)

    def real_in(self, f, dst, part=0, scale=1.0):
        """dst <- scale * (real part, part 0, or imaginary part, 1) of f"""
        if torch.is_tensor(f) and f.is_complex() or isinstance(f, np.ndarray) and np.iscomplexobj(f):
            t, host = self.field(f, torch.complex128)
            src = torch.view_as_real(t.permute(2, 1, 0)).reshape(-1)
            self.chk(self.L.isf_real_from_f64(self.h, C.c_void_p(src.data_ptr() + 8 * part), 2, float(scale),
                                              _vp(dst), self.N))
            return host, True
        t, host = self.field(f)
        if part == 0:
            self.chk(self.L.isf_real_from_f64(self.h, _vp(t), 1, float(scale), _vp(dst), self.N))
        else:
            dst.zero_()
        return host, False

    def real_out(self, src, host):
        t = self.new()
        self.chk(self.L.isf_real_to_f64(self.h, _vp(src), _vp(t), self.N))
        return _out(t, host)

    def complex_out(self, re, im, host):
        t = self.new(torch.complex128)
        self.chk(self.L.isf_complex_to_f64(self.h, _vp(re), _vp(im), _vp(t), self.N))
        return _out(t, host)


def _out(t: torch.Tensor, host: bool):
    return t.cpu().numpy() if host else t


_contexts: dict = {}
# the grid of the handle behind the particle calls that do not touch a field
_SLOT_GRID = (16, 8, 8)


def _context(shape, device) -> _Grid:
    """A grid for the operators without an ISF argument (Normalize,
    GaugeTransform): the box size does not enter them."""
    key = (tuple(int(s) for s in shape), int(device))
    g = _contexts.get(key)
    if g is None:
        g = _contexts[key] = _Grid(key[0], key[0], 1.0, 1.0, key[1])
    return g


def _device_of(*arrays) -> int:
    for a in arrays:
        if torch.is_tensor(a) and a.is_cuda:
            return a.device.index or 0
    return torch.cuda.current_device()


class ISF:
    """MatlabPort.ISF(vol_size, vol_res, hbar, dt) (MatlabPort.jl:38-73,
    BuildSchroedinger :75-83).  Scalar fields as in the reference; the grid
    arrays (iix.., px.., mask) are built on first use, as FP64 [x, y, z]
    tensors on the device."""

    def __init__(self, vol_size, vol_res, hbar, dt, device: int | None = None):
        self.sizex, self.sizey, self.sizez = (int(v) for v in vol_size)
        self.resx, self.resy, self.resz = (int(round(r)) for r in vol_res)
        self.dx = self.sizex / self.resx
        self.dy = self.sizey / self.resy
        self.dz = self.sizez / self.resz
        self.ix = range(1, self.resx + 1)
        self.iy = range(1, self.resy + 1)
        self.iz = range(1, self.resz + 1)
        self.hbar = float(hbar)
        self.dt = float(dt)
        dev = torch.cuda.current_device() if device is None else int(device)
        self._g = _Grid((self.sizex, self.sizey, self.sizez), (self.resx, self.resy, self.resz), self.hbar, self.dt,
                        dev)
        self._arrays = None

    def _grid_arrays(self):
        if self._arrays is None:
            iix, iiy, iiz = ndgrid(np.arange(1, self.resx + 1), np.arange(1, self.resy + 1),
                                   np.arange(1, self.resz + 1))
            fac = -4 * np.pi ** 2 * self.hbar
            kx = (iix - 1 - self.resx / 2) / self.sizex
            ky = (iiy - 1 - self.resy / 2) / self.sizey
            kz = (iiz - 1 - self.resz / 2) / self.sizez
            mask = np.exp(1j * fac * (kx ** 2 + ky ** 2 + kz ** 2) * self.dt / 2.0)
            g = self._g
            self._arrays = {
                "iix": g.field(iix, torch.int64)[0], "iiy": g.field(iiy, torch.int64)[0],
                "iiz": g.field(iiz, torch.int64)[0],
                "px": g.field((iix - 1) * self.dx)[0], "py": g.field((iiy - 1) * self.dy)[0],
                "pz": g.field((iiz - 1) * self.dz)[0], "mask": g.field(mask, torch.complex128)[0],
            }
        return self._arrays

    def __getattr__(self, name):
        if name in ("iix", "iiy", "iiz", "px", "py", "pz", "mask"):
            return self._grid_arrays()[name]
        raise AttributeError(name)


def SchroedingerFlow(obj: ISF, psi1, psi2):
    """MatlabPort.jl:87-93: solves the Schroedinger equation for dt."""
    g = obj._g
    host = g.psi_in(psi1, psi2)
    g.chk(g.L.isf_schroedinger_flow(g.h, _vp(g.psi)))
    return g.psi_out(host)


def StaggeredSharp(obj: ISF, vx, vy, vz):
    """MatlabPort.jl:99-104: the staggered vector field v^sharp = v / d."""
    g = obj._g
    host = g.vel_in(vx, vy, vz)
    g.chk(g.L.isf_staggered_sharp(g.h))
    return g.vel_out(host)


def VelocityOneForm(obj: ISF, psi1, psi2, hbar=1.0):
    """MatlabPort.jl:106-126: v_a = hbar angle(conj psi1 psi1[+e_a] + conj psi2 psi2[+e_a])."""
    g = obj._g
    host = g.psi_in(psi1, psi2)
    g.chk(g.L.isf_velocity_one_form(g.h, _vp(g.psi), float(hbar)))
    return g.vel_out(host)


def PoissonSolve(obj: ISF, f):
    """MatlabPort.jl:128-138: IFFT(fac FFT(f)), fac = -1/(4 sum sin^2(pi k/n)/d^2),
    zero mode 0; complex128 result.  A complex f is solved part by part
    (the solve is linear); for a real f the imaginary part is 0 (the
    reference's is round-off)."""
    g = obj._g
    host, cplx = g.real_in(f, g.f, 0)
    g.chk(g.L.isf_poisson_solve(g.h, _vp(g.f), _vp(g.q)))
    im = None
    if cplx:
        g.real_in(f, g.f, 1)
        g.chk(g.L.isf_poisson_solve(g.h, _vp(g.f), _vp(g.qi)))
        im = g.qi
    return g.complex_out(g.q, im, host)


def GaugeTransform(psi1, psi2, q):
    """MatlabPort.jl:140-145: psi * exp(i q) with complex q."""
    shape = tuple(psi1.shape)
    g = _context(shape, _device_of(psi1, psi2, q))
    host = g.psi_in(psi1, psi2)
    # the kernel multiplies by exp(-i q'): q' = -q
    _, cplx = g.real_in(q, g.q, 0, -1.0)
    if cplx:
        g.real_in(q, g.qi, 1, -1.0)
    g.chk(g.L.isf_gauge_transform(g.h, _vp(g.psi), _vp(g.q), _vp(g.qi) if cplx else None))
    return g.psi_out(host)


def PressureProject(obj: ISF, psi1, psi2):
    """MatlabPort.jl:147-153: one-form (hbar 1), Div, PoissonSolve, gauge."""
    g = obj._g
    host = g.psi_in(psi1, psi2)
    g.chk(g.L.isf_pressure_project(g.h, _vp(g.psi)))
    return g.psi_out(host)


def Normalize(psi1, psi2):
    """MatlabPort.jl:155-160: psi / sqrt(|psi1|^2 + |psi2|^2)."""
    g = _context(tuple(psi1.shape), _device_of(psi1, psi2))
    host = g.psi_in(psi1, psi2)
    g.chk(g.L.isf_normalize_psi(g.h, _vp(g.psi)))
    return g.psi_out(host)


def Div(obj: ISF, vx, vy, vz):
    """MatlabPort.jl:162-170: sum_a (v_a - v_a[-e_a]) / d_a^2."""
    g = obj._g
    host = g.vel_in(vx, vy, vz)
    g.chk(g.L.isf_div(g.h, _vp(g.f)))
    return g.real_out(g.f, host)


def is_jet(obj: ISF, cen, length, rad):
    """The nozzle mask of the MatlabPort driver (examples/matlabport/simple.jl:34-37),
    land(|px - c_x| <= len/2, (py - c_y)^2 + (pz - c_z)^2 <= rad^2), from the
    ISF's FP64 grid positions: a Bool [x, y, z] tensor (set-up, once)."""
    return land(torch.abs(obj.px - cen[0]) <= length / 2,
                (obj.py - cen[1]) ** 2 + (obj.pz - cen[2]) ** 2 <= rad ** 2)


def restrict(obj: ISF, psi1, psi2, is_jet, kvec, omega_t):
    """The nozzle constraint of the MatlabPort driver (examples/matlabport/simple.jl:104-111):
    inside is_jet (a Bool [x, y, z] array), psi_c = |psi_c| exp(i (k . x - omega t))."""
    g = obj._g
    host = g.psi_in(psi1, psi2)
    m, _ = g.field(is_jet, torch.uint8)
    g.chk(g.L.isf_restrict_velocity(g.h, _vp(g.psi), f3(kvec), _vp(m), f3((0.0, 0.0, 0.0)), 0.0, 0.0,
                                    float(omega_t), _lib.PHASE_DOT))
    return g.psi_out(host)


class Particles:
    """MatlabPort.Particles (MatlabPort.jl:178-196): Float32 x, y, z slot
    vectors, the number of filled slots and the list of active slots
    (0-based int64)."""

    def __init__(self, x, y, z, length: int = 0, active=None, device: int | None = None):
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else int(device))
        self.x, self.y, self.z = (torch.as_tensor(v, dtype=torch.float32).to(dev).contiguous() for v in (x, y, z))
        if not (self.x.shape == self.y.shape == self.z.shape) or self.x.dim() != 1:
            raise ISFError(_lib.ISF_ERR_INVALID, "x, y, z must be vectors of one length")
        self.length = int(length)
        self.active = (torch.zeros(0, dtype=torch.int64, device=dev) if active is None
                       else torch.as_tensor(active, dtype=torch.int64).to(dev).contiguous())

    def __len__(self):
        return self.length

    @property
    def nslots(self) -> int:
        return int(self.x.shape[0])


def append(p: Particles, x, y, z):
    """Base.append!(p::Particles, x, y, z) (MatlabPort.jl:186-196): the new
    positions fill the slots after p.length and become active."""
    n = len(x)
    if not n + p.length < p.nslots:
        raise ISFError(_lib.ISF_ERR_INVALID, "append: no free slots (the reference asserts length(x) + p.length < "
                                             "length(p.x))")
    r = slice(p.length, p.length + n)
    for dst, src in ((p.x, x), (p.y, y), (p.z, z)):
        dst[r].copy_(torch.as_tensor(src, dtype=torch.float32))
    p.active = torch.cat([p.active, torch.arange(p.length, p.length + n, dtype=torch.int64, device=p.x.device)])
    p.length += n


def add_ring(p: Particles, n: int, cen, rad: float, seed: int, counter: int):
    """The particle birth of the MatlabPort driver (examples/matlabport/simple.jl:112-116):
    n particles on the ring of radius 0.9 rad in the plane x = cen.x, angles
    from the seeded Philox stream (seed, counter) instead of rand(Float32),
    appended as by append!."""
    if not n + p.length < p.nslots:
        raise ISFError(_lib.ISF_ERR_INVALID, "add_ring: no free slots")
    g = _context(_SLOT_GRID, p.x.device.index or 0)
    g.chk(g.L.isf_add_particles_soa(g.h, _vp(p.x), _vp(p.y), _vp(p.z), p.nslots, p.length, int(n), f3(cen), 0.0,
                                    float(rad), int(seed), int(counter), EMIT_RING_PLANE))
    p.active = torch.cat([p.active, torch.arange(p.length, p.length + n, dtype=torch.int64, device=p.x.device)])
    p.length += int(n)


def StaggeredAdvect(p: Particles, torus: ISF, vx, vy, vz, dt):
    """MatlabPort.jl:200-222: RK4 of the active particles on the staggered
    velocity (vx, vy, vz), without a box test."""
    g = torus._g
    g.vel_in(vx, vy, vz)
    g.chk(g.L.isf_advect_active(g.h, _vp(p.x), _vp(p.y), _vp(p.z), p.nslots, _vp(p.active), int(p.active.numel()),
                                float(dt)))


def Keep(particle: Particles, ind):
    """MatlabPort.jl:228-233: x, y, z become x[ind], y[ind], z[ind]."""
    ind = torch.as_tensor(ind, dtype=torch.int64).to(particle.x.device).contiguous()
    n = int(ind.numel())
    if n and (int(ind.min()) < 0 or int(ind.max()) >= particle.nslots):
        raise ISFError(_lib.ISF_ERR_INVALID, "Keep: index out of range")
    g = _context(_SLOT_GRID, particle.x.device.index or 0)
    o = [torch.empty(n, dtype=torch.float32, device=particle.x.device) for _ in range(3)]
    g.chk(g.L.isf_gather_particles(g.h, _vp(particle.x), _vp(particle.y), _vp(particle.z), particle.nslots, _vp(ind),
                                   n, _vp(o[0]), _vp(o[1]), _vp(o[2])))
    particle.x, particle.y, particle.z = o


def StaggeredVelocity(pxf, pyf, pzf, torus: ISF, vx, vy, vz):
    """MatlabPort.jl:238-273: the staggered velocity at the points (float32
    positions; float64 results)."""
    g = torus._g
    host = g.vel_in(vx, vy, vz)
    pts = [torch.as_tensor(v).to(device=g.device, dtype=torch.float32).contiguous() for v in (pxf, pyf, pzf)]
    n = int(pts[0].numel())
    u = [torch.empty(n, dtype=torch.float32, device=g.device) for _ in range(3)]
    g.chk(g.L.isf_staggered_velocity(g.h, _vp(pts[0]), _vp(pts[1]), _vp(pts[2]), n, _vp(u[0]), _vp(u[1]),
                                     _vp(u[2])))
    out = []
    for t in u:
        d = torch.empty(n, dtype=torch.float64, device=g.device)
        g.chk(g.L.isf_real_to_f64(g.h, _vp(t), _vp(d), n))
        out.append(d.cpu().numpy() if host else d)
    return tuple(out)


def remove_dead(particles: Particles, torus: ISF):
    """removethedead! (examples/matlabport/simple.jl:67-74): keep the active
    slots strictly inside the box, in order."""
    g = torus._g
    n = int(particles.active.numel())
    out = torch.empty(max(n, 1), dtype=torch.int64, device=particles.x.device)
    cnt = torch.zeros(1, dtype=torch.int64, device=particles.x.device)
    g.chk(g.L.isf_keep_inside(g.h, _vp(particles.x), _vp(particles.y), _vp(particles.z), particles.nslots,
                              _vp(particles.active), n, _vp(out), _vp(cnt)))
    g.isf.sync()
    particles.active = out[:int(cnt.item())]
