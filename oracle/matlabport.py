"""ORACLE cross-spec -- test infrastructure only.

Independent FP64 numpy restatement of src/MatlabPort.jl (the reference's
line-by-line port of the paper's MATLAB code) and of its driver
examples/matlabport/simple.jl.  It shares no code with oracle/isf_oracle.cpp:
FFTs are numpy.fft, operators are whole-array numpy expressions in the
MatlabPort formulation (separate psi1/psi2 arrays, SoA velocity, fftshift
applied to the spectrum rather than to the mask).  tests/test_oracle_cpu.py
compares the two; tests/golden/make_golden.py uses this module to write the
golden fixtures.

Arrays are indexed [x, y, z] (shape (nx, ny, nz)), the Julia index order.
"""
from __future__ import annotations

import numpy as np


class MatlabISF:
    """MatlabPort.ISF (src/MatlabPort.jl:38-73) + BuildSchroedinger (:75-83)."""

    def __init__(self, vol_size, vol_res, hbar, dt):
        self.sizex, self.sizey, self.sizez = (float(v) for v in vol_size)
        self.resx, self.resy, self.resz = (int(r) for r in vol_res)
        self.dx = self.sizex / self.resx
        self.dy = self.sizey / self.resy
        self.dz = self.sizez / self.resz
        self.hbar = float(hbar)
        self.dt = float(dt)
        ix = np.arange(1, self.resx + 1)
        iy = np.arange(1, self.resy + 1)
        iz = np.arange(1, self.resz + 1)
        self.iix, self.iiy, self.iiz = np.meshgrid(ix, iy, iz, indexing="ij")  # ndgrid
        self.px = (self.iix - 1) * self.dx
        self.py = (self.iiy - 1) * self.dy
        self.pz = (self.iiz - 1) * self.dz
        fac = -4 * np.pi ** 2 * self.hbar
        kx = (self.iix - 1 - self.resx / 2) / self.sizex
        ky = (self.iiy - 1 - self.resy / 2) / self.sizey
        kz = (self.iiz - 1 - self.resz / 2) / self.sizez
        lam = fac * (kx ** 2 + ky ** 2 + kz ** 2)
        self.mask = np.exp(1j * lam * self.dt / 2.0)


def schroedinger_flow(obj, psi1, psi2):
    """MatlabPort.jl:87-93."""
    p1 = np.fft.fftshift(np.fft.fftn(psi1))
    p2 = np.fft.fftshift(np.fft.fftn(psi2))
    p1 = p1 * obj.mask
    p2 = p2 * obj.mask
    return np.fft.ifftn(np.fft.ifftshift(p1)), np.fft.ifftn(np.fft.ifftshift(p2))


def staggered_sharp(obj, vx, vy, vz):
    """MatlabPort.jl:99-104."""
    return vx / obj.dx, vy / obj.dy, vz / obj.dz


def velocity_one_form(obj, psi1, psi2, hbar=1.0):
    """MatlabPort.jl:106-126 (+1 neighbour with wrap)."""
    def nb(a, ax):
        return np.roll(a, -1, axis=ax)
    vx = np.angle(np.conj(psi1) * nb(psi1, 0) + np.conj(psi2) * nb(psi2, 0))
    vy = np.angle(np.conj(psi1) * nb(psi1, 1) + np.conj(psi2) * nb(psi2, 1))
    vz = np.angle(np.conj(psi1) * nb(psi1, 2) + np.conj(psi2) * nb(psi2, 2))
    return vx * hbar, vy * hbar, vz * hbar


def poisson_solve(obj, f):
    """MatlabPort.jl:128-138."""
    F = np.fft.fftn(f)
    sx = np.sin(np.pi * (obj.iix - 1) / obj.resx) / obj.dx
    sy = np.sin(np.pi * (obj.iiy - 1) / obj.resy) / obj.dy
    sz = np.sin(np.pi * (obj.iiz - 1) / obj.resz) / obj.dz
    denom = sx ** 2 + sy ** 2 + sz ** 2
    with np.errstate(divide="ignore"):
        fac = -0.25 / denom
    fac[0, 0, 0] = 0.0
    return np.fft.ifftn(F * fac)


def gauge_transform(psi1, psi2, q):
    """MatlabPort.jl:140-145."""
    eiq = np.exp(1j * q)
    return psi1 * eiq, psi2 * eiq


def div(obj, vx, vy, vz):
    """MatlabPort.jl:162-170 (-1 neighbour with wrap)."""
    f = (vx - np.roll(vx, 1, axis=0)) / obj.dx ** 2
    f = f + (vy - np.roll(vy, 1, axis=1)) / obj.dy ** 2
    f = f + (vz - np.roll(vz, 1, axis=2)) / obj.dz ** 2
    return f


def pressure_project(obj, psi1, psi2):
    """MatlabPort.jl:147-153."""
    vx, vy, vz = velocity_one_form(obj, psi1, psi2)
    d = div(obj, vx, vy, vz)
    q = -poisson_solve(obj, d)
    return gauge_transform(psi1, psi2, q)


def normalize(psi1, psi2):
    """MatlabPort.jl:155-160."""
    n = np.sqrt(np.abs(psi1) ** 2 + np.abs(psi2) ** 2)
    return psi1 / n, psi2 / n


def is_jet(obj, cen, length, rad):
    """examples/matlabport/simple.jl:34-37."""
    return (np.abs(obj.px - cen[0]) <= length / 2) & \
        ((obj.py - cen[1]) ** 2 + (obj.pz - cen[2]) ** 2 <= rad ** 2)


def restrict(obj, psi1, psi2, isjet, kvec, omega_t):
    """examples/matlabport/simple.jl:107-111 (phase k.x - omega t)."""
    phase = kvec[0] * obj.px + kvec[1] * obj.py + kvec[2] * obj.pz - omega_t
    a1, a2 = np.abs(psi1), np.abs(psi2)
    psi1 = psi1.copy()
    psi2 = psi2.copy()
    psi1[isjet] = a1[isjet] * np.exp(1j * phase[isjet])
    psi2[isjet] = a2[isjet] * np.exp(1j * phase[isjet])
    return psi1, psi2


def staggered_velocity(px, py, pz, obj, vx, vy, vz):
    """MatlabPort.jl:237-273."""
    px = np.mod(px, obj.sizex)
    py = np.mod(py, obj.sizey)
    pz = np.mod(pz, obj.sizez)
    ix = np.floor(px / obj.dx).astype(np.int64)
    iy = np.floor(py / obj.dy).astype(np.int64)
    iz = np.floor(pz / obj.dz).astype(np.int64)
    ixp = np.mod(ix + 1, obj.resx)
    iyp = np.mod(iy + 1, obj.resy)
    izp = np.mod(iz + 1, obj.resz)
    wx = px - ix * obj.dx
    wy = py - iy * obj.dy
    wz = pz - iz * obj.dz
    ux = (1 - wz) * ((1 - wy) * vx[ix, iy, iz] + wy * vx[ix, iyp, iz]) + \
        wz * ((1 - wy) * vx[ix, iy, izp] + wy * vx[ix, iyp, izp])
    uy = (1 - wz) * ((1 - wx) * vy[ix, iy, iz] + wx * vy[ixp, iy, iz]) + \
        wz * ((1 - wx) * vy[ix, iy, izp] + wx * vy[ixp, iy, izp])
    uz = (1 - wy) * ((1 - wx) * vz[ix, iy, iz] + wx * vz[ixp, iy, iz]) + \
        wy * ((1 - wx) * vz[ix, iyp, iz] + wx * vz[ixp, iyp, iz])
    return ux, uy, uz


def staggered_advect(px, py, pz, obj, vx, vy, vz, dt):
    """MatlabPort.jl:201-222 (all given particles are active)."""
    k1 = staggered_velocity(px, py, pz, obj, vx, vy, vz)
    k2 = staggered_velocity(px + k1[0] * dt / 2, py + k1[1] * dt / 2, pz + k1[2] * dt / 2, obj, vx, vy, vz)
    k3 = staggered_velocity(px + k2[0] * dt / 2, py + k2[1] * dt / 2, pz + k2[2] * dt / 2, obj, vx, vy, vz)
    k4 = staggered_velocity(px + k3[0] * dt, py + k3[1] * dt, pz + k3[2] * dt, obj, vx, vy, vz)
    nx = px + dt / 6 * (k1[0] + 2 * k2[0] + 2 * k3[0] + k4[0])
    ny = py + dt / 6 * (k1[1] + 2 * k2[1] + 2 * k3[1] + k4[1])
    nz = pz + dt / 6 * (k1[2] + 2 * k2[2] + 2 * k3[2] + k4[2])
    return nx, ny, nz


def inside(obj, px, py, pz):
    """removethedead! criterion (examples/matlabport/simple.jl:9-14, 63-70)."""
    return (px > 0) & (px < obj.sizex) & (py > 0) & (py < obj.sizey) & (pz > 0) & (pz < obj.sizez)


def jet_step(obj, psi1, psi2, isjet, kvec, omega_t, parts=None):
    """One iteration of the MatlabPort driver loop (simple.jl:99-124) without
    particle birth; dead particles become (-1,-1,-1) as in parallel.jl."""
    psi1, psi2 = schroedinger_flow(obj, psi1, psi2)
    psi1, psi2 = normalize(psi1, psi2)
    psi1, psi2 = pressure_project(obj, psi1, psi2)
    psi1, psi2 = restrict(obj, psi1, psi2, isjet, kvec, omega_t)
    psi1, psi2 = pressure_project(obj, psi1, psi2)
    if parts is not None:
        vx, vy, vz = velocity_one_form(obj, psi1, psi2, obj.hbar)
        vx, vy, vz = staggered_sharp(obj, vx, vy, vz)
        alive = inside(obj, parts[:, 0], parts[:, 1], parts[:, 2])
        nx, ny, nz = staggered_advect(parts[:, 0], parts[:, 1], parts[:, 2], obj, vx, vy, vz, obj.dt)
        parts = np.stack([nx, ny, nz], axis=1)
        parts[~alive] = -1.0
    return psi1, psi2, parts


def driver_step(obj, psi1, psi2, isjet, kvec, omega_t, x, y, z, length, active, births):
    """One iteration of the MatlabPort driver loop (examples/matlabport/simple.jl:99-124)
    with its Particles semantics: the births (bx, by, bz) fill the slots after
    `length` and become active (append!, MatlabPort.jl:186-196), removethedead!
    keeps the active slots strictly inside the box in order, and
    StaggeredAdvect moves the active slots with no box test
    (MatlabPort.jl:200-222).  x, y, z are float32 slot vectors, updated in
    place; returns (psi1, psi2, length, active)."""
    psi1, psi2 = schroedinger_flow(obj, psi1, psi2)
    psi1, psi2 = normalize(psi1, psi2)
    psi1, psi2 = pressure_project(obj, psi1, psi2)
    psi1, psi2 = restrict(obj, psi1, psi2, isjet, kvec, omega_t)
    psi1, psi2 = pressure_project(obj, psi1, psi2)
    bx, by, bz = births
    n = len(bx)
    assert n + length < len(x)
    x[length:length + n], y[length:length + n], z[length:length + n] = bx, by, bz
    active = np.concatenate([np.asarray(active, np.int64), np.arange(length, length + n, dtype=np.int64)])
    length += n
    keep = inside(obj, x[active], y[active], z[active])
    active = active[keep]
    vx, vy, vz = velocity_one_form(obj, psi1, psi2, obj.hbar)
    vx, vy, vz = staggered_sharp(obj, vx, vy, vz)
    px, py, pz = (v[active].astype(np.float64) for v in (x, y, z))
    nx, ny, nz = staggered_advect(px, py, pz, obj, vx, vy, vz, obj.dt)
    x[active], y[active], z[active] = nx, ny, nz
    return psi1, psi2, length, active


def face_margin(obj, px, py, pz):
    """Distance of each point (after mod) to the nearest cell face in units of
    the cell, min over the axes: where it is tiny, an FP32 and an FP64
    evaluation may pick different cells."""
    m = np.full(np.shape(px), np.inf)
    for p, L, d in ((px, obj.sizex, obj.dx), (py, obj.sizey, obj.dy), (pz, obj.sizez, obj.dz)):
        q = np.mod(np.asarray(p, np.float64), L) / d
        m = np.minimum(m, np.abs(q - np.round(q)))
    return m


# ---- layout helpers between [x,y,z] component arrays and the oracle's
# (nz, ny, nx, 4) AoS psi
def to_aos(psi1, psi2):
    a = np.transpose(psi1, (2, 1, 0))
    b = np.transpose(psi2, (2, 1, 0))
    return np.ascontiguousarray(np.stack([a.real, a.imag, b.real, b.imag], axis=-1))


def from_aos(psi):
    a = psi[..., 0] + 1j * psi[..., 1]
    b = psi[..., 2] + 1j * psi[..., 3]
    return np.transpose(a, (2, 1, 0)).copy(), np.transpose(b, (2, 1, 0)).copy()


def vel_to_aos(vx, vy, vz):
    return np.ascontiguousarray(np.stack([np.transpose(v, (2, 1, 0)) for v in (vx, vy, vz)], axis=-1))
