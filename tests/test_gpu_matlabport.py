"""GPU parity of the FP64 structure-of-arrays front-end (matlabport.py, the
MatlabPort.jl API over libisf) against the independent FP64 numpy
restatement of src/MatlabPort.jl in oracle/matlabport.py.

Tolerances: relative L2 error 2e-5 for single operators (FP32 arithmetic
inside, FP64 in and out); particle positions within 1e-5 of the box size for
one advection and 1e-4 after a driver loop, away from cell faces (margin
1e-4 of a cell, where FP32 and FP64 may pick different cells); slot lists
(removethedead!, Keep) exact."""
import importlib

import numpy as np
import pytest
import torch

import matlabport as orc_mp
from helpers import rel, smooth_field, smooth_psi

pytestmark = pytest.mark.gpu

HBAR = 0.1
DT = 1 / 48
GRIDS = [((4, 2, 2), (64, 32, 32)), ((3, 2, 2), (48, 32, 32))]


@pytest.fixture(scope="module")
def mp(isfpkg):
    return importlib.import_module(isfpkg.__name__ + ".matlabport")


def xyz(a):
    """(nz, ny, nx) -> [x, y, z]"""
    return np.ascontiguousarray(np.transpose(a, (2, 1, 0)))


def psi_xyz(dims, seed):
    return orc_mp.from_aos(smooth_psi(dims, seed=seed))


def vel_xyz(dims, seed, scale=0.8, offset=0.5):
    rng = np.random.default_rng(seed)
    return tuple(xyz(smooth_field(dims, rng, scale=scale)) + offset for _ in range(3))


@pytest.mark.parametrize("L,dims", GRIDS)
def test_fields_match_matlabport_oracle(mp, L, dims):
    obj = mp.ISF(L, dims, HBAR, DT)
    oo = orc_mp.MatlabISF(L, dims, HBAR, DT)
    psi1, psi2 = psi_xyz(dims, 3)
    # every front-end call runs on the legacy default stream (ordered with the others and with torch)
    assert obj._g.isf.stream == torch.cuda.default_stream()

    a = mp.SchroedingerFlow(obj, psi1, psi2)
    b = orc_mp.schroedinger_flow(oo, psi1, psi2)
    assert isinstance(a[0], np.ndarray) and a[0].shape == tuple(dims)
    assert rel(a[0], b[0]) < 2e-5 and rel(a[1], b[1]) < 2e-5

    a = mp.Normalize(2.0 * psi1, 2.0 * psi2)
    b = orc_mp.normalize(2.0 * psi1, 2.0 * psi2)
    assert rel(a[0], b[0]) < 2e-5 and rel(a[1], b[1]) < 2e-5

    va = mp.VelocityOneForm(obj, psi1, psi2, HBAR)
    vb = orc_mp.velocity_one_form(oo, psi1, psi2, HBAR)
    for u, w in zip(va, vb):
        assert rel(u, w) < 2e-5

    sa = mp.StaggeredSharp(obj, *vb)
    sb = orc_mp.staggered_sharp(oo, *vb)
    for u, w in zip(sa, sb):
        assert rel(u, w) < 2e-5

    v1 = orc_mp.velocity_one_form(oo, psi1, psi2)
    fa = mp.Div(obj, *v1)
    fb = orc_mp.div(oo, *v1)
    assert rel(fa, fb) < 2e-5

    qa = mp.PoissonSolve(obj, fb)
    qb = orc_mp.poisson_solve(oo, fb)
    assert np.iscomplexobj(qa) and rel(qa, qb) < 2e-5
    f2 = fb + 0.5j * np.roll(fb, 3, axis=0)   # a complex right-hand side: solved part by part
    assert rel(mp.PoissonSolve(obj, f2), orc_mp.poisson_solve(oo, f2)) < 2e-5

    q = -qb + 0.01j * xyz(smooth_field(dims, np.random.default_rng(5)))
    a = mp.GaugeTransform(psi1, psi2, q)
    b = orc_mp.gauge_transform(psi1, psi2, q)
    assert rel(a[0], b[0]) < 2e-5 and rel(a[1], b[1]) < 2e-5
    a = mp.GaugeTransform(psi1, psi2, q.real)
    b = orc_mp.gauge_transform(psi1, psi2, q.real)
    assert rel(a[0], b[0]) < 2e-5 and rel(a[1], b[1]) < 2e-5

    a = mp.PressureProject(obj, psi1, psi2)
    b = orc_mp.pressure_project(oo, psi1, psi2)
    assert rel(a[0], b[0]) < 2e-5 and rel(a[1], b[1]) < 2e-5
    # CUDA tensors in: CUDA tensors out, the same values
    t1 = torch.from_numpy(psi1).cuda()
    t2 = torch.from_numpy(psi2).cuda()
    c = mp.PressureProject(obj, t1, t2)
    assert c[0].is_cuda and c[0].dtype == torch.complex128 and c[0].stride() == (1, dims[0], dims[0] * dims[1])
    assert np.array_equal(c[0].cpu().numpy(), a[0]) and np.array_equal(c[1].cpu().numpy(), a[1])


def rk_margin(oo, px, py, pz, v, dt):
    """The smallest cell-face margin over the four RK4 sample points."""
    m = orc_mp.face_margin(oo, px, py, pz)
    k1 = orc_mp.staggered_velocity(px, py, pz, oo, *v)
    pts = [(px + k1[0] * dt / 2, py + k1[1] * dt / 2, pz + k1[2] * dt / 2)]
    k2 = orc_mp.staggered_velocity(*pts[0], oo, *v)
    pts.append((px + k2[0] * dt / 2, py + k2[1] * dt / 2, pz + k2[2] * dt / 2))
    k3 = orc_mp.staggered_velocity(*pts[1], oo, *v)
    pts.append((px + k3[0] * dt, py + k3[1] * dt, pz + k3[2] * dt))
    for p in pts:
        m = np.minimum(m, orc_mp.face_margin(oo, *p))
    return m


@pytest.mark.parametrize("L,dims", GRIDS)
def test_particles_match_matlabport_oracle(mp, L, dims):
    obj = mp.ISF(L, dims, HBAR, DT)
    oo = orc_mp.MatlabISF(L, dims, HBAR, DT)
    v = vel_xyz(dims, 9)
    rng = np.random.default_rng(12)
    Lv = np.asarray(L, np.float64)

    # StaggeredVelocity at points inside and up to one box outside (wrapped by mod)
    P = 20000
    pts = (rng.uniform(-0.5, 1.5, (3, P)) * Lv[:, None]).astype(np.float32)
    ua = mp.StaggeredVelocity(pts[0], pts[1], pts[2], obj, *v)
    ub = orc_mp.staggered_velocity(*(p.astype(np.float64) for p in pts), oo, *v)
    ok = orc_mp.face_margin(oo, *pts) > 1e-4
    for a, b in zip(ua, ub):
        assert a.dtype == np.float64
        assert np.abs(a - b)[ok].max() < 1e-5

    # StaggeredAdvect of an active subset, some of it outside the box (no box test)
    nslots, length = 30000, 20000
    x0 = (rng.uniform(0, 1, (3, nslots)) * Lv[:, None]).astype(np.float32)
    x0[0, :500] += np.float32(L[0])      # outside: still advected, wrapped inside the interpolation
    active = np.sort(rng.choice(length, 12000, replace=False)).astype(np.int64)
    p = mp.Particles(x0[0], x0[1], x0[2], length, active)
    vel = mp.StaggeredSharp(obj, *v)
    mp.StaggeredAdvect(p, obj, *vel, DT)
    out = np.stack([p.x.cpu().numpy(), p.y.cpu().numpy(), p.z.cpu().numpy()])
    velb = orc_mp.staggered_sharp(oo, *v)
    pa = [x0[k, active].astype(np.float64) for k in range(3)]
    nb = orc_mp.staggered_advect(*pa, oo, *velb, DT)
    ok = rk_margin(oo, *pa, velb, DT) > 1e-4
    assert ok.mean() > 0.95
    for k in range(3):
        assert (np.abs(out[k, active] - nb[k])[ok] / min(L)).max() < 1e-5
    rest = np.setdiff1d(np.arange(nslots), active)
    assert np.array_equal(out[:, rest], x0[:, rest])      # inactive slots untouched

    # removethedead!: the active slots strictly inside the box, in order
    out[1, active[::7]] = -0.25
    out[2, active[::11]] = np.float32(L[2])
    p = mp.Particles(out[0], out[1], out[2], length, active)
    mp.remove_dead(p, obj)
    keep = orc_mp.inside(oo, out[0, active], out[1, active], out[2, active])
    assert np.array_equal(p.active.cpu().numpy(), active[keep])
    q = mp.Particles(out[0], out[1], out[2], 0, np.zeros(0, np.int64))
    mp.remove_dead(q, obj)
    assert q.active.numel() == 0

    # Keep(particle, ind)
    ind = rng.integers(0, nslots, 777)
    mp.Keep(p, ind)
    assert np.array_equal(p.x.cpu().numpy(), out[0, ind]) and np.array_equal(p.z.cpu().numpy(), out[2, ind])
    with pytest.raises(Exception):
        mp.Keep(p, [0, 10 ** 6])


def test_ring_birth_matches_oracle(mp, oracle_mod, cfgs):
    """add_ring (the MatlabPort driver's birth ring, seeded Philox) against the
    oracle's emission in mode 3, and append! bookkeeping."""
    noz = cfgs.JET_NOZZLE
    n, slots = 3000, 10000
    p = mp.Particles(np.zeros(slots), np.zeros(slots), np.zeros(slots))
    mp.append(p, [0.5, 0.6], [0.5, 0.6], [0.5, 0.6])
    mp.add_ring(p, n, noz["cen"], noz["rad"], seed=4, counter=7)
    assert p.length == n + 2 and np.array_equal(p.active.cpu().numpy(), np.arange(n + 2))
    got = np.stack([p.x.cpu().numpy(), p.y.cpu().numpy(), p.z.cpu().numpy()], axis=1)
    orc = oracle_mod.Oracle((4, 2, 2), (64, 32, 32), HBAR, DT, prec=32)
    want = np.zeros((slots, 3), np.float32)
    orc.add_particles(want, 2, n, noz["cen"], noz["rad"], seed=4, counter=7, mode=oracle_mod.EMIT_RING_PLANE)
    assert np.abs(got[2:n + 2] - want[2:n + 2]).max() < 2e-6
    assert (got[2:n + 2, 0] == np.float32(noz["cen"][0])).all()
    r = np.hypot(got[2:n + 2, 1] - noz["cen"][1], got[2:n + 2, 2] - noz["cen"][2])
    assert np.abs(r - 0.9 * noz["rad"]).max() < 1e-5
    with pytest.raises(Exception):
        mp.append(p, np.zeros(slots), np.zeros(slots), np.zeros(slots))


def test_driver_loop_matches_oracle(mp, cfgs):
    """The MatlabPort driver (examples/matlabport/simple.jl:20-124) on the
    64x32x32 jet through the front-end, against oracle.matlabport.driver_step
    fed with the same births."""
    L, dims = (4, 2, 2), (64, 32, 32)
    noz = cfgs.JET_NOZZLE
    vjet = np.array([1.0, 0.0, 0.0])
    kvec = vjet / HBAR
    omega = float(np.sum(vjet ** 2) / (2 * HBAR))
    obj = mp.ISF(L, dims, HBAR, DT)
    oo = orc_mp.MatlabISF(L, dims, HBAR, DT)
    isjet = orc_mp.is_jet(oo, noz["cen"], noz["len"], noz["rad"])
    assert np.array_equal(mp.is_jet(obj, noz["cen"], noz["len"], noz["rad"]).cpu().numpy(), isjet)
    b1, b2 = orc_mp.normalize(np.ones(dims, np.complex128), 0.01 * np.ones(dims, np.complex128))
    for _ in range(10):
        b1, b2 = orc_mp.restrict(oo, b1, b2, isjet, kvec, 0.0)
        b1, b2 = orc_mp.pressure_project(oo, b1, b2)
    a1, a2 = mp.Normalize(torch.ones(dims, dtype=torch.complex128, device="cuda"),
                          0.01 * torch.ones(dims, dtype=torch.complex128, device="cuda"))
    for _ in range(10):
        a1, a2 = mp.restrict(obj, a1, a2, isjet, kvec, 0.0)
        a1, a2 = mp.PressureProject(obj, a1, a2)
    slots = 4000
    p = mp.Particles(np.zeros(slots), np.zeros(slots), np.zeros(slots))
    ox, oy, oz = (np.zeros(slots, np.float32) for _ in range(3))
    olen, oact = 0, np.zeros(0, np.int64)
    for it in range(1, 9):
        t = it * DT
        a1, a2 = mp.SchroedingerFlow(obj, a1, a2)
        a1, a2 = mp.Normalize(a1, a2)
        a1, a2 = mp.PressureProject(obj, a1, a2)
        a1, a2 = mp.restrict(obj, a1, a2, isjet, kvec, omega * t)
        a1, a2 = mp.PressureProject(obj, a1, a2)
        l0 = p.length
        mp.add_ring(p, 200, noz["cen"], noz["rad"], seed=0, counter=it)
        births = [v[l0:l0 + 200].cpu().numpy() for v in (p.x, p.y, p.z)]
        mp.remove_dead(p, obj)
        vx, vy, vz = mp.VelocityOneForm(obj, a1, a2, obj.hbar)
        vx, vy, vz = mp.StaggeredSharp(obj, vx, vy, vz)
        mp.StaggeredAdvect(p, obj, vx, vy, vz, obj.dt)
        b1, b2, olen, oact = orc_mp.driver_step(oo, b1, b2, isjet, kvec, omega * t, ox, oy, oz, olen, oact, births)
    assert rel(a1.cpu().numpy(), b1) < 1e-4 and rel(a2.cpu().numpy(), b2) < 1e-4
    assert p.length == olen == 1600
    assert np.array_equal(p.active.cpu().numpy(), oact)
    got = np.stack([p.x.cpu().numpy(), p.y.cpu().numpy(), p.z.cpu().numpy()])[:, oact]
    want = np.stack([ox, oy, oz])[:, oact]
    assert (np.abs(got - want).max(axis=0) / min(L) < 1e-4).mean() > 0.99
