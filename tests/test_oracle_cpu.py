"""Pins of the CPU oracle (no GPU): numpy.fft, the golden fixtures written by
the independent MatlabPort restatement, and analytic known answers."""
import os

import numpy as np
import pytest

import matlabport as mp
from helpers import philox4x32_10_py, rel, smooth_field, smooth_psi

HBAR = float(np.float32(0.1))
DT = float(np.float32(1 / 48))
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "isf_16x8x8.npz")


@pytest.mark.parametrize("dims", [(16, 8, 8), (12, 24, 48), (64, 32, 32), (96, 48, 48), (32, 32, 32),
                                  (80, 40, 40), (100, 50, 50), (56, 20, 40)])
@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 2e-6)])
def test_fft_matches_numpy(oracle_mod, dims, prec, tol):
    o = oracle_mod.Oracle((1, 1, 1), dims, HBAR, DT, prec=prec)
    rng = np.random.default_rng(0)
    a = rng.normal(size=dims[::-1]) + 1j * rng.normal(size=dims[::-1])
    A = o.fft3(a, -1)
    assert rel(A, np.fft.fftn(a)) < tol
    assert rel(o.fft3(A, +1), a) < tol


def test_mask_and_fac_tables(oracle_mod):
    L, dims = (4, 2, 2), (16, 8, 12)
    o = oracle_mod.Oracle(L, dims, HBAR, DT)
    m = mp.MatlabISF(L, dims, HBAR, DT)
    # parallel.jl stores fftshift(mask); MatlabPort shifts the spectrum instead
    ref = np.transpose(np.fft.ifftshift(m.mask), (2, 1, 0))
    assert np.abs(o.mask() - ref).max() < 1e-14
    fac = o.fac()
    assert fac[0, 0, 0] == 0
    kx = np.arange(dims[0])
    ky = np.arange(dims[1])
    kz = np.arange(dims[2])
    Z, Y, X = np.meshgrid(kz, ky, kx, indexing="ij")
    d = [Lk / nk for Lk, nk in zip(L, dims)]
    den = (np.sin(np.pi * X / dims[0]) / d[0]) ** 2 + (np.sin(np.pi * Y / dims[1]) / d[1]) ** 2 + \
        (np.sin(np.pi * Z / dims[2]) / d[2]) ** 2
    den[0, 0, 0] = 1
    ref = -0.25 / den
    ref[0, 0, 0] = 0
    assert np.abs(fac.real - ref).max() < 1e-14 and np.abs(fac.imag).max() == 0


class TestGolden:
    """Oracle (parallel.jl formulation, C++) == MatlabPort restatement (numpy)."""

    @pytest.fixture(scope="class")
    @classmethod
    def g(cls):
        return dict(np.load(GOLDEN))

    @pytest.fixture(scope="class")
    @classmethod
    def o(cls, oracle_mod):
        return oracle_mod.Oracle((4, 2, 2), (16, 8, 8), HBAR, DT)

    def test_schroedinger_flow(self, g, o):
        assert np.abs(o.schroedinger_flow(g["psi_in"].copy()) - g["schroedinger_flow"]).max() < 1e-13

    def test_normalize(self, g, o):
        assert np.abs(o.normalize(1.3 * g["psi_in"]) - g["normalize"]).max() < 1e-14

    def test_one_form_div_poisson(self, g, o):
        assert np.abs(o.velocity_one_form(g["psi_in"], HBAR) - g["one_form_hbar"]).max() < 1e-14
        assert np.abs(o.velocity_one_form(g["psi_in"], 1.0) - g["one_form_hbar1"]).max() < 1e-14
        assert np.abs(o.div() - g["div"]).max() < 1e-11
        assert np.abs(o.poisson_solve() - g["poisson_q"]).max() < 1e-13

    def test_pressure_project(self, g, o):
        assert np.abs(o.pressure_project(g["psi_in"].copy()) - g["pressure_project"]).max() < 1e-13

    def test_isjet_and_restrict(self, g, o):
        cen = tuple(float(np.float32(v)) for v in (2 - 1.7, 1 - 0.034, 1 + 0.066))
        assert np.array_equal(o.isjet(cen, 0.5, 0.5), g["isjet"])
        omega_t = float(np.float32(5.0 * DT))
        psi = o.restrict_velocity(g["psi_in"].copy(), (10.0, 0, 0), omega_t, cen, 0.5, 0.5, phase_mode=1)
        # positions: FP64 here, Float32 in the numpy restatement's grid -> equal on this exact grid
        assert np.abs(psi - g["restrict_dot"]).max() < 1e-12

    def test_jet_step(self, g, o, oracle_mod):
        cen = tuple(float(np.float32(v)) for v in (2 - 1.7, 1 - 0.034, 1 + 0.066))
        psi = g["psi_in"].copy()
        parts = g["parts_in"].copy()
        jet = dict(kvec=(10.0, 0, 0), omega_t=float(np.float32(5.0 * DT)), cen=cen, len=0.5, rad=0.5,
                   emit_count=0, phase_mode=oracle_mod.PHASE_DOT)
        # the MatlabPort driver has no normalize between its projections -> compare a step without it:
        # run the same sequence by hand
        o.schroedinger_flow(psi)
        o.normalize(psi)
        o.pressure_project(psi)
        o.restrict_velocity(psi, jet["kvec"], jet["omega_t"], cen, 0.5, 0.5, phase_mode=1)
        o.pressure_project(psi)
        o.velocity_one_form(psi, HBAR)
        o.staggered_sharp()
        o.staggered_advect(parts)
        assert np.abs(psi - g["jet_step_psi"]).max() < 1e-12
        assert np.abs(parts - g["jet_step_parts"]).max() < 1e-12


def test_step_entry_matches_operator_sequence(oracle_mod):
    """orc_step == the simloop body assembled from single operators."""
    L, dims = (4, 2, 2), (32, 16, 16)
    cen = tuple(float(np.float32(v)) for v in (2 - 1.7, 1 - 0.034, 1 + 0.066))
    a = oracle_mod.Oracle(L, dims, HBAR, DT)
    b = oracle_mod.Oracle(L, dims, HBAR, DT)
    psi = smooth_psi(dims, seed=3)
    pa = np.full((3000, 3), -1.0)
    pb = pa.copy()
    jet = dict(kvec=(10.0, 0, 0), omega_t=0.1, cen=cen, len=0.5, rad=0.5, emit_start=100, emit_count=1000, seed=5,
               counter=2, emit_mode=oracle_mod.EMIT_RING, phase_mode=oracle_mod.PHASE_REFERENCE_SUM)
    x = psi.copy()
    a.step(x, pa, jet)
    y = psi.copy()
    b.schroedinger_flow(y)
    b.normalize(y)
    b.pressure_project(y)
    b.add_particles(pb, 100, 1000, cen, 0.5, seed=5, counter=2, mode=oracle_mod.EMIT_RING)
    b.restrict_velocity(y, jet["kvec"], 0.1, cen, 0.5, 0.5, phase_mode=oracle_mod.PHASE_REFERENCE_SUM)
    b.pressure_project(y)
    b.velocity_one_form(y, HBAR)
    b.staggered_sharp()
    b.staggered_advect(pb)
    assert np.array_equal(x, y) and np.array_equal(pa, pb)


def test_matlabport_advection_cross_check(oracle_mod):
    L, dims = (3, 2, 2), (48, 32, 32)
    o = oracle_mod.Oracle(L, dims, HBAR, DT)
    m = mp.MatlabISF(L, dims, HBAR, DT)
    rng = np.random.default_rng(5)
    vel = np.stack([smooth_field(dims, rng) for _ in range(3)], axis=-1)
    o.set_velocity(vel)
    parts = rng.uniform(0.1, 0.9, (4000, 3)) * np.asarray(L, np.float64)
    po = o.staggered_advect(parts.copy())
    vx, vy, vz = (np.transpose(vel[..., a], (2, 1, 0)) for a in range(3))
    nx, ny, nz = mp.staggered_advect(parts[:, 0], parts[:, 1], parts[:, 2], m, vx, vy, vz, m.dt)
    assert np.abs(po - np.stack([nx, ny, nz], 1)).max() < 1e-12


# ---- analytic known answers -------------------------------------------------

def test_plane_wave_gets_mask_phase(oracle_mod):
    L, dims = (4, 2, 2), (32, 16, 16)
    o = oracle_mod.Oracle(L, dims, HBAR, DT)
    k = (3, -2, 1)
    nx, ny, nz = dims
    Z, Y, X = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    ph = 2 * np.pi * (k[0] * X / nx + k[1] * Y / ny + k[2] * Z / nz)
    psi = np.stack([np.cos(ph), np.sin(ph), 0 * ph, 0 * ph], -1)
    out = o.schroedinger_flow(psi.copy())
    kk = sum((ki / Li) ** 2 for ki, Li in zip(k, L))
    th = -4 * np.pi ** 2 * HBAR * kk * DT / 2
    expect = np.exp(1j * (ph + th))
    assert np.abs(out[..., 0] + 1j * out[..., 1] - expect).max() < 1e-12


def test_constant_psi_is_fixed_point(oracle_mod):
    L, dims = (4, 2, 2), (16, 8, 8)
    o = oracle_mod.Oracle(L, dims, HBAR, DT)
    psi = o.new_psi(1.0, 0.01)
    o.normalize(psi)
    ref = psi.copy()
    o.pressure_project(psi)
    o.schroedinger_flow(psi)
    assert np.abs(psi - ref).max() < 1e-13


def test_projection_makes_one_form_divergence_free(oracle_mod):
    L, dims = (4, 2, 2), (32, 16, 16)
    o = oracle_mod.Oracle(L, dims, HBAR, DT)
    psi = smooth_psi(dims, seed=8)
    o.velocity_one_form(psi, 1.0)
    before = np.abs(o.div()).max()
    o.pressure_project(psi)
    o.velocity_one_form(psi, 1.0)
    after = np.abs(o.div()).max()
    assert before > 1.0 and after < 1e-9 * before


def test_poisson_inverts_discrete_laplacian(oracle_mod):
    L, dims = (4, 2, 2), (32, 16, 16)
    o = oracle_mod.Oracle(L, dims, HBAR, DT)
    f = smooth_field(dims, np.random.default_rng(9), modes=6)
    f -= f.mean()
    o.set_f(f)
    q = o.poisson_solve().real
    d = [Lk / nk for Lk, nk in zip(L, dims)]
    lap = sum((np.roll(q, -1, ax) - 2 * q + np.roll(q, 1, ax)) / d[2 - ax] ** 2 for ax in range(3))
    assert np.abs(lap - f).max() < 1e-10 * np.abs(f).max()


def test_constant_velocity_advection_is_exact(oracle_mod):
    L, dims = (4, 2, 2), (32, 16, 16)
    o = oracle_mod.Oracle(L, dims, HBAR, DT)
    u = np.array([0.3, -0.2, 0.1])
    o.set_velocity(np.broadcast_to(u, dims[::-1] + (3,)).copy())
    rng = np.random.default_rng(10)
    p = rng.uniform(0.2, 0.8, (1000, 3)) * np.asarray(L, np.float64)
    p[:5] = -1.0
    p[5:10, 2] = 2.5  # outside the open box
    out = o.staggered_advect(p.copy())
    assert np.abs(out[10:] - (p[10:] + DT * u)).max() < 1e-14
    assert (out[:10] == -1).all()


def test_fp32_restatement_tracks_fp64(oracle_mod):
    L, dims = (4, 2, 2), (32, 16, 16)
    a = oracle_mod.Oracle(L, dims, HBAR, DT, prec=64)
    b = oracle_mod.Oracle(L, dims, HBAR, DT, prec=32)
    psi = smooth_psi(dims, seed=11)
    x = psi.copy()
    y = psi.astype(np.float32)
    for _ in range(5):
        a.step(x, None)
        b.step(y, None)
    assert rel(y, x) < 1e-5


def test_philox_matches_independent_python(oracle_mod):
    for ctr, key in [((0, 0, 0, 0), (0, 0)), ((1, 2, 3, 4), (5, 6)), ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2),
                     ((123456, 7, 0, 0x15F0015F), (42, 0))]:
        assert oracle_mod.philox(ctr, key) == philox4x32_10_py(ctr, key)


def test_emission_modes_geometry(oracle_mod):
    L, dims = (4, 2, 2), (32, 16, 16)
    o = oracle_mod.Oracle(L, dims, HBAR, DT)
    cen = (0.3, 0.966, 1.066)
    for mode in (0, 1, 2, 3):
        p = np.full((2000, 3), -1.0)
        o.add_particles(p, 0, 2000, cen, 0.5, seed=1, counter=0, mode=mode, length=0.5)
        r = np.hypot(p[:, 1] - cen[1], p[:, 2] - cen[2])
        if mode == 0:   # ring of radius 0.9 r, +-0.05 jitter (particles.jl:86-90)
            assert np.abs(p[:, 0] - (cen[0] - 0.1)).max() <= 0.05 + 1e-9
            assert (np.abs(r - 0.45) <= 0.05 * np.sqrt(2) + 1e-9).all()
        elif mode == 1:
            assert (p[:, 0] == np.float64(np.float32(cen[0]))).all() and (r <= 0.5 + 1e-9).all()
        elif mode == 3:   # MatlabPort driver ring: 0.9 r in the plane x = cen.x (simple.jl:112-115)
            assert (p[:, 0] == np.float64(np.float32(cen[0]))).all() and np.abs(r - 0.45).max() < 1e-6
        else:
            assert (np.abs(p[:, 0] - cen[0]) <= 0.25 + 1e-6).all() and (r <= 0.5 + 1e-9).all()


def test_matlabport_driver_step_particle_semantics():
    """oracle.matlabport.driver_step: psi as jet_step; births appended and
    active; slots outside the box leave the active list and are not moved;
    the others move by StaggeredAdvect."""
    L, dims = (4, 2, 2), (32, 16, 16)
    oo = mp.MatlabISF(L, dims, HBAR, DT)
    isjet = mp.is_jet(oo, (0.3, 0.966, 1.066), 0.5, 0.5)
    p1, p2 = mp.from_aos(smooth_psi(dims, seed=2))
    x, y, z = (np.full(100, 1.0, np.float32) for _ in range(3))
    x[1] = -0.5                                     # outside: dropped from the list, kept as is
    births = (np.float32([0.3, 0.3]), np.float32([0.9, 1.0]), np.float32([1.0, 1.1]))
    a1, a2, n, act = mp.driver_step(oo, p1, p2, isjet, (10, 0, 0), 0.1, x, y, z, 3, np.arange(3), births)
    b1, b2, _ = mp.jet_step(oo, p1, p2, isjet, (10, 0, 0), 0.1)
    assert rel(a1, b1) == 0 and rel(a2, b2) == 0
    assert n == 5 and list(act) == [0, 2, 3, 4]
    assert x[1] == -0.5 and (x[[0, 2]] != 1.0).all()
