"""GPU parity of each ISF operator (libisf through the C ABI) against the FP64
oracle on seeded inputs.  Tolerances: relative L2 error 1e-5 for single
operators (FP32 arithmetic vs FP64), bit-exact for the integer isjet mask."""
import numpy as np
import pytest
import torch

from helpers import rel, smooth_field, smooth_psi

pytestmark = pytest.mark.gpu

GRIDS = [
    ((4, 2, 2), (16, 8, 8)),
    ((4, 2, 2), (64, 32, 32)),
    ((3, 2, 2), (48, 32, 32)),
    ((6, 3, 3), (96, 48, 48)),
    ((2, 1, 1), (32, 12, 24)),
    # lengths with factors 5 and 7; rows and x extents that are not whole tiles
    ((4, 2, 2), (80, 40, 40)),
    ((4, 2, 2), (100, 50, 50)),
    ((2, 1, 1), (56, 20, 40)),
    # the 128 x 128 plane solver (radix 16 x 8)
    ((1, 4, 4), (32, 128, 128)),
]
HBAR = float(np.float32(0.1))
DT = float(np.float32(1 / 48))


def cuda(a, dtype=torch.float32):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def host(t):
    return t.detach().double().cpu().numpy()


@pytest.mark.parametrize("dims", [(16, 8, 8), (32, 12, 24), (48, 32, 32), (96, 48, 48), (256, 128, 128),
                                  (512, 16, 8), (384, 8, 16), (192, 64, 8), (80, 40, 40), (100, 50, 50),
                                  (56, 112, 20), (200, 50, 160),
                                  # x rows whose pencils share a warp (16 and 8 lanes each), and a
                                  # row of 8 whose pencils are single lanes
                                  (128, 16, 8), (64, 8, 16), (8, 16, 32)])
def test_fft3_matches_numpy(isfpkg, dims):
    isf = isfpkg.ISF((1, 1, 1), dims, HBAR, DT)
    rng = np.random.default_rng(1)
    nx, ny, nz = dims
    a = rng.normal(size=(nz, ny, nx)) + 1j * rng.normal(size=(nz, ny, nx))
    t = torch.tensor(a.astype(np.complex64), device="cuda")
    isf.fft3(t, -1)
    isf.sync()
    ref = np.fft.fftn(a)
    assert rel(t.cpu().numpy(), ref) < 2e-6
    isf.fft3(t, +1)
    isf.sync()
    assert rel(t.cpu().numpy(), a) < 2e-6


@pytest.mark.parametrize("L,dims", GRIDS)
def test_schroedinger_flow_and_normalize(isfpkg, oracle_mod, L, dims):
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    psi64 = smooth_psi(dims, seed=2)
    psi = cuda(psi64)
    isfpkg.schroedinger_flow(isf, psi)
    isf.sync()
    orc.schroedinger_flow(psi64)
    assert rel(host(psi), psi64) < 1e-5
    # perturb the norm, then normalize
    psi64 *= 1.0 + 0.3 * np.cos(np.arange(psi64.shape[2]))[None, None, :, None]
    psi = cuda(psi64)
    isfpkg.normalize_psi(isf, psi)
    isf.sync()
    orc.normalize(psi64)
    assert rel(host(psi), psi64) < 1e-6


@pytest.mark.parametrize("L,dims", GRIDS)
@pytest.mark.parametrize("hbar", [1.0, HBAR])
def test_velocity_one_form_and_div(isfpkg, oracle_mod, L, dims, hbar):
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    psi64 = smooth_psi(dims, seed=3)
    psi = cuda(psi64)
    isfpkg.velocity_one_form(isf, psi, hbar)
    v = isf.velocity
    vo = orc.velocity_one_form(psi64, hbar)
    assert np.abs(host(v) - vo).max() < 2e-6 * max(1.0, hbar)
    f = isf.div()
    isf.sync()
    fo = orc.div()
    assert rel(host(f), fo) < 1e-4  # difference of nearby angles / d^2: cancellation
    isfpkg.staggered_sharp(isf)
    orc.staggered_sharp()
    assert rel(host(isf.velocity), orc.velocity()) < 1e-6


def test_one_form_angles_all_quadrants(isfpkg, oracle_mod):
    """Random (non-smooth) psi: one-form angles cover (-pi, pi]; the kernel's
    atan2 stays within 2.5e-7 rad of the FP64 oracle (compared modulo 2 pi,
    so a +-pi branch flip of a value within rounding of the cut is not an error)."""
    L, dims = (4, 2, 2), (64, 32, 32)
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    rng = np.random.default_rng(12)
    ph = rng.uniform(-np.pi, np.pi, dims[::-1] + (2,))
    amp = rng.uniform(0.2, 1.0, dims[::-1] + (2,))
    psi64 = np.stack([amp[..., 0] * np.cos(ph[..., 0]), amp[..., 0] * np.sin(ph[..., 0]),
                      amp[..., 1] * np.cos(ph[..., 1]), amp[..., 1] * np.sin(ph[..., 1])], -1)
    psi64 = psi64.astype(np.float32).astype(np.float64)
    isfpkg.velocity_one_form(isf, cuda(psi64), 1.0)
    v = host(isf.velocity)
    vo = orc.velocity_one_form(psi64, 1.0)
    d = np.abs((v - vo + np.pi) % (2 * np.pi) - np.pi)
    # |z| of z = conj(a1) b1 + conj(a2) b2: FP32 rounding of re / im moves the
    # angle by ~1e-7 / |z| on top of the atan2 error itself
    zabs = np.zeros_like(vo)
    c = psi64[..., 0] + 1j * psi64[..., 1], psi64[..., 2] + 1j * psi64[..., 3]
    for ax, npax in enumerate((2, 1, 0)):
        zabs[..., ax] = np.abs(np.conj(c[0]) * np.roll(c[0], -1, npax) + np.conj(c[1]) * np.roll(c[1], -1, npax))
    assert np.abs(vo).max() > 3.1
    assert (d <= 3e-7 + 3e-7 / zabs).all(), (d * zabs).max()


@pytest.mark.parametrize("L,dims", GRIDS)
def test_poisson_solve(isfpkg, oracle_mod, L, dims):
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    rng = np.random.default_rng(4)
    f = smooth_field(dims, rng, modes=6) + 0.1 * rng.normal(size=dims[::-1])
    f -= f.mean()
    q = isf.poisson_solve(cuda(f))
    isf.sync()
    orc.set_f(f)
    qo = orc.poisson_solve()
    assert np.abs(qo.imag).max() < 1e-10
    assert rel(host(q), qo.real) < 1e-5


@pytest.mark.parametrize("L,dims", GRIDS)
def test_pressure_project(isfpkg, oracle_mod, L, dims):
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    psi64 = smooth_psi(dims, seed=5)
    psi = cuda(psi64)
    isfpkg.pressure_project(isf, psi)
    isf.sync()
    orc.pressure_project(psi64)
    assert rel(host(psi), psi64) < 1e-5


@pytest.mark.parametrize("L,dims", [((4, 2, 2), (64, 32, 32)), ((4, 2, 2), (128, 64, 64)), ((4, 2, 2), (16, 8, 8))])
def test_isjet_bit_exact(isfpkg, oracle_mod, cfgs, L, dims):
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    noz = cfgs.JET_NOZZLE
    m = isfpkg.isjet(isf, noz["cen"], noz["len"], noz["rad"])
    isf.sync()
    mo = orc.isjet(noz["cen"], noz["len"], noz["rad"])
    assert m.sum().item() > 0
    assert np.array_equal(m.cpu().numpy(), mo)


@pytest.mark.parametrize("phase_mode", [0, 1])
@pytest.mark.parametrize("use_mask", [False, True])
def test_restrict_velocity(isfpkg, oracle_mod, cfgs, phase_mode, use_mask):
    L, dims = (4, 2, 2), (64, 32, 32)
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    noz = cfgs.JET_NOZZLE
    kvec, omega = cfgs.jet_omega()
    psi64 = smooth_psi(dims, seed=6)
    psi = cuda(psi64)
    mask = isfpkg.isjet(isf, noz["cen"], noz["len"], noz["rad"]) if use_mask else None
    isfpkg.restrict_velocity(isf, psi, kvec, mask, omega * 0.5, nozzle=(noz["cen"], noz["len"], noz["rad"]),
                             phase_mode=phase_mode)
    isf.sync()
    orc.restrict_velocity(psi64, kvec, omega * 0.5, noz["cen"], noz["len"], noz["rad"], phase_mode=phase_mode)
    assert rel(host(psi), psi64) < 2e-6


@pytest.mark.parametrize("mode", [0, 1, 2, 3])
def test_add_particles(isfpkg, oracle_mod, cfgs, mode):
    L, dims = (4, 2, 2), (64, 32, 32)
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    noz = cfgs.JET_NOZZLE
    P = 5000
    parts = torch.full((P, 3), -1.0, device="cuda")
    isfpkg.add_particles(isf, parts, range(4000, 4000 + 3000), noz["cen"], noz["rad"], seed=11, counter=3,
                         mode=mode, nozzle_len=noz["len"])
    isf.sync()
    for prec, tol in ((32, 2e-6), (64, 2e-6)):
        orc = oracle_mod.Oracle(L, dims, HBAR, DT, prec=prec)
        po = np.full((P, 3), -1.0, dtype=orc.dtype)
        orc.add_particles(po, 4000, 3000, noz["cen"], noz["rad"], seed=11, counter=3, mode=mode,
                          length=noz["len"])
        assert np.abs(host(parts) - po).max() < tol
    # wrapped slots
    assert (host(parts)[:2000] != -1).all() and (host(parts)[2000:4000] == -1).all()


@pytest.mark.parametrize("L,dims", [((4, 2, 2), (64, 32, 32)), ((3, 2, 2), (48, 32, 32))])
def test_staggered_advect(isfpkg, oracle_mod, L, dims):
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    rng = np.random.default_rng(7)
    vel = np.stack([smooth_field(dims, rng, scale=0.8) + 0.5 for _ in range(3)], axis=-1)
    P = 20000
    parts64 = rng.uniform(0, 1, (P, 3)) * np.asarray(L, np.float64)
    parts64[:100] = -1.0              # dead slots
    parts64[100:110, 0] = L[0] + 0.5  # outside the box -> killed
    parts64 = parts64.astype(np.float32).astype(np.float64)
    isf.velocity = cuda(vel)
    orc.set_velocity(vel.astype(np.float32).astype(np.float64))
    parts = cuda(parts64)
    isfpkg.staggered_advect(parts, isf)
    isf.sync()
    assert isf.counters()["check_failures"] == 0  # nonzero only in a -DISF_CHECK build
    po, margin = orc.staggered_advect(parts64.copy(), margin=True)
    err = np.abs(host(parts) - po).max(axis=1) / min(L)
    near_face = margin < 1e-4
    assert (err[~near_face] < 1e-5).all(), err[~near_face].max()
    assert near_face.mean() < 0.01
    assert (host(parts)[:110] == -1).all()


@pytest.mark.parametrize("L,dims", [((4, 2, 2), (64, 32, 32)), ((6, 3, 3), (96, 48, 48))])
def test_step_sequences(isfpkg, oracle_mod, cfgs, L, dims):
    """isf_step (fused) == oracle simloop body for jet and plain steps."""
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    noz = cfgs.JET_NOZZLE
    kvec, omega = cfgs.jet_omega()
    psi64 = cfgs.jet_init_psi(dims)
    for _ in range(3):
        orc.restrict_velocity(psi64, kvec, 0.0, noz["cen"], noz["len"], noz["rad"], phase_mode=1)
        orc.pressure_project(psi64)
    P = 8000
    parts64 = np.full((P, 3), -1.0)
    orc.add_particles(parts64, 0, 2000, noz["cen"], noz["rad"], seed=0, counter=0, mode=1)
    psi = cuda(psi64)
    parts = cuda(parts64)
    margin_min = np.full(P, 1e30)
    for it in range(1, 6):
        jet = dict(kvec=kvec, omega_t=float(np.float32(omega) * np.float32(it * np.float32(DT))), cen=noz["cen"],
                   len=noz["len"], rad=noz["rad"], emit_start=(it * 1000) % P, emit_count=1000, seed=0, counter=it,
                   emit_mode=1, phase_mode=1)
        isfpkg.step(isf, psi, parts, jet if it % 2 else None)
        m = np.zeros(P)
        orc.step(psi64, parts64, jet if it % 2 else None, margin=m)
        margin_min = np.minimum(margin_min, m)
    isf.sync()
    assert rel(host(psi), psi64) < 2e-5
    err = np.abs(host(parts) - parts64).max(axis=1) / min(L)
    ok = margin_min > 1e-4
    assert (err[ok] < 1e-4).all(), err[ok].max()


@pytest.mark.parametrize("dims", [(64, 32, 128), (32, 16, 64), (16, 8, 256), (24, 8, 96), (40, 12, 192)])
def test_schroedinger_z_pass_tma_matches_register_staging(isfpkg, dims):
    """The z pass of schroedinger_flow! with its pencils copied into shared
    memory by the TMA (ISF_FLAG_TMA_Z_PASS: cp.async.bulk.tensor,
    double-buffered, bounded mbarrier waits) against the same pass staged
    through registers
    (the default): the arithmetic of a pencil is the same, so psi is bitwise
    equal, and no wait ran out."""
    psi0 = smooth_psi(dims, 12)
    out = []
    for flags in (isfpkg.FLAG_TMA_Z_PASS, 0):
        isf = isfpkg.ISF((1, 1, 1), dims, HBAR, DT, flags=flags)
        psi = cuda(psi0)
        for _ in range(2):
            isfpkg.schroedinger_flow(isf, psi)
        isf.sync()
        assert isf.counters()["wait_timeouts"] == 0
        out.append(psi.cpu().numpy())
        isf.close()
    assert np.array_equal(out[0].view(np.uint32), out[1].view(np.uint32))


def test_tma_z_pass_wait_times_out_and_the_gpu_keeps_answering(isfpkg):
    """ISF_FLAG_TMA_Z_STALL makes every CTA of the TMA z pass wait, after its
    first tile has arrived, on a flag that nothing sets: the bounded wait runs
    out, each CTA counts it in counter 14, waits for its copy still in flight
    and returns.  No fault and no trap: the same handle and a fresh one then
    run the pass normally and match the register-staged pass."""
    dims = (32, 16, 64)
    psi0 = smooth_psi(dims, 12)
    isf = isfpkg.ISF((1, 1, 1), dims, HBAR, DT, flags=isfpkg.FLAG_TMA_Z_PASS | isfpkg.FLAG_TMA_Z_STALL)
    psi = cuda(psi0)
    isfpkg.schroedinger_flow(isf, psi)
    isf.sync()
    c = isf.counters(reset=True)
    assert c["wait_timeouts"] > 0, c
    isf.close()
    out = []
    for flags in (isfpkg.FLAG_TMA_Z_PASS, 0):
        h = isfpkg.ISF((1, 1, 1), dims, HBAR, DT, flags=flags)
        p = cuda(psi0)
        isfpkg.schroedinger_flow(h, p)
        h.sync()
        assert h.counters()["wait_timeouts"] == 0
        out.append(p.cpu().numpy())
        h.close()
    assert np.array_equal(out[0].view(np.uint32), out[1].view(np.uint32))


def test_invalid_arguments(isfpkg):
    with pytest.raises(isfpkg.ISFError):
        isfpkg.ISF((1, 1, 1), (22, 8, 8), HBAR, DT)  # 22 = 2 x 11: no radix plan
    with pytest.raises(isfpkg.ISFError):
        isfpkg.ISF((1, 1, 1), (16, 8, 28), HBAR, DT)  # 28 is not one of the plans' lengths
    isf = isfpkg.ISF((1, 1, 1), (16, 8, 8), HBAR, DT)
    bad = torch.zeros((8, 8, 8, 4), device="cuda")
    with pytest.raises(isfpkg.ISFError):
        isfpkg.schroedinger_flow(isf, bad)
    parts = torch.zeros((10, 3), device="cuda")
    with pytest.raises(isfpkg.ISFError):
        isfpkg.add_particles(isf, parts, range(0, 11), (0, 0, 0), 0.1)


def test_counters_async_match(isfpkg):
    """isf_counters_async queues the same counters isf_counters reads, behind
    the queued work, and resets them when asked."""
    L, dims = (4, 2, 2), (64, 32, 32)
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    rng = np.random.default_rng(8)
    isf.velocity = cuda(np.stack([smooth_field(dims, rng, scale=0.5) for _ in range(3)], axis=-1))
    parts = cuda(rng.uniform(0.1, 0.9, (5000, 3)) * np.asarray(L))
    parts[:700] = -1.0
    out = torch.zeros((2, 2), dtype=torch.int64).pin_memory()
    isfpkg.staggered_advect(parts, isf)
    isf.counters_async(out[0], reset=True)
    isfpkg.staggered_advect(parts, isf)
    isf.counters_async(out[1], reset=False)
    isf.sync()
    assert int(out[0, 1]) == 4300 and int(out[1, 1]) <= 4300
    c = isf.counters(reset=True)
    assert c["live"] == int(out[1, 1]) and c["clamp_events"] == int(out[1, 0])


@pytest.mark.parametrize("L,dims", [((4, 2, 2), (64, 32, 32)), ((5, 2, 2), (48, 32, 32))])
def test_staggered_advect_normalized_weights(isfpkg, oracle_mod, L, dims):
    """ISF_FLAG_NORMALIZED_WEIGHTS: the staggered weights divided by d, against
    the oracle with the same switch (power-of-two and general d)."""
    isf = isfpkg.ISF(L, dims, HBAR, DT, flags=isfpkg.FLAG_NORMALIZED_WEIGHTS)
    orc = oracle_mod.Oracle(L, dims, HBAR, DT, normalized_weights=True)
    rng = np.random.default_rng(17)
    vel = np.stack([smooth_field(dims, rng, scale=0.8) + 0.5 for _ in range(3)], axis=-1)
    P = 20000
    parts64 = (rng.uniform(0, 1, (P, 3)) * np.asarray(L, np.float64)).astype(np.float32).astype(np.float64)
    isf.velocity = cuda(vel)
    orc.set_velocity(vel.astype(np.float32).astype(np.float64))
    parts = cuda(parts64)
    isfpkg.staggered_advect(parts, isf)
    po, margin = orc.staggered_advect(parts64.copy(), margin=True)
    err = np.abs(host(parts) - po).max(axis=1) / min(L)
    near_face = margin < 1e-4
    assert (err[~near_face] < 1e-5).all(), err[~near_face].max()
    # the weights matter: the reference's unnormalised weights give other positions
    ref = oracle_mod.Oracle(L, dims, HBAR, DT)
    ref.set_velocity(vel.astype(np.float32).astype(np.float64))
    assert np.abs(ref.staggered_advect(parts64.copy()) - po).max() > 1e-3


def test_step_nan_check(isfpkg):
    """ISF_FLAG_CHECK_NAN: a non-finite psi cell makes isf_step fail with
    ISF_ERR_NAN; a finite state steps normally."""
    L, dims = (4, 2, 2), (32, 16, 16)
    isf = isfpkg.ISF(L, dims, HBAR, DT, flags=isfpkg.FLAG_CHECK_NAN)
    psi = cuda(smooth_psi(dims, 3))
    isfpkg.step(isf, psi, None, None)
    psi[3, 2, 1, 0] = float("nan")
    with pytest.raises(isfpkg.ISFError, match="not finite") as e:
        isfpkg.step(isf, psi, None, None)
    assert e.value.code == 4
    with pytest.raises(isfpkg.ISFError, match="unknown flags"):
        isfpkg.ISF(L, dims, HBAR, DT, flags=64)


def test_particle_stream_matches_single_stream(isfpkg, cfgs):
    """A handle that owns its stream runs the particle work of isf_step on a
    second stream, overlapped with the next step's psi passes, and alternates
    two velocity plane sets; a handle on a caller stream runs everything in
    order on that stream.  Both give the same bits: psi, particles, velocity and
    the per-step counters read with isf_counters_async."""
    L, dims = (4, 2, 2), (64, 32, 32)
    noz = cfgs.JET_NOZZLE
    kvec, omega = cfgs.jet_omega()
    rng = np.random.default_rng(21)
    psi0 = cuda(cfgs.jet_init_psi(dims))
    P = 30000
    p0 = rng.uniform(0, 1, (P, 3)) * np.asarray(L)
    p0[:10000] = -1.0  # slots the jet fills
    parts0 = cuda(p0)
    caller = torch.cuda.Stream()
    two = isfpkg.ISF(L, dims, HBAR, DT)
    one = isfpkg.ISF(L, dims, HBAR, DT, stream=caller)
    steps = 12
    res = {}
    out = {}
    torch.cuda.synchronize()
    for name, isf in (("two", two), ("one", one)):
        psi, parts = psi0.clone(), parts0.clone()
        torch.cuda.synchronize()
        rows = torch.zeros((steps, 2), dtype=torch.int64).pin_memory()
        for it in range(1, steps + 1):
            jet = dict(kvec=kvec, omega_t=float(np.float32(omega) * np.float32(it * np.float32(DT))),
                       cen=noz["cen"], len=noz["len"], rad=noz["rad"], emit_start=(it * 800) % 10000,
                       emit_count=800, seed=5, counter=it, emit_mode=1, phase_mode=1)
            isfpkg.step(isf, psi, parts, jet if it % 3 else None)
            isf.counters_async(rows[it - 1], reset=True)
        if name == "two":
            # work queued on the handle's stream after isf_join sees the advection
            isf.join()
            with torch.cuda.stream(isf.stream):
                snap = parts.clone()
            isf.sync()
            out["snap"] = snap
        else:
            isf.sync()
        res[name] = rows.clone()
        out[name] = (psi, parts, isf.velocity)
    psi_a, parts_a, vel_a = out["two"]
    psi_b, parts_b, vel_b = out["one"]
    assert torch.equal(psi_a, psi_b)
    assert torch.equal(parts_a, parts_b)
    assert torch.equal(out["snap"], parts_b)
    assert torch.equal(vel_a, vel_b)
    assert torch.equal(res["two"], res["one"])
    assert int(res["two"][-1, 1]) > 20000


@pytest.mark.parametrize("phase_mode", [0, 1])
def test_init_jet_matches_loop_and_oracle(isfpkg, oracle_mod, cfgs, phase_mode):
    """isf_init_jet (the jet set-up loop in one call, restriction fused into
    the projection) against the same loop of restrict_velocity + pressure_project
    through the API, and against the FP64 oracle."""
    L, dims = (4, 2, 2), (64, 32, 32)
    noz = cfgs.JET_NOZZLE
    kvec, _ = cfgs.jet_omega()
    isf = isfpkg.ISF(L, dims, HBAR, DT)
    psi0 = cfgs.jet_init_psi(dims)
    a = cuda(psi0)
    isfpkg.init_jet(isf, a, 10, kvec, nozzle=(noz["cen"], noz["len"], noz["rad"]), phase_mode=phase_mode)
    b = cuda(psi0)
    for _ in range(10):
        isfpkg.restrict_velocity(isf, b, kvec, None, 0.0, nozzle=(noz["cen"], noz["len"], noz["rad"]),
                                 phase_mode=phase_mode)
        isfpkg.pressure_project(isf, b)
    isf.sync()
    assert rel(host(a), host(b)) < 1e-6
    orc = oracle_mod.Oracle(L, dims, HBAR, DT)
    psi64 = psi0.copy()
    for _ in range(10):
        orc.restrict_velocity(psi64, kvec, 0.0, noz["cen"], noz["len"], noz["rad"], phase_mode=phase_mode)
        orc.pressure_project(psi64)
    assert rel(host(a), psi64) < 2e-5
    with pytest.raises(Exception):
        isfpkg.init_jet(isf, a, -1, kvec, nozzle=(noz["cen"], noz["len"], noz["rad"]))


def test_step_without_particles_both_stream_kinds(isfpkg, cfgs):
    """isf_step with no particle slots queues no particle work: a handle with
    its own streams and one on a caller stream give the same psi bits, and a
    later call with particles still orders correctly after it."""
    L, dims = (4, 2, 2), (64, 32, 32)
    psi0 = cuda(smooth_psi(dims, seed=4))
    own = isfpkg.ISF(L, dims, HBAR, DT)
    caller = isfpkg.ISF(L, dims, HBAR, DT, stream=torch.cuda.Stream())
    out = []
    for isf in (own, caller):
        psi = psi0.clone()
        torch.cuda.synchronize()
        for _ in range(3):
            isfpkg.step(isf, psi, None, None)
        parts = cuda(np.random.default_rng(2).uniform(0.2, 0.8, (1000, 3)) * np.asarray(L))
        torch.cuda.synchronize()
        isfpkg.step(isf, psi, parts, None)
        isf.sync()
        out.append((psi, parts))
    assert torch.equal(out[0][0], out[1][0])
    assert torch.equal(out[0][1], out[1][1])
