"""Adjoint (isf_adj_*, through the C ABI) against FP64 central differences of
the oracle: for an operator A at input x, a direction u and a cotangent ybar,

    < A^T ybar (GPU, FP32), u >   ==   < ybar, (A(x + h u) - A(x - h u)) / 2h >  (oracle, FP64)

within 1e-3 relative.  Inputs are smooth (neighbour phase steps well below
pi), where the operators are differentiable: the angle's branch cut, the
staggered weights' jumps at cell faces and particle death carry no
derivative, and the steps are small enough to cross none of them."""
import numpy as np
import pytest
import torch

from helpers import smooth_field, smooth_psi

pytestmark = pytest.mark.gpu

L, DIMS = (4, 2, 2), (32, 16, 16)
HBAR, DT = float(np.float32(0.1)), float(np.float32(1 / 48))
NOZZLE = ((1.0, 1.0, 1.0), 0.8, 0.6)


def cuda(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def host(t):
    return t.detach().double().cpu().numpy()


def dot(a, b):
    return float(np.sum(np.asarray(a, np.float64) * np.asarray(b, np.float64)))


def close(adj, fd, scale=0.0, tol=1e-3):
    return abs(adj - fd) <= tol * max(abs(fd), scale)


def fd(f, x, u, h):
    return (f(x + h * u) - f(x - h * u)) / (2 * h)


@pytest.fixture
def setup(isfpkg, oracle_mod):
    isf = isfpkg.ISF(L, DIMS, HBAR, DT)
    orc = oracle_mod.Oracle(L, DIMS, HBAR, DT)
    return isf, orc


def f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


def test_adj_schroedinger_flow_is_the_transpose(isfpkg, setup):
    isf, orc = setup
    rng = np.random.default_rng(1)
    u = rng.normal(size=isf.shape + (4,))
    yb = rng.normal(size=u.shape)
    t = cuda(yb)
    isfpkg.adj_schroedinger_flow(isf, t)
    lhs = dot(host(t), f32(u))
    rhs = dot(f32(yb), orc.schroedinger_flow(f32(u).copy()))   # linear: no finite difference needed
    assert close(lhs, rhs, tol=1e-4), (lhs, rhs)


def test_adj_normalize(isfpkg, setup):
    isf, orc = setup
    rng = np.random.default_rng(2)
    x = f32(smooth_psi(DIMS, 2) * (1.0 + 0.3 * rng.uniform(size=isf.shape + (1,))))
    u = rng.normal(size=x.shape)
    yb = rng.normal(size=x.shape)
    t = cuda(yb)
    isfpkg.adj_normalize_psi(isf, cuda(x), t)
    g = dot(yb, fd(lambda v: orc.normalize(v.copy()), x, u, 1e-6))
    assert close(dot(host(t), u), g), (dot(host(t), u), g)


def test_adj_pressure_project(isfpkg, setup):
    isf, orc = setup
    rng = np.random.default_rng(3)
    x = f32(smooth_psi(DIMS, 3))
    for k in range(2):
        u = rng.normal(size=x.shape)
        yb = rng.normal(size=x.shape)
        t = cuda(yb)
        isfpkg.adj_pressure_project(isf, cuda(x), t)
        g = dot(yb, fd(lambda v: orc.pressure_project(v.copy()), x, u, 1e-6))
        assert close(dot(host(t), u), g), (k, dot(host(t), u), g)


@pytest.mark.parametrize("phase_mode", [0, 1])
def test_adj_restrict_velocity(isfpkg, oracle_mod, setup, phase_mode):
    isf, orc = setup
    rng = np.random.default_rng(4)
    x = f32(smooth_psi(DIMS, 4))
    kvec = tuple(float(np.float32(k)) for k in (10.0, 1.5, -0.7))
    om = float(np.float32(0.7))
    cen, ln, rad = NOZZLE
    u = rng.normal(size=x.shape)
    yb = rng.normal(size=x.shape)
    t = cuda(yb)
    jb = isfpkg.adj_restrict_velocity(isf, cuda(x), t, kvec, om, nozzle=NOZZLE, phase_mode=phase_mode)

    def R(v, k=kvec, w=om):
        return orc.restrict_velocity(v.copy(), k, w, cen, ln, rad, phase_mode=phase_mode)

    assert close(dot(host(t), u), dot(yb, fd(R, x, u, 1e-6)))
    for a in range(3):
        e = np.zeros(3)
        e[a] = 1.0
        g = dot(yb, (R(x, tuple(np.add(kvec, 1e-6 * e))) - R(x, tuple(np.add(kvec, -1e-6 * e)))) / 2e-6)
        assert close(jb[a], g, scale=1e-3 * abs(jb[3]) + 1e-6), (a, jb[a], g)
    g = dot(yb, (R(x, kvec, om + 1e-6) - R(x, kvec, om - 1e-6)) / 2e-6)
    assert close(jb[3], g), (jb[3], g)


def test_adj_velocity_one_form_with_sharp(isfpkg, setup):
    isf, orc = setup
    rng = np.random.default_rng(5)
    x = f32(smooth_psi(DIMS, 5))
    ub = rng.normal(size=isf.shape + (3,))
    u = rng.normal(size=x.shape)
    isfpkg.set_velocity_bar(isf, cuda(ub))
    t = torch.zeros(isf.shape + (4,), dtype=torch.float32, device="cuda")
    isfpkg.adj_velocity_one_form(isf, cuda(x), t, hbar=HBAR, sharp=True)

    def V(v):
        orc.velocity_one_form(v.copy(), HBAR)
        orc.staggered_sharp()
        return orc.velocity()

    g = dot(f32(ub), fd(V, x, u, 1e-6))
    assert close(dot(host(t), u), g), (dot(host(t), u), g)


@pytest.mark.parametrize("norm", [False, True])
@pytest.mark.parametrize("grid", [((4, 2, 2), (32, 16, 16)), ((5, 2, 2), (48, 16, 16))])
def test_adj_staggered_advect(isfpkg, oracle_mod, grid, norm):
    """Power-of-two and general cell sizes, the reference's and normalised
    weights; cotangents of the positions and of the velocity planes."""
    Lg, dims = grid
    isf = isfpkg.ISF(Lg, dims, HBAR, DT, flags=isfpkg.FLAG_NORMALIZED_WEIGHTS if norm else 0)
    orc = oracle_mod.Oracle(Lg, dims, HBAR, DT, normalized_weights=norm)
    rng = np.random.default_rng(6)
    v = np.stack([smooth_field(dims, rng, scale=0.8) for _ in range(3)], axis=-1)
    v = f32(v)
    P = 4096
    p = f32(rng.uniform(0.15, 0.85, (P, 3)) * np.asarray(Lg))
    lam = rng.normal(size=(P, 3))
    isf.velocity = cuda(v)
    lb = cuda(lam)
    isfpkg.adj_staggered_advect(isf, cuda(p), lb)
    vb = host(isfpkg.get_velocity_bar(isf))

    def X(pp, vv=v):
        orc.set_velocity(vv)
        return orc.staggered_advect(pp.copy())

    up = rng.normal(size=p.shape)
    g = dot(lam, fd(X, p, up, 1e-7))
    assert close(dot(host(lb), up), g), (dot(host(lb), up), g)
    uv = rng.normal(size=v.shape)
    g = dot(lam, (X(p, v + 1e-7 * uv) - X(p, v - 1e-7 * uv)) / 2e-7)
    assert close(dot(vb, uv), g), (dot(vb, uv), g)


def test_adj_step_jet_with_emission(isfpkg, setup):
    """One fused jet step (both projections, restriction, emission into part
    of the slots, one-form, RK4) reversed by isf_adj_step."""
    isf, orc = setup
    rng = np.random.default_rng(7)
    x = f32(smooth_psi(DIMS, 7))
    P = 2048
    p = f32(rng.uniform(0.15, 0.85, (P, 3)) * np.asarray(L))
    kvec = tuple(float(np.float32(k)) for k in (6.0, 0.5, 0.0))
    cen, ln, rad = NOZZLE
    jet = dict(kvec=kvec, omega_t=float(np.float32(0.35)), cen=cen, len=ln, rad=rad, emit_start=100, emit_count=64,
               seed=3, counter=1, emit_mode=1, phase_mode=1)
    yb = rng.normal(size=x.shape)
    lam = rng.normal(size=p.shape)
    tb, lb = cuda(yb), cuda(lam)
    jb = isfpkg.adj_step(isf, cuda(x), cuda(p), jet, tb, lb)

    def F(xx, pp, **kw):
        j = dict(jet, **kw)
        a, b = xx.copy(), pp.copy()
        orc.step(a, b, j)
        return dot(yb, a) + dot(lam, b)

    ux, up = rng.normal(size=x.shape), rng.normal(size=p.shape)
    h = 1e-7
    g = (F(x + h * ux, p + h * up) - F(x - h * ux, p - h * up)) / (2 * h)
    a = dot(host(tb), ux) + dot(host(lb), up)
    assert close(a, g), (a, g)
    assert float(lb[100:164].abs().max()) == 0.0      # emitted slots do not depend on their old positions
    for k in range(3):
        e = np.zeros(3)
        e[k] = 1e-6
        g = (F(x, p, kvec=tuple(np.add(kvec, e))) - F(x, p, kvec=tuple(np.add(kvec, -e)))) / 2e-6
        assert close(jb[k], g, scale=1e-2 * abs(jb[3]) + 1e-6), (k, jb[k], g)
    g = (F(x, p, omega_t=jet["omega_t"] + 1e-6) - F(x, p, omega_t=jet["omega_t"] - 1e-6)) / 2e-6
    assert close(jb[3], g), (jb[3], g)


def driver_forward(orc, psi0, p0, tgt, T, init_iters, kvec, omega):
    cen, ln, rad = NOZZLE
    psi = psi0.copy()
    for _ in range(init_iters):
        orc.restrict_velocity(psi, kvec, 0.0, cen, ln, rad, phase_mode=1)
        orc.pressure_project(psi)
    x = p0.copy()
    for n in range(1, T + 1):
        tn = float(np.float32(n) * np.float32(DT))
        orc.step(psi, x, dict(kvec=kvec, omega_t=omega * tn, cen=cen, len=ln, rad=rad, emit_count=0, counter=n,
                              phase_mode=1))
    alive = x[:, 0] >= 0
    return float(((x[alive] - tgt[alive]) ** 2).sum())


# central-difference steps tried in order for one direction of the driver tests
H_LADDER = (1e-7, 1e-8, 1e-9)


def fd_without_crossing(f, ladder=H_LADDER, agree=1e-4):
    """Central difference of t -> f(t) at 0 from the first h of `ladder` at
    which the differences over +-h and +-h/10 agree to `agree` relative.

    The particle loss is piecewise smooth: a particle whose RK sample point
    crosses a cell face (the staggered interpolation jumps there) or a
    one-form angle that crosses its branch cut makes it jump.  A jump at
    distance delta from t = 0 enters the difference over +-h only when
    delta < h, and then as J / 2h, ten times larger at h/10 than at h; so two
    agreeing differences show that +-h crosses none.  Shrinking h moves every
    crossing out of reach, so each direction gets a derivative; the function
    fails (it does not skip) if the ladder runs out."""
    seen = []
    for h in ladder:
        g1 = (f(h) - f(-h)) / (2 * h)
        g2 = (f(0.1 * h) - f(-0.1 * h)) / (0.2 * h)
        seen.append((h, g1, g2))
        if abs(g1 - g2) <= agree * abs(g1):
            return g1, h
    raise AssertionError(f"no crossing-free step in {ladder}: {seen}")


def test_adj_gradient_checkpointed(isfpkg, setup):
    """isf_adj_gradient over 2 init iterations and 4 steps with checkpoints
    every 2 steps: the loss, dL/dpsi0 and dL/dparticles0 along random
    directions, and dL/d(kvec, omega), against FP64 central differences.
    Every direction drawn is checked (fd_without_crossing picks its step)."""
    isf, orc = setup
    rng = np.random.default_rng(8)
    psi0 = f32(smooth_psi(DIMS, 8))
    P = 2048
    p0 = f32(rng.uniform(0.15, 0.85, (P, 3)) * np.asarray(L))
    kvec = (float(np.float32(6.0)), 0.0, 0.0)
    omega = float(np.float32(1.8))
    T, K, I = 4, 2, 2
    # targets: the FP64 end positions plus noise
    x = p0.copy()
    ps = psi0.copy()
    cen, ln, rad = NOZZLE
    for _ in range(I):
        orc.restrict_velocity(ps, kvec, 0.0, cen, ln, rad, phase_mode=1)
        orc.pressure_project(ps)
    for n in range(1, T + 1):
        tn = float(np.float32(n) * np.float32(DT))
        orc.step(ps, x, dict(kvec=kvec, omega_t=omega * tn, cen=cen, len=ln, rad=rad, emit_count=0, counter=n,
                             phase_mode=1))
    tgt = f32(x + rng.normal(0, 0.1, x.shape))
    prob = isfpkg.adj_problem(T, K, kvec, omega, NOZZLE, init_iters=I)
    loss, gpsi, gp, jb = isfpkg.adj_gradient(isf, prob, cuda(psi0), cuda(p0), cuda(tgt))
    lossf = isfpkg.adj_loss(isf, prob, cuda(psi0), cuda(p0), cuda(tgt))
    ref = driver_forward(orc, psi0, p0, tgt, T, I, kvec, omega)
    assert abs(loss - ref) <= 1e-4 * ref and abs(lossf - ref) <= 1e-4 * ref, (loss, lossf, ref)
    gpsi, gp = host(gpsi), host(gp)

    def Lf(dpsi=0.0, dp=0.0, k=kvec, w=omega):
        return driver_forward(orc, psi0 + dpsi, p0 + dp, tgt, T, I, k, w)

    for d in range(4):
        u = rng.normal(size=psi0.shape)
        g, h = fd_without_crossing(lambda t: Lf(dpsi=t * u))
        assert close(dot(gpsi, u), g, tol=2e-3), (d, h, dot(gpsi, u), g)
    up = rng.normal(size=p0.shape)
    g, h = fd_without_crossing(lambda t: Lf(dp=t * up))
    assert close(dot(gp, up), g, tol=2e-3), (h, dot(gp, up), g)
    # the jet phase is common to both components: a gauge, so dL/dkvec and
    # dL/domega vanish (up to rounding) on the GPU and in the FP64 differences
    scale = abs(dot(gp, up))
    for a in range(3):
        e = np.zeros(3)
        e[a] = 1e-6
        g = (Lf(k=tuple(np.add(kvec, e))) - Lf(k=tuple(np.add(kvec, -e)))) / 2e-6
        assert abs(jb[a] - g) <= 1e-3 * scale, (a, jb[a], g)
    g = (Lf(w=omega + 1e-6) - Lf(w=omega - 1e-6)) / 2e-6
    assert abs(jb[3] - g) <= 1e-3 * scale, (jb[3], g)


def test_adj_gradient_jet_64x32x32_50_steps(isfpkg, oracle_mod, cfgs):
    """The adjoint workload at full size: the 64x32x32 jet, 65 536 particles
    uniform in the box, 10 initialisation projections, 50 steps with psi
    checkpointed every 10 steps, targets the FP64 end positions plus Gaussian
    offsets of sigma 0.1 (seed 4).

    psi0 is a smooth non-uniform state.  At the jet's uniform psi0
    (psi1 = 1, psi2 = 0.01) the loss is stationary: a perturbation changes the
    velocity to first order only by an exact one-form, which the projection
    removes, so positions move as h^2 and every directional derivative in psi0
    vanishes (as do those in kvec and omega, a gauge).

    Over 50 steps the FP32 and FP64 trajectories of a particle whose RK
    sample points pass within rounding distance of a cell face can use
    different cells, where the unnormalised interpolation's derivative
    differs (about 0.2 % of the gradient with every particle kept).  As in
    the forward parity tests, the particles whose FP64 sample points came
    within 1e-4 cells of a face are left out (dead from the start, so
    neither the GPU loss nor the oracle's includes them).  Every one of the 8
    psi0 directions and 2 particle directions drawn is checked, each with a
    crossing-free step from fd_without_crossing, within 1e-3."""
    c = cfgs.CONFIGS["C1"]
    Lc, dims = c["L"], c["dims"]
    isf = isfpkg.ISF(Lc, dims, c["hbar"], c["dt"])
    orc = oracle_mod.Oracle(Lc, dims, c["hbar"], c["dt"])
    kvec, omega = cfgs.jet_omega(c["hbar"])
    noz = cfgs.JET_NOZZLE
    nozzle = (noz["cen"], noz["len"], noz["rad"])
    T, K, I, P = 50, 10, 10, 65536
    rng = np.random.Generator(np.random.Philox(4))
    p0 = f32(rng.uniform(0.1, 0.9, (P, 3)) * np.asarray(Lc))
    psi0 = f32(smooth_psi(dims, 5))

    def forward(psi, x, margin=None):
        psi, x = psi.copy(), x.copy()
        for _ in range(I):
            orc.restrict_velocity(psi, kvec, 0.0, *nozzle, phase_mode=1)
            orc.pressure_project(psi)
        for n in range(1, T + 1):
            tn = float(np.float32(n) * np.float32(c["dt"]))
            m = np.zeros(len(x)) if margin is not None else None
            orc.step(psi, x, dict(kvec=kvec, omega_t=omega * tn, cen=noz["cen"], len=noz["len"], rad=noz["rad"],
                                  emit_count=0, counter=n, phase_mode=1), margin=m)
            if margin is not None:
                np.minimum(margin, m, out=margin)
        return x

    margin = np.full(P, 1e30)
    xT = forward(psi0, p0, margin)
    near = margin <= 1e-4
    assert near.mean() < 0.2, near.mean()
    p0[near] = -1.0
    tgt = f32(xT + rng.normal(0, 0.1, p0.shape))

    def Lf(dpsi=0.0, dp=0.0):
        x = forward(psi0 + dpsi, p0 + dp)
        alive = x[:, 0] >= 0
        return float(((x[alive] - tgt[alive]) ** 2).sum())

    prob = isfpkg.adj_problem(T, K, kvec, omega, nozzle, init_iters=I)
    loss, gpsi, gp, jb = isfpkg.adj_gradient(isf, prob, cuda(psi0), cuda(p0), cuda(tgt))
    ref = Lf()
    assert abs(loss - ref) <= 1e-4 * ref, (loss, ref)
    gpsi, gp = host(gpsi), host(gp)
    worst = 0.0
    for d in range(8):
        u = rng.normal(size=psi0.shape)
        g, h = fd_without_crossing(lambda t: Lf(dpsi=t * u))
        worst = max(worst, abs(dot(gpsi, u) - g) / abs(g))
        assert close(dot(gpsi, u), g), (d, h, dot(gpsi, u), g)
    for d in range(2):
        up = rng.normal(size=p0.shape)
        g, h = fd_without_crossing(lambda t: Lf(dp=t * up))
        worst = max(worst, abs(dot(gp, up) - g) / abs(g))
        assert close(dot(gp, up), g), (d, h, dot(gp, up), g)
    print(f"jet 64x32x32, 50 steps, 10 directions: worst relative error {worst:.2e}")
    isf.close()


def test_particle_loss_autograd(isfpkg, setup):
    """ParticleLoss (the rrule counterpart) returns the gradient of
    isf_adj_gradient through torch.autograd."""
    isf, orc = setup
    rng = np.random.default_rng(9)
    psi0 = cuda(smooth_psi(DIMS, 9)).requires_grad_(True)
    P = 1024
    p0 = cuda(rng.uniform(0.15, 0.85, (P, 3)) * np.asarray(L))
    tgt = p0 + 0.05
    kvec = torch.tensor([6.0, 0.0, 0.0], device="cuda", requires_grad=True)
    omega = torch.tensor(1.8, device="cuda", requires_grad=True)
    prob = isfpkg.adj_problem(3, 2, (6.0, 0.0, 0.0), 1.8, NOZZLE, init_iters=1)
    loss = isfpkg.ParticleLoss.apply(psi0, kvec, omega, isf, prob, p0, tgt)
    (2.0 * loss).backward()
    l2, g, _, jb = isfpkg.adj_gradient(isf, prob, psi0.detach(), p0, tgt)
    assert abs(float(loss) - l2) <= 1e-6 * abs(l2)
    assert torch.allclose(psi0.grad, 2.0 * g, rtol=1e-5, atol=1e-7)
    # kvec and omega act as a gauge (see test_adj_gradient_checkpointed): their
    # gradients are rounding noise, which the atomic accumulation orders
    # differently from run to run
    scale = float(psi0.grad.abs().sum())
    assert float(omega.grad.abs()) <= 1e-6 * scale and float(kvec.grad.abs().max()) <= 1e-6 * scale


def test_adj_errors(isfpkg, setup):
    isf, _ = setup
    t = torch.zeros(isf.shape + (4,), device="cuda")
    with pytest.raises(isfpkg.ISFError):
        isfpkg.adj_restrict_velocity(isf, t, t, (1, 0, 0), 0.0, nozzle=NOZZLE, phase_mode=7)
    prob = isfpkg.adj_problem(0, 1, (1, 0, 0), 1.0, NOZZLE)
    p = torch.zeros((8, 3), device="cuda")
    with pytest.raises(isfpkg.ISFError, match="nsteps"):
        isfpkg.adj_loss(isf, prob, t, p, p)
