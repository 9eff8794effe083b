"""Synthetic workloads of the ISF benchmarks (host-side set-up only).

C1  jet, 4x2x2 torus, 64x32x32, hbar 0.1, dt 1/48, 1000 particles/step from
    the nozzle disc (seed 0), 100 steps            (examples/benchmark.jl:4-38
    with the metric's nozzle; the reference's CPU test is the 128x64x64 one)
C2  jet, 4x2x2 torus, 128x64x64, 1M particles seeded in the nozzle (seed 1)
C3  leapfrogging vortex rings, 10x5x5 torus, 256x128x128, hbar 0.1, dt 1/24,
    4M particles in thin tori around the rings (seed 2), no nozzle
C4  ensemble of jets on {32^3, 48x32x32, 64x32x32, 96x48x48} with d = 1/16 (ensemble())
C5  adjoint jet on the C1 grid (65536 particles)

The reference ships only the jet set-up (examples/benchmark.jl:4-38).  The
vortex-ring initial phase has no reference code; it is defined here: for a
ring of radius R about an axis through c with unit normal n, a cell at
axial offset s = (p - c).n and distance rho from the axis gets the phase

    alpha = pi (1 - 2 s / delta)      for 0 <  s <= delta/2, rho < R
    alpha = -pi (1 + 2 s / delta)     for -delta/2 <= s <= 0, rho < R
    alpha = 0                         elsewhere,

i.e. a 2 pi phase jump across the disc spanned by the ring, spread linearly
over a slab of thickness delta, so the phase winds once around the ring
(the standard construction of a quantised vortex ring).  Inside the disc the
phase falls along n, so the flow through the ring, and the ring itself, move
along -n.  psi1 is the product of exp(i alpha) over the rings, psi2 = 0.01,
and psi is normalised.  C3 starts the smaller (faster) ring 1.5 behind the
larger one, both travelling +x, so that the pair leapfrogs and stays inside
the 10-long box for the configuration's 500 steps.
"""
from __future__ import annotations

import numpy as np

HBAR = float(np.float32(0.1))

JET_NOZZLE = {
    # examples/benchmark.jl:9-12
    "velocity": (1.0, 0.0, 0.0),
    "cen": tuple(float(np.float32(v)) for v in (2 - 1.7, 1 - 0.034, 1 + 0.066)),
    "len": 0.5,
    "rad": 0.5,
}

CONFIGS = {
    "C1": dict(name="jet_64x32x32", L=(4, 2, 2), dims=(64, 32, 32), hbar=HBAR, dt=float(np.float32(1 / 48)),
               jet=True, steps=100, emit_per_step=1000, slots=100_000, seed=0, emit_mode=1),
    "C2": dict(name="jet_128x64x64", L=(4, 2, 2), dims=(128, 64, 64), hbar=HBAR, dt=float(np.float32(1 / 48)),
               jet=True, steps=200, emit_per_step=0, particles=1 << 20, seed=1),
    "C3": dict(name="vortex_rings_256x128x128", L=(10, 5, 5), dims=(256, 128, 128), hbar=HBAR,
               dt=float(np.float32(1 / 24)), jet=False, steps=500, particles=4 * 1024 * 1024, seed=2,
               rings=((1.5, 0.6), (3.0, 0.9)), ring_yz=(2.5, 2.5), normal=(-1.0, 0.0, 0.0), delta=0.2,
               torus_minor=0.1),
}


def jet_omega(hbar: float = HBAR):
    v = np.asarray(JET_NOZZLE["velocity"], np.float32)
    h = np.float32(hbar)
    kvec = v / h                                         # examples/benchmark.jl:24
    omega = np.float32(np.sum(v ** np.float32(2)) / (np.float32(2) * h))  # :25
    return tuple(float(k) for k in kvec), float(omega)


def vortex_ring_phase(dims, L, rings, ring_yz, delta, normal=(1.0, 0.0, 0.0)):
    """Total phase alpha(x) (nz, ny, nx) of coaxial rings [(x_centre, R), ...]."""
    nx, ny, nz = dims
    d = [np.float64(np.float32(Lk / nk)) for Lk, nk in zip(L, dims)]
    x = np.arange(nx) * d[0]
    y = np.arange(ny) * d[1]
    z = np.arange(nz) * d[2]
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    n = np.asarray(normal, np.float64)
    n = n / np.linalg.norm(n)
    alpha = np.zeros(X.shape)
    for xc, R in rings:
        rx, ry, rz = X - xc, Y - ring_yz[0], Z - ring_yz[1]
        s = rx * n[0] + ry * n[1] + rz * n[2]
        rho2 = rx * rx + ry * ry + rz * rz - s * s
        inside = rho2 < R * R
        up = inside & (s > 0) & (s <= delta / 2)
        dn = inside & (s <= 0) & (s >= -delta / 2)
        alpha[up] += np.pi * (1 - 2 * s[up] / delta)
        alpha[dn] += -np.pi * (1 + 2 * s[dn] / delta)
    return alpha


def vortex_rings_psi(cfg) -> np.ndarray:
    """Normalised psi (nz, ny, nx, 4) float64 of the leapfrog configuration."""
    a = vortex_ring_phase(cfg["dims"], cfg["L"], cfg["rings"], cfg["ring_yz"], cfg["delta"],
                          cfg.get("normal", (1.0, 0.0, 0.0)))
    p1 = np.exp(1j * a)
    p2 = np.full(a.shape, 0.01 + 0j)
    nrm = np.sqrt(np.abs(p1) ** 2 + np.abs(p2) ** 2)
    p1, p2 = p1 / nrm, p2 / nrm
    return np.ascontiguousarray(np.stack([p1.real, p1.imag, p2.real, p2.imag], axis=-1))


def torus_particles(n, rings, ring_yz, minor, seed, normal_axis=0) -> np.ndarray:
    """n points uniform in volume in thin tori (minor radius `minor`) around
    each ring, split evenly between the rings; numpy Philox stream `seed`."""
    rng = np.random.Generator(np.random.Philox(seed))
    out = []
    per = [n // len(rings) + (1 if i < n % len(rings) else 0) for i in range(len(rings))]
    for (xc, R), m in zip(rings, per):
        got = []
        need = m
        while need > 0:
            k = int(need * 1.3) + 64
            phi = rng.uniform(0, 2 * np.pi, k)
            rr = minor * np.sqrt(rng.uniform(0, 1, k))
            th = rng.uniform(0, 2 * np.pi, k)
            # volume element of the torus ~ (R + rr cos th): rejection
            keep = rng.uniform(0, 1, k) * (R + minor) <= (R + rr * np.cos(th))
            rad = (R + rr * np.cos(th))[keep]
            ax = (rr * np.sin(th))[keep]
            ph = phi[keep]
            pts = np.stack([xc + ax, ring_yz[0] + rad * np.cos(ph), ring_yz[1] + rad * np.sin(ph)], axis=1)
            got.append(pts[:need])
            need -= len(pts[:need])
        out.append(np.concatenate(got))
    return np.ascontiguousarray(np.concatenate(out)).astype(np.float64)


def jet_init_psi(dims) -> np.ndarray:
    """psi = (1, 0.01) everywhere, normalised (examples/benchmark.jl:20-22), float64."""
    nx, ny, nz = dims
    p = np.zeros((nz, ny, nx, 4))
    a, b = 1.0, 0.01
    nrm = np.hypot(a, b)
    p[..., 0] = a / nrm
    p[..., 2] = b / nrm
    return p


def cell_sort_order(parts: np.ndarray, L, dims) -> np.ndarray:
    """Permutation that orders particles by their cell index (x fastest)."""
    d = np.asarray([Lk / nk for Lk, nk in zip(L, dims)])
    ijk = np.clip(np.floor(parts / d).astype(np.int64), 0, np.asarray(dims) - 1)
    key = ijk[:, 0] + dims[0] * (ijk[:, 1] + dims[1] * ijk[:, 2])
    return np.argsort(key, kind="stable")


# C4: the ensemble grids, d = 1/16 (physical sizes are integers, as the
# reference's IntType physical_size requires, src/parallel.jl:12)
ENSEMBLE_GRIDS = (((32, 32, 32), (2, 2, 2)), ((48, 32, 32), (3, 2, 2)), ((64, 32, 32), (4, 2, 2)),
                  ((96, 48, 48), (6, 3, 3)))


def nozzle_particles(n, cen, length, rad, seed) -> np.ndarray:
    """n points uniform in the nozzle cylinder (axis x), numpy Philox stream `seed`."""
    rng = np.random.Generator(np.random.Philox(seed))
    th = rng.uniform(0, 2 * np.pi, n)
    r = rad * np.sqrt(rng.uniform(0, 1, n))
    x = cen[0] + (rng.uniform(0, 1, n) - 0.5) * length
    return np.ascontiguousarray(np.stack([x, cen[1] + r * np.cos(th), cen[2] + r * np.sin(th)], axis=1))


def ensemble(nsims=64, seed=3, nslots=65536, hbar=HBAR, dt=float(np.float32(1 / 48))):
    """The C4 ensemble: nsims jets on grids drawn uniformly from
    ENSEMBLE_GRIDS, nozzle speed U[0.5, 1.5] along x, each with nslots
    particles seeded in its nozzle cylinder at t = 0 and no emission.
    Returns (batch simulation dicts, psi0 list, particles0 list)."""
    rng = np.random.Generator(np.random.Philox(seed))
    picks = rng.integers(0, len(ENSEMBLE_GRIDS), nsims)
    speeds = rng.uniform(0.5, 1.5, nsims)
    noz = JET_NOZZLE
    sims, psi0, parts0 = [], [], []
    h = np.float32(hbar)
    for i in range(nsims):
        dims, L = ENSEMBLE_GRIDS[picks[i]]
        v = np.float32(speeds[i])
        kvec = (float(v / h), 0.0, 0.0)
        omega = float(np.float32(v * v / (np.float32(2) * h)))
        sims.append(dict(dims=dims, physical_size=L, hbar=hbar, dt=dt, nslots=nslots,
                         jet=dict(kvec=kvec, omega=omega, cen=noz["cen"], len=noz["len"], rad=noz["rad"],
                                  phase_mode=1, emit_mode=1, emit_per_step=0, seed=seed)))
        psi0.append(jet_init_psi(dims).astype(np.float32))
        p = nozzle_particles(nslots, noz["cen"], noz["len"], noz["rad"], seed * 1000 + i)
        parts0.append(p[cell_sort_order(p, L, dims)].astype(np.float32))
    return sims, psi0, parts0


def sim_cost(sim) -> int:
    """Bytes one no-jet step of a simulation moves by the per-step convention
    of the step roofline: 196 B per cell + 24 B per particle slot (a jet step
    adds 76 B per cell on every simulation alike, so the ranking is the same)."""
    n = sim["dims"]
    return 196 * int(n[0]) * int(n[1]) * int(n[2]) + 24 * int(sim.get("nslots", 0))


def shard(costs, world: int):
    """Split independent simulations over `world` ranks (one GPU each, no
    collective): longest first onto the least loaded rank, ties to the lower
    rank and the lower index, so every rank computes the same split.  Returns
    one ascending index list per rank."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += costs[i]
        parts[r].append(i)
    return [sorted(p) for p in parts]
