"""Cell-sorted traversal of the particle slots (isf_set_particle_order,
isf_sort_particles, isf_get_particle_order), through the C ABI.

staggered_advect! (src/parallel.jl:248-261) advects every slot in storage
order.  The ordered traversal visits the same slots in a permutation that
groups live particles by 2 x 2 x 2 cell tile and puts dead slots last; a
slot is never moved and each particle's arithmetic is unchanged, so the
positions must be bitwise those of storage order."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def tile_keys(parts, L, dims):
    """The sort key of every slot, in float32 arithmetic like the kernel."""
    L32 = np.asarray(L, np.float32)
    d = (L32 / np.asarray(dims, np.float32)).astype(np.float32)
    dinv = (np.float32(1) / d).astype(np.float32)
    p = parts.astype(np.float32)
    inside = np.all((p > 0) & (p < L32), axis=1)
    c = np.minimum((p * dinv).astype(np.int64), np.asarray(dims) - 1) >> 1
    t = (np.asarray(dims) + 1) >> 1
    key = c[:, 0] + t[0] * (c[:, 1] + t[1] * c[:, 2])
    return np.where(inside, key, t.prod())


def test_sort_particles_gives_a_cell_sorted_permutation(isfpkg, cfgs):
    L, dims = (4, 2, 2), (64, 32, 32)
    isf = isfpkg.ISF(L, dims, cfgs.HBAR, float(np.float32(1 / 48)))
    rng = np.random.default_rng(5)
    P = 50_000
    parts = (rng.uniform(-0.1, 1.1, (P, 3)) * np.asarray(L)).astype(np.float32)
    parts[rng.random(P) < 0.2] = -1.0          # dead slots
    t = cuda(parts)
    assert isf.particle_order() is None
    isf.sort_particles(t)
    order = isf.particle_order().cpu().numpy().astype(np.int64)
    assert np.array_equal(np.sort(order), np.arange(P))          # every slot exactly once
    keys = tile_keys(parts, L, dims)[order]
    assert np.all(np.diff(keys) >= 0)                            # grouped by tile, dead slots last
    live = int(np.all((parts > 0) & (parts < np.asarray(L, np.float32)), axis=1).sum())
    assert np.all(keys[:live] < keys[-1]) and np.all(keys[live:] == keys[-1])
    isf.set_particle_order(0)
    assert isf.particle_order() is None
    isf.close()


@pytest.mark.parametrize("jet", [False, True])
def test_ordered_steps_are_bitwise_storage_order(isfpkg, cfgs, jet):
    """9 steps with the permutation rebuilt every 3 steps against the same
    steps in storage order: psi, positions and the live and clamp counters
    bitwise equal.  The jet case emits 500 particles per step into a ring of
    slots, so slots come alive between rebuilds."""
    L, dims = (4, 2, 2), (64, 32, 32)
    hbar, dt = cfgs.HBAR, float(np.float32(1 / 48))
    kvec, omega = cfgs.jet_omega(hbar)
    noz = cfgs.JET_NOZZLE
    rng = np.random.default_rng(6)
    P = 40_000
    if jet:
        psi0 = cfgs.jet_init_psi(dims)
        p0 = np.full((P, 3), -1.0, np.float32)
        p0[: P // 2] = rng.uniform(0.05, 0.95, (P // 2, 3)) * np.asarray(L)
    else:
        from helpers import smooth_psi
        psi0 = smooth_psi(dims, 6)
        p0 = (rng.uniform(0.02, 0.98, (P, 3)) * np.asarray(L)).astype(np.float32)
    out = []
    for every in (0, 3):
        isf = isfpkg.ISF(L, dims, hbar, dt)
        isf.set_particle_order(every)
        psi, parts = cuda(psi0), cuda(p0)
        live = []
        for it in range(1, 10):
            args = None
            if jet:
                t = np.float32(it) * np.float32(dt)
                args = dict(kvec=kvec, omega_t=float(np.float32(omega) * t), cen=noz["cen"], len=noz["len"],
                            rad=noz["rad"], emit_start=P // 2 + (it - 1) * 500, emit_count=500, seed=3, counter=it,
                            emit_mode=isfpkg.EMIT_DISC, phase_mode=isfpkg.PHASE_DOT)
            isfpkg.step(isf, psi, parts, args)
            c = isf.counters(reset=True)
            live.append((c["live"], c["clamp_events"]))
        isf.sync()
        if every:
            assert isf.particle_order() is not None
        out.append((psi.cpu().numpy(), parts.cpu().numpy(), live))
        isf.close()
    (psi_a, parts_a, live_a), (psi_b, parts_b, live_b) = out
    assert np.array_equal(psi_a.view(np.uint32), psi_b.view(np.uint32))
    assert np.array_equal(parts_a.view(np.uint32), parts_b.view(np.uint32))
    assert live_a == live_b


_INDEX_RUN = r"""
import hashlib, sys, numpy as np, torch
sys.path.insert(0, sys.argv[1])
sys.path.insert(0, sys.argv[2])
import __graft_entry__ as ge
from helpers import smooth_psi
pkg = ge.load_package()
L, dims = (4, 2, 2), (64, 32, 32)
rng = np.random.default_rng(7)
p0 = (rng.uniform(-0.05, 1.05, (30000, 3)) * np.asarray(L)).astype(np.float32)
p0[:16] = np.asarray(L, np.float32) * np.float32(0.999999)   # near the upper faces
isf = pkg.ISF(L, dims, float(np.float32(0.1)), float(np.float32(1 / 48)))
psi = torch.tensor(smooth_psi(dims, 6), dtype=torch.float32, device="cuda")
parts = torch.tensor(p0, device="cuda")
cnt = []
for _ in range(12):
    pkg.step(isf, psi, parts, None)
    c = isf.counters(reset=True)
    cnt.append((c["live"], c["clamp_events"]))
isf.sync()
print(hashlib.md5(parts.cpu().numpy().tobytes()).hexdigest(), cnt)
"""


def test_float_and_integer_cell_index_agree_bitwise():
    """The advection forms the base cell index from the three floors in float
    (exact below 2^24 padded cells) or in integers (larger grids).  The same
    12 steps, in two processes, one forced onto the integer index: the
    positions and the live / clamp counters agree bitwise."""
    import os
    import subprocess
    import sys
    repo = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    tests = os.path.dirname(os.path.abspath(__file__))
    outs = []
    for force in (False, True):
        env = dict(os.environ)
        env.pop("ISF_ADVECT_INT_INDEX", None)
        if force:
            env["ISF_ADVECT_INT_INDEX"] = "1"
        r = subprocess.run([sys.executable, "-c", _INDEX_RUN, repo, tests], env=env, capture_output=True, text=True,
                           timeout=600)
        assert r.returncode == 0, r.stderr[-2000:]
        outs.append(r.stdout.strip().splitlines()[-1])
    assert outs[0] == outs[1], outs
