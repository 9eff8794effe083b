"""The batched ensemble (isf_batch_*, through the C ABI): every simulation of
a batch must follow exactly the path of a single-simulation handle stepped
with isf_step (bit for bit, whatever tiles the autotuner picks), and stay
within the parity bar of the FP64 oracle."""
import numpy as np
import pytest
import torch

from helpers import rel

pytestmark = pytest.mark.gpu


def cuda(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float32, device="cuda")


def small_ensemble(cfgs, nslots=4096):
    """Two simulations in the 64x32x32 class, one in each other class, one
    jet with ring emission, one plain (no jet) simulation."""
    sims, psi0, parts0 = cfgs.ensemble(nsims=6, seed=3, nslots=nslots)
    sims[0]["dims"], sims[0]["physical_size"] = (64, 32, 32), (4, 2, 2)
    sims[1]["dims"], sims[1]["physical_size"] = (64, 32, 32), (4, 2, 2)
    sims[2]["dims"], sims[2]["physical_size"] = (32, 32, 32), (2, 2, 2)
    sims[3]["dims"], sims[3]["physical_size"] = (48, 32, 32), (3, 2, 2)
    sims[4]["dims"], sims[4]["physical_size"] = (96, 48, 48), (6, 3, 3)
    sims[5]["dims"], sims[5]["physical_size"] = (32, 32, 32), (2, 2, 2)
    sims[4]["jet"].update(emit_mode=0, emit_per_step=300, seed=11)   # reference ring emission
    sims[5]["jet"] = None                                           # plain step
    psi0 = [cfgs.jet_init_psi(s["dims"]).astype(np.float32) for s in sims]
    for i, s in enumerate(sims):
        p = cfgs.nozzle_particles(nslots, cfgs.JET_NOZZLE["cen"], 0.5, 0.5, 100 + i)
        if i == 4:
            p[:] = -1.0   # filled by emission only
        parts0[i] = p.astype(np.float32)
    return sims, psi0, parts0


def plain_run(isfpkg, s, psi0, parts0, init_iters, steps):
    """The same simulation through a single-simulation handle and isf_step."""
    isf = isfpkg.ISF(s["physical_size"], s["dims"], s["hbar"], s["dt"])
    psi = cuda(psi0)
    parts = cuda(parts0)
    j = s["jet"]
    if j is not None:
        for _ in range(init_iters):
            isfpkg.restrict_velocity(isf, psi, j["kvec"], None, 0.0, nozzle=(j["cen"], j["len"], j["rad"]),
                                     phase_mode=j["phase_mode"])
            isfpkg.pressure_project(isf, psi)
    dt32 = np.float32(s["dt"])
    for k in range(1, steps + 1):
        jet = None
        if j is not None:
            t = np.float32(k) * dt32
            jet = dict(kvec=j["kvec"], omega_t=float(np.float32(j["omega"]) * t), cen=j["cen"], len=j["len"],
                       rad=j["rad"], phase_mode=j["phase_mode"], emit_mode=j["emit_mode"],
                       emit_start=((k - 1) * j["emit_per_step"]) % s["nslots"], emit_count=j["emit_per_step"],
                       seed=j["seed"], counter=k)
        isfpkg.step(isf, psi, parts, jet)
    isf.sync()
    return psi, parts


def batch_run(isfpkg, sims, psi0, parts0, init_iters, steps, tune):
    b = isfpkg.ISFBatch(sims, tune=tune)
    for i in range(len(sims)):
        b.set_psi(i, cuda(psi0[i]))
        b.set_particles(i, cuda(parts0[i]))
    b.init_jet(init_iters)
    b.step(steps)
    b.sync()
    return b


def test_batch_equals_plain_runs_bitwise(isfpkg, cfgs):
    sims, psi0, parts0 = small_ensemble(cfgs)
    steps = 6
    b = batch_run(isfpkg, sims, psi0, parts0, 10, steps, tune=True)
    ncls, sim_class = b.classes()
    assert ncls == 5
    assert sim_class[0] == sim_class[1]
    for c in range(ncls):
        assert set(b.tiles(c).values()) <= {1, 2, 4}
    for i, s in enumerate(sims):
        psi, parts = plain_run(isfpkg, s, psi0[i], parts0[i], 10, steps)
        assert torch.equal(b.psi(i), psi), i
        assert torch.equal(b.particles(i), parts), i
    live = b.counters(4)["live"]        # live particles summed over the advections since create
    assert 0 < live <= 300 * steps * (steps + 1) // 2


def test_batch_tiles_do_not_change_results(isfpkg, cfgs):
    sims, psi0, parts0 = small_ensemble(cfgs)
    a = batch_run(isfpkg, sims, psi0, parts0, 3, 4, tune=False)
    b = batch_run(isfpkg, sims, psi0, parts0, 3, 4, tune=True)
    for c in range(a.classes()[0]):
        assert set(a.tiles(c).values()) == {1}
    for i in range(len(sims)):
        assert torch.equal(a.psi(i), b.psi(i)), i
        assert torch.equal(a.particles(i), b.particles(i)), i


def test_batch_step_counter_and_restart(isfpkg, cfgs):
    """Stepping 3 + 2 equals stepping 5; set_step rewinds the jet clock."""
    sims, psi0, parts0 = small_ensemble(cfgs)
    a = batch_run(isfpkg, sims, psi0, parts0, 2, 5, tune=False)
    b = batch_run(isfpkg, sims, psi0, parts0, 2, 3, tune=False)
    b.step(2)
    b.sync()
    for i in range(len(sims)):
        assert torch.equal(a.psi(i), b.psi(i)), i
        assert torch.equal(a.particles(i), b.particles(i)), i
    # restart from step 3's state with the counter at 3
    c = batch_run(isfpkg, sims, psi0, parts0, 2, 3, tune=False)
    psi3 = [c.psi(i) for i in range(len(sims))]
    parts3 = [c.particles(i) for i in range(len(sims))]
    d = isfpkg.ISFBatch(sims, tune=False)
    for i in range(len(sims)):
        d.set_psi(i, psi3[i])
        d.set_particles(i, parts3[i])
    d.set_step(3)
    d.step(2)
    d.sync()
    for i in range(len(sims)):
        assert torch.equal(a.psi(i), d.psi(i)), i
        assert torch.equal(a.particles(i), d.particles(i)), i


def test_batch_against_fp64_oracle(isfpkg, oracle_mod, cfgs):
    """Two simulations of the batch, 10 steps, against the FP64 oracle."""
    sims, psi0, parts0 = small_ensemble(cfgs)
    steps = 10
    b = batch_run(isfpkg, sims, psi0, parts0, 10, steps, tune=True)
    for i in (2, 4):
        s, j = sims[i], sims[i]["jet"]
        orc = oracle_mod.Oracle(s["physical_size"], s["dims"], s["hbar"], s["dt"])
        psi = psi0[i].astype(np.float64)
        parts = parts0[i].astype(np.float64)
        for _ in range(10):
            orc.restrict_velocity(psi, j["kvec"], 0.0, j["cen"], j["len"], j["rad"], phase_mode=j["phase_mode"])
            orc.pressure_project(psi)
        margin = np.full(len(parts), 1e30)
        dt32 = np.float32(s["dt"])
        for k in range(1, steps + 1):
            t = np.float32(k) * dt32
            jet = dict(kvec=j["kvec"], omega_t=float(np.float32(j["omega"]) * t), cen=j["cen"], len=j["len"],
                       rad=j["rad"], phase_mode=j["phase_mode"], emit_mode=j["emit_mode"],
                       emit_start=((k - 1) * j["emit_per_step"]) % s["nslots"], emit_count=j["emit_per_step"],
                       seed=j["seed"], counter=k)
            m = np.zeros(len(parts))
            orc.step(psi, parts, jet, margin=m)
            margin = np.minimum(margin, m)
        g = b.psi(i).double().cpu().numpy()
        assert rel(g, psi) < 1e-4, i
        pg = b.particles(i).double().cpu().numpy()
        both = (pg[:, 0] >= 0) & (parts[:, 0] >= 0) & (margin > 1e-4)
        assert both.sum() > 0.5 * (pg[:, 0] >= 0).sum()
        assert (np.abs(pg - parts).max(axis=1)[both] / min(s["physical_size"])).max() < 1e-4
        assert ((pg[:, 0] >= 0) != (parts[:, 0] >= 0)).sum() <= 1e-3 * len(parts)


def test_batch_errors(isfpkg, cfgs):
    sims, psi0, parts0 = small_ensemble(cfgs)
    bad = [dict(sims[0]), dict(sims[1])]
    bad[1]["dims"] = (22, 32, 32)
    with pytest.raises(isfpkg.ISFError, match="simulation 1"):
        isfpkg.ISFBatch(bad)
    bad = [dict(sims[0])]
    bad[0]["jet"] = dict(sims[0]["jet"], emit_per_step=5000)
    with pytest.raises(isfpkg.ISFError, match="emit_per_step"):
        isfpkg.ISFBatch(bad)
    b = isfpkg.ISFBatch(sims[:2], tune=False)
    with pytest.raises(isfpkg.ISFError, match="out of range"):
        b.counters(7)
    with pytest.raises(isfpkg.ISFError):
        b.set_psi(0, cuda(psi0[2]))   # wrong shape
    with pytest.raises(isfpkg.ISFError, match="nsteps"):
        b.step(-1)


def persistent_run(isfpkg, sims, psi0, parts0, init_iters, chunks, tune=True):
    b = isfpkg.ISFBatch(sims, tune=tune)
    b.set_persistent(True)
    for i in range(len(sims)):
        b.set_psi(i, cuda(psi0[i]))
        b.set_particles(i, cuda(parts0[i]))
    b.init_jet(init_iters)
    for k in chunks:
        b.step(k)
    b.sync()
    return b


def test_persistent_batch_equals_plain_runs_bitwise(isfpkg, cfgs):
    """All steps of a call in one launch of the persistent kernel (passes as
    work items with bounded device-side waits between them): bit for bit the
    single-simulation isf_step runs, across two calls (4 + 2 steps)."""
    sims, psi0, parts0 = small_ensemble(cfgs)
    b = persistent_run(isfpkg, sims, psi0, parts0, 10, (4, 2))
    for i, s in enumerate(sims):
        psi, parts = plain_run(isfpkg, s, psi0[i], parts0[i], 10, 6)
        assert torch.equal(b.psi(i), psi), i
        assert torch.equal(b.particles(i), parts), i
    live = b.counters(4)["live"]
    assert 0 < live <= 300 * 6 * 7 // 2


def test_persistent_wait_times_out_and_the_gpu_keeps_answering(isfpkg, cfgs):
    """A wait that cannot be satisfied (stall: dependent passes also wait for
    a flag that nothing sets) runs out after spin_limit polls: the kernel
    reports ISF_ERR_TIMEOUT through its status word, every block stops, and
    sync raises.  The context stays usable: the same batch, reset and
    stepped again without the stall, matches a graph-mode batch bitwise."""
    sims, psi0, parts0 = small_ensemble(cfgs)
    b = isfpkg.ISFBatch(sims, tune=False)
    for i in range(len(sims)):
        b.set_psi(i, cuda(psi0[i]))
        b.set_particles(i, cuda(parts0[i]))
    b.set_persistent(True, spin_limit=2000, stall=True)
    b.step(3)
    with pytest.raises(isfpkg.ISFError) as err:
        b.sync()
    assert err.value.code == isfpkg._lib.ISF_ERR_TIMEOUT
    assert "ran out" in str(err.value)
    b.set_persistent(True)
    b.set_step(0)
    for i in range(len(sims)):
        b.set_psi(i, cuda(psi0[i]))
        b.set_particles(i, cuda(parts0[i]))
    b.init_jet(2)
    b.step(3)
    b.sync()
    ref = batch_run(isfpkg, sims, psi0, parts0, 2, 3, tune=False)
    for i in range(len(sims)):
        assert torch.equal(b.psi(i), ref.psi(i)), i
        assert torch.equal(b.particles(i), ref.particles(i)), i


def test_persistent_rejects_grids_it_is_not_built_for(isfpkg, cfgs):
    sims, _, _ = cfgs.ensemble(nsims=2, seed=3, nslots=64)
    sims[1]["dims"], sims[1]["physical_size"] = (64, 32, 16), (4, 2, 1)   # ny != nz: no plane solver
    b = isfpkg.ISFBatch(sims, tune=False)
    with pytest.raises(isfpkg.ISFError, match="persistent kernel needs"):
        b.set_persistent(True)
    b.close()
