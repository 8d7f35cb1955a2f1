"""GPU parity of the XPBD path (spatial hash, contact Jacobi passes, sleeping,
MPM contact impulses, swelling) against the CPU oracle, through the C ABI.

The hash (cells, sorted point order, cell ranges) is integer work and must be
bit-exact.  The XPBD kernels use no floating-point atomics and visit
neighbours in the same order as the oracle, so their outputs are compared
exactly as well (tolerance 0 unless stated)."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.harness import gpu_fields, oracle, rel_err, to_oracle, xpbd_scene

pytestmark = pytest.mark.gpu


def test_hash_grid_bit_exact():
    import torch
    from mpmwarpydw_b200.utils.xpbdRoutines import HashGrid
    rng = np.random.default_rng(7)
    for n, w in ((1, 0.5), (5000, 0.25), (70_000, 1.0)):
        x = rng.uniform(-3, 40, (n, 3)).astype(np.float32)
        if n > 10:
            x[: n // 10] = x[0]  # a crowded cell
        hg = HashGrid(128, 128, 128, device="cuda:0")
        hg.build(torch.as_tensor(x, device="cuda:0"), w)
        torch.cuda.synchronize()
        ref = oracle("f32").hash_build(x, w)
        assert np.array_equal(hg.point_cells[:n].cpu().numpy(), ref.point_cells)
        assert np.array_equal(hg.point_ids[:n].cpu().numpy(), ref.point_ids)
        assert np.array_equal(hg.cell_starts.cpu().numpy(), ref.cell_starts)
        assert np.array_equal(hg.cell_ends.cpu().numpy(), ref.cell_ends)


@pytest.mark.parametrize("lock,xpbd_only", [(1, False), (0, False), (1, True)])
def test_xpbd_step_matches_oracle(lock, xpbd_only):
    import torch
    from mpmwarpydw_b200.utils import simulationRoutines as S
    sim, mpm, xpbd = xpbd_scene(seed=3, lock=lock)
    s = to_oracle(sim, mpm, xpbd)
    S.xpbdSimulationStep(sim, mpm, xpbd, "cuda:0", xpbd_only=xpbd_only)
    torch.cuda.synchronize()
    orc.xpbd_step(oracle("f32"), s, xpbd_only=xpbd_only)
    g = gpu_fields(sim, mpm, xpbd)
    assert np.array_equal(g["materialLabel"], s.materialLabel)
    assert int(sim.numTotalXPBD.item()) == s.numTotalXPBD and int(sim.numSleepingXPBD.item()) == s.numSleepingXPBD
    assert s.numTotalXPBD > 0
    for k in ("particle_x", "particle_v", "particle_x_integrated", "particle_v_integrated", "particle_delta",
              "particle_x_deltaInt", "particle_v_deltaInt", "particle_v_before_contact", "particle_cumDist_xpbd",
              "particle_radius"):
        a, b = g[k], getattr(s, k)
        assert np.array_equal(a, b), (k, rel_err(a, b))


@pytest.mark.parametrize("case", ["no_xpbd_labels", "xpbd_labels_inactive"])
def test_xpbd_step_without_active_xpbd_particles(case):
    """A step with no particle labelled XPBD (the contact passes then return at
    once) is bit-exact with the oracle's full step: contact-locked labels are
    reset, x/v pass through the integrate and impulse copies, deltas stay 0.
    With XPBD labels on inactive particles only, the contact passes run in
    full: the reference's kernel tests activity on the sorted slot, not on the
    particle it works on, so inactive XPBD particles still lock MPM neighbours."""
    import torch
    from mpmwarpydw_b200.utils import simulationRoutines as S
    if case == "no_xpbd_labels":
        sim, mpm, xpbd = xpbd_scene(seed=6, frac_xpbd=0.0, lock=1)
    else:
        sim, mpm, xpbd = xpbd_scene(seed=7, lock=1)
        ml = sim.materialLabel.clone()
        al = sim.activeLabel.clone()
        al[ml == 2] = 0
        sim.activeLabel = al
        assert int((ml == 2).sum().item()) > 0
    s = to_oracle(sim, mpm, xpbd)
    locked = (s.activeLabel == 1) & (s.materialLabel == 0)
    assert int(locked.sum()) > 0  # contact-locked MPM particles, which the step resets
    S.xpbdSimulationStep(sim, mpm, xpbd, "cuda:0")
    torch.cuda.synchronize()
    orc.xpbd_step(oracle("f32"), s)
    g = gpu_fields(sim, mpm, xpbd)
    assert s.numTotalXPBD == 0 and int(sim.numTotalXPBD.item()) == 0
    if case == "no_xpbd_labels":
        assert np.all(g["materialLabel"][locked] == 1)
    assert np.array_equal(g["materialLabel"], s.materialLabel)
    for k in ("particle_x", "particle_v", "particle_x_integrated", "particle_v_integrated", "particle_delta",
              "particle_x_deltaInt", "particle_v_deltaInt", "particle_v_before_contact", "particle_cumDist_xpbd",
              "particle_radius"):
        a, b = g[k], getattr(s, k)
        assert np.array_equal(a, b), (k, rel_err(a, b))


def test_xpbd_step_with_xpbd_particles_in_one_slab():
    """XPBD particles only in a slab at one side of the block: most MPM
    particles have no XPBD-labelled particle in their query box and skip their
    neighbour walk (per-hash-cell presence bits).  Bit-exact with the oracle's
    full step, contact-lock labels included."""
    import torch
    from mpmwarpydw_b200.utils import simulationRoutines as S
    sim, mpm, xpbd = xpbd_scene(seed=9, frac_xpbd=0.0, lock=1)
    x = sim.particle_x
    ml = sim.materialLabel.clone()
    slab = x[:, 0] < float(x[:, 0].min().item()) + 0.6
    ml[slab] = 2
    sim.materialLabel = ml
    s = to_oracle(sim, mpm, xpbd)
    S.xpbdSimulationStep(sim, mpm, xpbd, "cuda:0")
    torch.cuda.synchronize()
    orc.xpbd_step(oracle("f32"), s)
    g = gpu_fields(sim, mpm, xpbd)
    assert 0 < s.numTotalXPBD < sim.nPoints // 3
    assert int(((s.materialLabel == 0) & ~slab.cpu().numpy()).sum()) > 0  # locks next to the slab
    assert np.array_equal(g["materialLabel"], s.materialLabel)
    assert int(sim.numTotalXPBD.item()) == s.numTotalXPBD and int(sim.numSleepingXPBD.item()) == s.numSleepingXPBD
    for k in ("particle_x", "particle_v", "particle_x_integrated", "particle_v_integrated", "particle_delta",
              "particle_x_deltaInt", "particle_v_deltaInt", "particle_v_before_contact", "particle_cumDist_xpbd",
              "particle_radius"):
        a, b = g[k], getattr(s, k)
        assert np.array_equal(a, b), (k, rel_err(a, b))


def test_xpbd_kernels_one_by_one():
    """The reference-named per-kernel callables, in the reference's launch order."""
    import torch
    from mpmwarpydw_b200.utils import xpbdRoutines as X
    sim, mpm, xpbd = xpbd_scene(seed=4, lock=1)
    s = to_oracle(sim, mpm, xpbd)
    o = oracle("f32")
    xpbd.particle_grid.build(sim.particle_x, sim.dx)
    hg = o.hash_build(s.particle_x, s.dx)
    xpbd.particle_x_integrated = sim.particle_x
    xpbd.particle_v_integrated = sim.particle_v
    s.particle_x_integrated[...] = s.particle_x
    s.particle_v_integrated[...] = s.particle_v
    X.integrateParticlesXPBD(sim.activeLabel, sim.materialLabel, xpbd.particle_x_integrated, xpbd.particle_v_integrated,
                             sim.gravity, sim.dtxpbd, xpbd.particle_x_integrated, xpbd.particle_v_integrated,
                             xpbd.particle_v_max)
    o.integrateParticlesXPBD(s.activeLabel, s.materialLabel, s.particle_x_integrated, s.particle_v_integrated,
                             s.gravity, s.dtxpbd, s.particle_v_max)
    X.reset_mpm_contact_labels(sim.activeLabel, sim.materialLabel)
    o.reset_mpm_contact_labels(s.activeLabel, s.materialLabel)
    xpbd.particle_delta.zero_()
    s.particle_delta[...] = 0
    X.my_solve_particle_bound_contacts(sim.activeLabel, sim.materialLabel, xpbd.particle_x_integrated,
                                       xpbd.particle_v_integrated, sim.particle_mass, sim.particle_radius,
                                       xpbd.dynamicParticleFriction, xpbd.staticVelocityThreshold,
                                       xpbd.staticParticleFriction, xpbd.minBoundsXPBD, xpbd.maxBoundsXPBD,
                                       sim.dtxpbd, xpbd.xpbd_relaxation, xpbd.particle_delta)
    o.my_solve_particle_bound_contacts(s.activeLabel, s.materialLabel, s.particle_x_integrated,
                                       s.particle_v_integrated, s.particle_mass, s.particle_radius,
                                       s.dynamicParticleFriction, s.staticVelocityThreshold, s.staticParticleFriction,
                                       s.minBoundsXPBD, s.maxBoundsXPBD, s.dtxpbd, s.xpbd_relaxation, s.particle_delta)
    X.my_solve_particle_particle_contacts(sim.activeLabel, sim.materialLabel, xpbd.particle_grid.id,
                                          xpbd.particle_x_integrated, xpbd.particle_v_integrated, sim.particle_mass,
                                          sim.particle_radius, xpbd.dynamicParticleFriction,
                                          xpbd.staticVelocityThreshold, xpbd.staticParticleFriction,
                                          xpbd.particle_cohesion, xpbd.max_radius, sim.dtxpbd, xpbd.xpbd_relaxation,
                                          1, xpbd.particle_delta)
    o.my_solve_particle_particle_contacts(s.activeLabel, s.materialLabel, hg, s.particle_x_integrated,
                                          s.particle_v_integrated, s.particle_mass, s.particle_radius,
                                          s.dynamicParticleFriction, s.staticVelocityThreshold,
                                          s.staticParticleFriction, s.particle_cohesion, s.max_radius, s.dtxpbd,
                                          s.xpbd_relaxation, 1, s.particle_delta)
    xo = torch.zeros_like(xpbd.particle_x_integrated); vo = torch.zeros_like(xo)
    X.my_apply_particle_deltas(sim.activeLabel, sim.materialLabel, sim.particle_x, xpbd.particle_x_integrated,
                               xpbd.particle_delta, sim.dtxpbd, xpbd.particle_v_max, xo, vo)
    xo_o = np.zeros_like(s.particle_x); vo_o = np.zeros_like(xo_o)
    o.my_apply_particle_deltas(s.activeLabel, s.materialLabel, s.particle_x, s.particle_x_integrated,
                               s.particle_delta, s.dtxpbd, s.particle_v_max, xo_o, vo_o)
    torch.cuda.synchronize()
    g = gpu_fields(sim, mpm, xpbd)
    assert np.array_equal(g["materialLabel"], s.materialLabel)
    assert np.array_equal(g["particle_delta"], s.particle_delta)
    assert np.array_equal(xo.cpu().numpy(), xo_o) and np.array_equal(vo.cpu().numpy(), vo_o)
    tot = torch.zeros(1, dtype=torch.int32, device="cuda"); slp = torch.zeros(1, dtype=torch.int32, device="cuda")
    X.sleepParticles(sim.activeLabel, sim.materialLabel, xpbd.sleepThreshold, sim.particle_radius, sim.particle_x,
                     xo, xpbd.particle_cumDist_xpbd, sim.dtxpbd, tot, slp)
    t2, s2 = o.sleepParticles(s.activeLabel, s.materialLabel, s.sleepThreshold, s.particle_radius, s.particle_x,
                              xo_o, s.particle_cumDist_xpbd, s.dtxpbd)
    torch.cuda.synchronize()
    assert (int(tot.item()), int(slp.item())) == (t2, s2)
    assert np.array_equal(xo.cpu().numpy(), xo_o)
    assert np.array_equal(xpbd.particle_cumDist_xpbd.cpu().numpy(), s.particle_cumDist_xpbd)
