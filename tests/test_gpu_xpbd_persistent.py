"""The XPBD step as one persistent kernel (a cooperative launch whose phases
are separated by bounded grid barriers) against the step as one launch per
pass (utils/simulationRoutines.py:295-526).  Both forms run the same
per-element device code, so every output is compared bit for bit: particle
fields, labels, XPBD counts and the hash arrays.  The per-pass form is itself
pinned to the oracle (tests/test_gpu_xpbd_parity.py); the small scenes here
are also checked against the oracle directly.

Sizes: the small block (1,728 particles, one sort tile), the caving block
(509,696 particles, 35 % XPBD particles, 125 sort tiles) and the tunnel
(3,873,600 particles, 946 sort tiles, more tiles than CTAs in the
cooperative grid, so each CTA sorts several)."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.harness import gpu_fields, oracle, rel_err, to_oracle, xpbd_scene

pytestmark = pytest.mark.gpu

KEYS = ("particle_x", "particle_v", "particle_x_integrated", "particle_v_integrated", "particle_delta",
        "particle_x_deltaInt", "particle_v_deltaInt", "particle_v_before_contact", "particle_cumDist_xpbd",
        "particle_radius", "materialLabel")


def _set_persistent(on):
    from mpmwarpydw_b200 import _lib
    _lib.check(_lib.lib().mpmw_xpbd_set_options(int(on)), "xpbd options")


def _launches():
    from mpmwarpydw_b200 import _lib
    return int(_lib.lib().mpmw_xpbd_persistent_launches())


def _snapshot(sim, mpm, xpbd):
    g = {k: v for k, v in gpu_fields(sim, mpm, xpbd).items() if k in KEYS}
    hg = xpbd.particle_grid
    n = sim.nPoints
    g["point_ids"] = hg.point_ids[:n].cpu().numpy()
    g["cell_starts"] = hg.cell_starts.cpu().numpy()
    g["cell_ends"] = hg.cell_ends.cpu().numpy()
    g["counts"] = np.array([int(sim.numTotalXPBD.item()), int(sim.numSleepingXPBD.item())])
    return g


def _run_both(build, steps, xpbd_only=False):
    """Build the scene twice and step it with each form; returns the two
    snapshots and the number of persistent launches the first form made."""
    import torch

    from mpmwarpydw_b200.bind import read_status
    from mpmwarpydw_b200.utils import simulationRoutines as S
    out, made = [], 0
    try:
        for on in (1, 0):
            _set_persistent(on)
            sim, mpm, xpbd = build()
            read_status(sim.device)
            before = _launches()
            for _ in range(steps):
                S.xpbdSimulationStep(sim, mpm, xpbd, sim.device, xpbd_only=xpbd_only)
            torch.cuda.synchronize()
            if on:
                made = _launches() - before
            assert read_status(sim.device) == 0
            out.append(_snapshot(sim, mpm, xpbd))
    finally:
        _set_persistent(1)
    return out[0], out[1], made


def _assert_same(a, b):
    for k in a:
        assert np.array_equal(a[k], b[k]), (k, rel_err(a[k], b[k]) if a[k].dtype.kind == "f" else "labels")


@pytest.mark.parametrize("lock,xpbd_only", [(1, False), (0, False), (1, True)])
def test_persistent_step_small_block(lock, xpbd_only):
    """Two steps on the small block both ways, and one step against the oracle."""
    import torch

    from mpmwarpydw_b200.utils import simulationRoutines as S
    a, b, made = _run_both(lambda: xpbd_scene(seed=3, lock=lock), 2, xpbd_only)
    assert made == 2
    _assert_same(a, b)
    sim, mpm, xpbd = xpbd_scene(seed=3, lock=lock)
    s = to_oracle(sim, mpm, xpbd)
    before = _launches()
    S.xpbdSimulationStep(sim, mpm, xpbd, "cuda:0", xpbd_only=xpbd_only)
    torch.cuda.synchronize()
    assert _launches() == before + 1
    orc.xpbd_step(oracle("f32"), s, xpbd_only=xpbd_only)
    g = gpu_fields(sim, mpm, xpbd)
    for k in KEYS:
        assert np.array_equal(g[k], getattr(s, k)), (k, rel_err(g[k], getattr(s, k)))
    assert int(sim.numTotalXPBD.item()) == s.numTotalXPBD > 0


def _caving():
    import torch

    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.engine import sort_particles
    dev = torch.device("cuda", 0)
    sim, mpm, xpbd = domains.build(domains.caving_block(), device=dev)
    sort_particles(sim, mpm, xpbd)
    g = torch.Generator(device=dev).manual_seed(5)
    xp = torch.rand(sim.nPoints, generator=g, device=dev) < 0.35
    sim.materialLabel.copy_(torch.where(xp, 2, sim.materialLabel))
    return sim, mpm, xpbd


def test_persistent_step_caving_block():
    """Two XPBD steps of the caving block with 35 % XPBD particles."""
    a, b, made = _run_both(_caving, 2)
    assert made == 2
    assert a["counts"][0] > 100_000
    _assert_same(a, b)


def _tunnel_ring():
    import torch

    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.engine import sort_particles
    dev = torch.device("cuda", 0)
    sim, mpm, xpbd = domains.build(domains.tunnel(), device=dev)
    sort_particles(sim, mpm, xpbd)
    x = sim.particle_x
    r = torch.sqrt((x[:, 0] - 50.0) ** 2 + (x[:, 2] - 50.0) ** 2)  # the tunnel's axis (x, z) = (50, 50) m
    ring = r < 11.0
    sim.materialLabel.copy_(torch.where(ring, 2, sim.materialLabel))
    return sim, mpm, xpbd


def test_persistent_step_tunnel():
    """One XPBD step of the 3,873,600-particle tunnel with a 1 m ring of XPBD
    particles at the tunnel wall: more sort tiles than cooperative CTAs."""
    a, b, made = _run_both(_tunnel_ring, 1)
    assert made == 1
    assert a["counts"][0] > 1000
    _assert_same(a, b)


@pytest.mark.parametrize("over", [{"xpbd_iterations": 0}, {"xpbd_iterations": 1, "swellingRatio": 0.0}])
def test_persistent_step_edge_parameters(over):
    """No Jacobi iteration at all (the step is hash, integrate, sleep and
    impulses only), and one iteration without swelling: both forms and the
    oracle agree bit for bit."""
    import torch

    from mpmwarpydw_b200.utils import simulationRoutines as S
    a, b, made = _run_both(lambda: xpbd_scene(seed=8, lock=1, **over), 1)
    assert made == 1
    _assert_same(a, b)
    sim, mpm, xpbd = xpbd_scene(seed=8, lock=1, **over)
    s = to_oracle(sim, mpm, xpbd)
    S.xpbdSimulationStep(sim, mpm, xpbd, "cuda:0")
    torch.cuda.synchronize()
    orc.xpbd_step(oracle("f32"), s)
    g = gpu_fields(sim, mpm, xpbd)
    for k in KEYS:
        assert np.array_equal(g[k], getattr(s, k)), (k, rel_err(g[k], getattr(s, k)))
