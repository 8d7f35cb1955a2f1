"""The batched sweep on one GPU: scenes stepped together through one captured
CUDA graph (per-scene streams) equal the same scenes stepped one by one."""
import numpy as np
import pytest

from tests.harness import rel_err

pytestmark = pytest.mark.gpu


def _scenes():
    from mpmwarpydw_b200 import domains
    return [domains.block_collapse(n_side=s, spacing=0.25, jitter=0.025, seed=40 + s, box=6.0, dx=0.5, cohesion=c)
            for s, c in ((12, 2e5), (16, 1e6), (20, 5e5))]


def test_batch_graph_equals_scenes_one_by_one():
    import torch

    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.engine import sort_particles
    from mpmwarpydw_b200.sweep import SceneBatch
    from mpmwarpydw_b200.utils.simulationRoutines import run_mpm_substeps
    scenes = _scenes()
    b = SceneBatch(scenes)
    b.capture(5)          # eager warm-up (5 substeps) + capture
    b.replay()            # 5 more
    torch.cuda.synchronize()
    for i, d in enumerate(scenes):
        sim, mpm, xpbd = domains.build(d, device="cuda:0")
        sort_particles(sim, mpm, xpbd)
        run_mpm_substeps(sim, mpm, xpbd, 5)
        run_mpm_substeps(sim, mpm, xpbd, 5)
        torch.cuda.synchronize()
        bs, bm, _ = b.states[i]
        assert np.array_equal(sim.materialLabel.cpu().numpy(), bs.materialLabel.cpu().numpy())
        for a, c in ((sim.particle_x, bs.particle_x), (sim.particle_v, bs.particle_v), (mpm.particle_F, bm.particle_F)):
            assert rel_err(a.cpu().numpy(), c.cpu().numpy()) <= 1e-5
    res = b.results()
    assert [r.particles for r in res] == [d.n for d in scenes]


def test_concatenated_batch_equals_scenes_one_by_one():
    """One launch per kernel over the concatenated scenes (mpmw_batch_run_substeps,
    eager and graph-replayed) gives each scene the state of stepping it alone."""
    import torch

    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.engine import sort_particles
    from mpmwarpydw_b200.sweep import ConcatBatch
    from mpmwarpydw_b200.utils.simulationRoutines import run_mpm_substeps
    scenes = _scenes()
    b = ConcatBatch(scenes)
    assert all(o % 256 == 0 for o in b.offsets) and b.offsets[-1] == b.total
    b.step(4)             # eager, one launch per kernel
    b.groups = 2          # two scene ranges on two streams from here on
    b.capture(3)          # eager warm-up (3 substeps) + capture
    b.replay()            # 3 more: 10 in all
    torch.cuda.synchronize()
    from mpmwarpydw_b200.bind import read_status
    assert read_status("cuda:0") == 0
    b.sync_scenes()
    for i, d in enumerate(scenes):
        sim, mpm, xpbd = domains.build(d, device="cuda:0")
        sort_particles(sim, mpm, xpbd)
        for k in (4, 3, 3):
            run_mpm_substeps(sim, mpm, xpbd, k)
        torch.cuda.synchronize()
        bs, bm, _ = b.states[i]
        assert np.array_equal(sim.materialLabel.cpu().numpy(), bs.materialLabel.cpu().numpy())
        for a, c in ((sim.particle_x, bs.particle_x), (sim.particle_v, bs.particle_v), (mpm.particle_F, bm.particle_F),
                     (mpm.particle_C, bm.particle_C), (mpm.particle_stress, bm.particle_stress)):
            assert rel_err(a.cpu().numpy(), c.cpu().numpy()) <= 1e-5
        # the padding stays inactive and untouched
        pad = b.fields["active"][b.offsets[i] + b.counts[i]:b.offsets[i + 1]]
        assert int(pad.abs().sum().item()) == 0
    res = b.results()
    assert [r.particles for r in res] == [d.n for d in scenes]


def test_batch_options_and_tuner():
    """Every launch option the tuner searches (grid tile by TMA or L1 gathers,
    read-ahead by bulk copies or plain loads) gives the same scenes (to the
    scatter's atomic-order noise); the tuner keeps the configuration it timed
    fastest and the batch then still steps correctly."""
    import torch

    from mpmwarpydw_b200.sweep import ConcatBatch
    scenes = _scenes()
    ref = None
    for opts in ((True, True), (False, True), (True, False), (False, False)):
        b = ConcatBatch(scenes)
        b.set_options(*opts)
        b.step(6)
        torch.cuda.synchronize()
        x = b.fields["x"].cpu().numpy()
        if ref is None:
            ref = x
        else:
            assert rel_err(x, ref) <= 1e-5, opts
    b = ConcatBatch(scenes)
    g = b.tune(2, reuse=False)
    assert len(b.tuning) >= 5 and b.tuning[(g, b.options)] == max(b.tuning.values())
    b.step(3)
    torch.cuda.synchronize()
    from mpmwarpydw_b200.bind import read_status
    assert read_status("cuda:0") == 0
