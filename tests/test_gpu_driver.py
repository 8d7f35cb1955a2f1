"""The runMPMYDW driver on a synthetic block collapse: a big step runs to
nSteps with XPBD steps on the driver's counters, saves its output as the
reference's .vtp/.vti files, reading the residual back every 10 substeps
(fused substeps in between) gives the same state as reading it every substep
(the reference's loop), and a run restarted from a big step's checkpoint
continues as the uninterrupted run does."""
import glob

import numpy as np
import pytest

from tests.harness import rel_err

pytestmark = pytest.mark.gpu


def _args(tmp, **over):
    from mpmwarpydw_b200.utils.getArgs import get_args
    argv = ["--domainFile", "synthetic:block_collapse", "--bigSteps", "1", "--bigStepDuration", "0.003",
            "--xpbdOnlyDuration", "0.001", "--saveFlag", "1", "--outputFolder", str(tmp), "--render_interval", "0.001"]
    a = get_args(argv, verbose=False)
    for k, v in over.items():
        setattr(a, k, v)
    return a


def test_driver_check_interval_matches_per_substep_checks(tmp_path):
    import torch

    from mpmwarpydw_b200.runMPMYDW import run
    a1 = _args(tmp_path / "a")
    s1, m1, x1, saved1 = run(a1, check_interval=1, verbose=False)
    a2 = _args(tmp_path / "b")
    s2, m2, x2, saved2 = run(a2, check_interval=10, verbose=False)
    torch.cuda.synchronize()
    assert s1.nPoints == 64000
    # the big step's checkpoint and its last regular save can share a time and so a file name
    # (as in the reference, whose names hold the big step, counter and time)
    assert len(saved1) >= 2 and len(glob.glob(str(tmp_path / "a" / "*_particles.vtp"))) == len(set(saved1))
    assert len(glob.glob(str(tmp_path / "a" / "*_grid.vti"))) == len(set(saved1))
    assert np.array_equal(s1.materialLabel.cpu().numpy(), s2.materialLabel.cpu().numpy())
    assert rel_err(s1.particle_x.cpu().numpy(), s2.particle_x.cpu().numpy()) <= 1e-5
    assert rel_err(m1.particle_F.cpu().numpy(), m2.particle_F.cpu().numpy()) <= 1e-5


def test_driver_resort_interval_matches_no_resort(tmp_path):
    """Re-sorting the particles into block order every 10 substeps during the
    big step gives the same state, in input order, as sorting only at set-up
    (to the atomic-order noise of the scatter)."""
    import torch

    from mpmwarpydw_b200.engine import original_order
    from mpmwarpydw_b200.runMPMYDW import run
    s1, m1, _, _ = run(_args(tmp_path / "a", saveFlag=0), check_interval=5, verbose=False)
    s2, m2, _, _ = run(_args(tmp_path / "b", saveFlag=0), check_interval=5, verbose=False, resort_interval=10)
    torch.cuda.synchronize()
    o = lambda s, t: original_order(s, t).cpu().numpy()  # noqa: E731
    assert np.array_equal(o(s1, s1.materialLabel), o(s2, s2.materialLabel))
    assert rel_err(o(s2, s2.particle_x), o(s1, s1.particle_x)) <= 1e-5
    assert rel_err(o(s2, m2.particle_F), o(s1, m1.particle_F)) <= 1e-5


def test_driver_restart_from_checkpoint_matches_continuous_run(tmp_path):
    """Two big steps in one run, against one big step, its checkpoint, and a
    second run restarted from that checkpoint (runMPMYDW.py:498-576): the same
    particles in input order after the second big step.  A restart starts the
    next substep's return map from F_trial = F, as the reference's restart
    does, where the uninterrupted run has the last G2P's F_trial (one
    dt grad v F apart), so positions and F agree to 1e-4, not to atomic-order
    noise."""
    import torch

    from mpmwarpydw_b200.engine import original_order
    from mpmwarpydw_b200.runMPMYDW import run
    over = dict(bigSteps=2, render_interval=1.0)
    s1, m1, _, saved1 = run(_args(tmp_path / "a", **over), check_interval=5, verbose=False)
    s2, _, _, saved2 = run(_args(tmp_path / "b", **over), check_interval=5, verbose=False, max_big_steps=1)
    ckpt = [p for p in saved2 if "sim_step_0000" in p]
    assert ckpt, saved2
    s3, m3, _, _ = run(_args(tmp_path / "c", restart=ckpt[-1], **over), check_interval=5, verbose=False)
    torch.cuda.synchronize()
    o = lambda s, t: original_order(s, t).cpu().numpy()  # noqa: E731
    assert abs(s3.t - s1.t) <= 1e-9 * max(1.0, abs(s1.t))
    assert np.array_equal(o(s1, s1.materialLabel), o(s3, s3.materialLabel))
    assert rel_err(o(s3, s3.particle_x), o(s1, s1.particle_x)) <= 1e-4
    assert rel_err(o(s3, m3.particle_F), o(s1, m1.particle_F)) <= 1e-4
