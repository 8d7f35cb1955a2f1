"""The phase-1 loop with its stop test on the device (mpmw_loop_*): the same
decisions, counters and state as the driver's host-side check after every
chunk of fused substeps, and the driver gives the same result either way."""
import numpy as np
import pytest

from tests.harness import rel_err

pytestmark = pytest.mark.gpu


def _scene():
    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.engine import sort_particles
    d = domains.block_collapse(n_side=16, spacing=0.25, jitter=0.025, seed=7, box=6.0, dx=0.5, cohesion=2e5)
    sim, mpm, xpbd = domains.build(d, device="cuda:0")
    sort_particles(sim, mpm, xpbd)
    return sim, mpm, xpbd


def _host_loop(chunk, n_steps, threshold, stall_threshold, stall_steps, min_steps, segment):
    """The driver's check (PhaseOneMonitor) after every chunk, on the host."""
    from mpmwarpydw_b200.runMPMYDW import PhaseOneMonitor, _stats
    from mpmwarpydw_b200.utils.simulationRoutines import run_mpm_substeps
    sim, mpm, xpbd = _scene()
    mon = PhaseOneMonitor(n_steps, threshold, stall_threshold, stall_steps, min_steps)
    mon.prev_damage = _stats(sim, mpm)[1]
    ran = 0
    while mon.running() and ran + chunk <= segment:
        run_mpm_substeps(sim, mpm, xpbd, chunk)
        ran += chunk
        r, d, _ = _stats(sim, mpm)
        if not mon.update(chunk, r, d):
            break
    return mon, (sim, mpm, xpbd)


def _device_loop(chunk, n_steps, threshold, stall_threshold, stall_steps, min_steps, segment):
    from mpmwarpydw_b200.engine import DeviceLoop
    from mpmwarpydw_b200.runMPMYDW import _stats
    sim, mpm, xpbd = _scene()
    loop = DeviceLoop(sim, mpm, xpbd, chunk, n_steps, threshold, stall_threshold, stall_steps, min_steps)
    st = loop.run(0, 0, 1e10, _stats(sim, mpm)[1], segment)
    loop.close()
    return st, (sim, mpm, xpbd)


@pytest.mark.parametrize("case", [
    # below the initial residual (1e10, as the reference starts), above any real one
    dict(chunk=4, n_steps=40, threshold=1e9, stall_threshold=-1e30, stall_steps=10 ** 9, min_steps=0, segment=40),
    dict(chunk=4, n_steps=40, threshold=0.0, stall_threshold=-1e30, stall_steps=10 ** 9, min_steps=0, segment=40),
    dict(chunk=4, n_steps=40, threshold=0.0, stall_threshold=-1e30, stall_steps=10 ** 9, min_steps=0, segment=14),
    dict(chunk=5, n_steps=60, threshold=0.0, stall_threshold=1e30, stall_steps=10, min_steps=0, segment=60),
    dict(chunk=3, n_steps=30, threshold=1e9, stall_threshold=-1e30, stall_steps=10 ** 9, min_steps=12, segment=30),
], ids=["residual-stop", "to-n_steps", "segment-budget", "damage-stall", "min-steps"])
def test_device_decisions_match_the_host_check(case):
    import torch
    mon, (s1, m1, _) = _host_loop(**case)
    st, (s2, m2, _) = _device_loop(**case)
    torch.cuda.synchronize()
    assert st.counter == mon.counter
    assert st.stall == mon.stall and bool(st.stopped_early) == mon.stopped_early
    # the residual is a sum over the state, which FP32 atomics leave equal to ~1e-5
    assert st.residual == pytest.approx(mon.residual, rel=1e-4, abs=1e-12)
    assert np.array_equal(s1.materialLabel.cpu().numpy(), s2.materialLabel.cpu().numpy())
    assert rel_err(s1.particle_x.cpu().numpy(), s2.particle_x.cpu().numpy()) <= 1e-5
    assert rel_err(m1.particle_F.cpu().numpy(), m2.particle_F.cpu().numpy()) <= 1e-5


def test_driver_device_loop_matches_host_checks(tmp_path):
    import torch

    from mpmwarpydw_b200.runMPMYDW import run
    from mpmwarpydw_b200.utils.getArgs import get_args
    argv = ["--domainFile", "synthetic:block_collapse", "--bigSteps", "1", "--bigStepDuration", "0.003",
            "--xpbdOnlyDuration", "0.001", "--saveFlag", "0", "--outputFolder", str(tmp_path)]
    s1, m1, _, _ = run(get_args(argv, verbose=False), check_interval=5, verbose=False)
    s2, m2, _, _ = run(get_args(argv, verbose=False), check_interval=5, verbose=False, device_loop=True)
    torch.cuda.synchronize()
    assert s1.t == pytest.approx(s2.t)
    assert np.array_equal(s1.materialLabel.cpu().numpy(), s2.materialLabel.cpu().numpy())
    assert rel_err(s1.particle_x.cpu().numpy(), s2.particle_x.cpu().numpy()) <= 1e-5
    assert rel_err(m1.particle_F.cpu().numpy(), m2.particle_F.cpu().numpy()) <= 1e-5


def test_driver_phase_loop_crosses_xpbd_steps_and_pulse_end(tmp_path):
    """The whole of phase 1 in one device-loop launch (mpmw_phase_loop_*): the
    XPBD step every 5 substeps and the end of a 2x gravity pulse after 12
    substeps happen inside the graph, and phase 2's XPBD-only steps run as
    their own device loop (mpmw_xpbd_loop_*).  The final state equals the host
    path's (the same substeps, XPBD steps and gravities by counter) to the
    scatter's atomic-order noise."""
    import torch

    from mpmwarpydw_b200.engine import original_order
    from mpmwarpydw_b200.runMPMYDW import run
    from mpmwarpydw_b200.utils.getArgs import get_args
    from mpmwarpydw_b200 import domains
    d = domains.block_collapse(n_side=20, spacing=0.25, seed=8)
    dom = str(tmp_path / "block.npz")
    np.savez(dom, x=d.x.T, particle_volume=d.vol)
    # the domain file carries geometry only, so these flags set the scene
    argv = ["--domainFile", dom, "--bigSteps", "1", "--bigStepDuration", "0.004", "--dt", "1e-4",
            "--xpbdOnlyDuration", "0.0015", "--saveFlag", "0", "--outputFolder", str(tmp_path),
            "--dtxpbd", "5e-4", "--gravity_pulse_duration", "0.0012", "--gravity_pulse_factor", "2.0",
            "--ys", "2e4", "--gravity", "-9.81"]
    a1, a2 = get_args(argv, verbose=False), get_args(argv, verbose=False)
    s1, m1, _, _ = run(a1, check_interval=5, verbose=False)
    s2, m2, _, _ = run(a2, check_interval=5, verbose=False, device_loop=True)
    torch.cuda.synchronize()
    assert s1.mpmStepsPerXpbdStep == 5 and s1.nSteps == 40
    assert s1.t == pytest.approx(s2.t)
    o = lambda s, t: original_order(s, t).cpu().numpy()  # noqa: E731
    assert np.array_equal(o(s1, s1.materialLabel), o(s2, s2.materialLabel))
    assert rel_err(o(s2, s2.particle_x), o(s1, s1.particle_x)) <= 1e-5
    assert rel_err(o(s2, s2.particle_v), o(s1, s1.particle_v)) <= 1e-4
    assert rel_err(o(s2, m2.particle_F), o(s1, m1.particle_F)) <= 1e-5
