"""The CUDA path against the golden vectors of the reference itself (its
mpmSimulationStep / xpbdSimulationStep source executed in float64, written
by tests/golden/gen_golden.py), through the C ABI, one step from identical
inputs.  FP32 against FP64, so the rules are those of the FP64 comparisons in
test_gpu_mpm_parity.py: x, v, C, F_trial and the grid to 1e-5 of each array's
magnitude; stress per particle within 1e-5 |tau| + 16 * 2mu * 2^-23 (the stress
worth of a few ulps of F near identity); labels equal to the reference's;
XPBD positions and velocities to 1e-5."""
import numpy as np
import pytest

from tests.golden_io import MPM_FIXTURES, XPBD_FIXTURES, array_rel, gpu_states, load
from tests.harness import gpu_fields, stress_parity_violation

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", MPM_FIXTURES)
@pytest.mark.parametrize("mode", [0, 1])
def test_cuda_mpm_step_matches_reference(name, mode):
    import torch

    from mpmwarpydw_b200.utils import simulationRoutines as S
    sim, mpm, xpbd = gpu_states(name)
    mpm.stress_mode = mode
    s_in, exp = load(name)
    S.mpmSimulationStep(sim, mpm, xpbd, "cuda:0")
    torch.cuda.synchronize()
    g = gpu_fields(sim, mpm, xpbd)
    assert np.array_equal(g["materialLabel"], exp["materialLabel"])
    for k in ("particle_x", "particle_v", "particle_C", "particle_F_trial", "grid_m", "grid_v_out"):
        e = array_rel(g[k], exp[k].reshape(g[k].shape))
        assert e <= 1e-5, (k, e)
    twomu = 2.0 * np.asarray(s_in.mu, np.float64)
    ref = exp["particle_stress"].reshape(g["particle_stress"].shape)
    assert stress_parity_violation(g["particle_stress"], ref, ref, twomu) <= 1.0
    for k in ("particle_accumulated_strain", "particle_damage", "ys"):
        e = array_rel(g[k], exp[k])
        assert e <= 1e-4, (k, e)


@pytest.mark.parametrize("name", XPBD_FIXTURES)
def test_cuda_xpbd_step_matches_reference(name):
    import torch

    from mpmwarpydw_b200.utils import simulationRoutines as S
    sim, mpm, xpbd = gpu_states(name)
    _, exp = load(name)
    S.xpbdSimulationStep(sim, mpm, xpbd, "cuda:0")
    torch.cuda.synchronize()
    g = gpu_fields(sim, mpm, xpbd)
    assert np.array_equal(g["materialLabel"], exp["materialLabel"])
    assert int(sim.numTotalXPBD.item()) == int(exp["numTotalXPBD"][0])
    assert int(sim.numSleepingXPBD.item()) == int(exp["numSleepingXPBD"][0])
    for k in ("particle_x", "particle_v", "particle_radius"):
        e = array_rel(g[k], exp[k].reshape(g[k].shape))
        assert e <= 1e-5, (k, e)
