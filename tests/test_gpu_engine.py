"""engine.SubstepGraph: k substeps captured once into a CUDA graph and
replayed give what the same substeps give as direct library calls (to the
atomic-order noise of the fused scatter)."""
import numpy as np
import pytest

from tests.harness import gpu_fields, rel_err, small_scene

pytestmark = pytest.mark.gpu


def test_substep_graph_replay_matches_direct_calls():
    import torch

    from mpmwarpydw_b200.engine import SubstepGraph
    from mpmwarpydw_b200.utils import simulationRoutines as S
    a = small_scene(seed=16)
    b = small_scene(seed=16)
    g = SubstepGraph(*a, k=3, warmup=True)   # the warm-up run is 3 substeps
    g.replay()
    g.replay()
    for _ in range(3):
        S.run_mpm_substeps(*b, 3)
    torch.cuda.synchronize()
    ga, gb = gpu_fields(*a), gpu_fields(*b)
    assert np.array_equal(ga["materialLabel"], gb["materialLabel"])
    for k, tol in (("particle_x", 1e-5), ("particle_v", 1e-4), ("particle_C", 1e-4), ("particle_F", 1e-5),
                   ("particle_stress", 1e-3)):
        assert rel_err(ga[k], gb[k]) <= tol, (k, rel_err(ga[k], gb[k]))
    assert float(np.abs(ga["particle_x"] - small_scene(seed=16)[0].particle_x.cpu().numpy()).max()) > 0
