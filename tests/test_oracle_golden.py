"""The oracle against golden vectors from the reference itself: the
reference's mpmSimulationStep / xpbdSimulationStep source executed in float64
(tests/golden/gen_golden.py).  The FP64 oracle must agree to 1e-9 of each
array's magnitude with exactly equal labels and counts; the FP32 oracle to its
rounding floor."""
import numpy as np
import pytest

from oracle import oracle as orc
from tests.golden_io import MPM_FIXTURES, XPBD_FIXTURES, array_rel, load
from tests.harness import oracle

MPM_FIELDS = ("particle_x", "particle_v", "particle_C", "particle_F", "particle_F_trial", "particle_stress",
              "particle_accumulated_strain", "particle_damage", "particle_cov", "ys", "mu", "lam", "alpha",
              "grid_m", "grid_v_in", "grid_v_out", "particle_x_initial_xpbd", "particle_v_initial_xpbd",
              "cell_div_v_weighted", "cell_vol_sum")
XPBD_FIELDS = ("particle_x", "particle_v", "particle_x_integrated", "particle_v_integrated", "particle_delta",
               "particle_x_deltaInt", "particle_v_deltaInt", "particle_v_before_contact", "particle_cumDist_xpbd",
               "particle_radius")


@pytest.mark.parametrize("name", MPM_FIXTURES)
def test_fp64_oracle_mpm_step_matches_reference(name):
    s, exp = load(name)
    orc.mpm_step(oracle("f64"), s)
    assert np.array_equal(s.materialLabel, exp["materialLabel"])
    for k in MPM_FIELDS:
        got = getattr(s, k).reshape(exp[k].shape)
        assert array_rel(got, exp[k]) <= 1e-9, (k, array_rel(got, exp[k]))


@pytest.mark.parametrize("name", XPBD_FIXTURES)
def test_fp64_oracle_xpbd_step_matches_reference(name):
    s, exp = load(name)
    orc.xpbd_step(oracle("f64"), s)
    assert np.array_equal(s.materialLabel, exp["materialLabel"])
    assert s.numTotalXPBD == int(exp["numTotalXPBD"][0]) and s.numSleepingXPBD == int(exp["numSleepingXPBD"][0])
    for k in XPBD_FIELDS:
        got = getattr(s, k).reshape(exp[k].shape)
        assert array_rel(got, exp[k]) <= 1e-9, (k, array_rel(got, exp[k]))


@pytest.mark.parametrize("name", MPM_FIXTURES)
def test_fp32_oracle_mpm_step_near_reference(name):
    """FP32 restatement: positions and grid to 1e-5 of the array magnitude."""
    s, exp = load(name, np.float32)
    orc.mpm_step(oracle("f32"), s)
    for k in ("particle_x", "grid_m", "grid_v_out"):
        got = getattr(s, k).reshape(exp[k].shape)
        assert array_rel(got, exp[k]) <= 1e-5, (k, array_rel(got, exp[k]))
