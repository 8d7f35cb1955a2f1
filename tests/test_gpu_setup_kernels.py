"""The set-up, end-of-step and statistics kernels against the oracle, through the
reference-named Python surface (utils.mpmRoutines / utils.simulationRoutines),
which calls the C ABI:

  compute_mu_lam_bulk_from_E_nu         utils/mpmRoutines.py:206-226
  initialize_geostatic_F (+ planestrain) utils/mpmRoutines.py:51-124, :127-203
  deactivate_and_teleport_xpbd_below_datum  utils/mpmRoutines.py:1446-1475
  creep_by_damage_with_baseline         utils/mpmRoutines.py:3-21
  the per-step reductions               utils/simulationRoutines.py:538-675
"""
import numpy as np
import pytest

from tests.harness import oracle, rel_err

pytestmark = pytest.mark.gpu


def _t(a, dtype=None):
    import torch
    return torch.as_tensor(np.ascontiguousarray(a, dtype=dtype), device="cuda:0")


def test_mu_lam_bulk_matches_oracle():
    """Lame constants and bulk modulus from E and nu: within 2 ulp of the FP32
    oracle (one division each) and 1e-6 of FP64."""
    import torch

    from mpmwarpydw_b200.utils import mpmRoutines as M
    rng = np.random.default_rng(1)
    n = 100_003
    E = (1e9 * 50.0 ** rng.random(n)).astype(np.float32)
    nu = rng.uniform(0.0, 0.45, n).astype(np.float32)
    mu, lam, bulk = (torch.zeros(n, device="cuda:0") for _ in range(3))
    M.compute_mu_lam_bulk_from_E_nu(_t(E), _t(nu), mu, lam, bulk)
    torch.cuda.synchronize()
    r32 = oracle("f32").mu_lam_bulk(E, nu)
    r64 = oracle("f64").mu_lam_bulk(E.astype(np.float64), nu.astype(np.float64))
    for g, a, b in zip((mu, lam, bulk), r32, r64):
        g = g.cpu().numpy()
        assert np.all(np.abs(g - a) <= 2 * np.spacing(np.abs(a).astype(np.float32)))
        assert rel_err(g, b) <= 1e-6


@pytest.mark.parametrize("planestrain", [False, True])
def test_geostatic_F_matches_oracle(planestrain):
    """Geostatic pre-stress F (K0 = 0.5, gravity 9.81, density 2600, z_top the
    highest particle) on a tunnel slab: per entry within 1e-6 of FP64, or equal
    to the FP32 oracle to 4 ulp of 1."""
    import torch

    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.utils import mpmRoutines as M
    d = domains.tunnel(nx=60, ny=20, nz=60)
    x = d.x.astype(np.float32)
    n = x.shape[0]
    rng = np.random.default_rng(2)
    E = (20e9 * np.exp(0.2 * rng.standard_normal(n))).astype(np.float32)
    nu = rng.uniform(0.15, 0.35, n).astype(np.float32)
    o32, o64 = oracle("f32"), oracle("f64")
    mu, lam, _ = o32.mu_lam_bulk(E, nu)
    dens = np.full(n, 2600.0, np.float32)
    z_top = float(x[:, 2].max())
    F = torch.zeros(n, 3, 3, device="cuda:0")
    fn = M.initialize_geostatic_F_planestrain if planestrain else M.initialize_geostatic_F
    fn(_t(x), F, _t(mu), _t(lam), _t(dens), 9.81, z_top, 0.5)
    torch.cuda.synchronize()
    F32 = np.zeros((n, 3, 3), np.float32)
    o32.geostatic_F(x, F32, mu, lam, dens, 9.81, z_top, 0.5, planestrain=planestrain)
    F64 = np.zeros((n, 3, 3), np.float64)
    o64.geostatic_F(x.astype(np.float64), F64, mu.astype(np.float64), lam.astype(np.float64),
                    dens.astype(np.float64), 9.81, z_top, 0.5, planestrain=planestrain)
    g = F.cpu().numpy()
    assert np.abs(g - np.eye(3)).max() > 1e-5          # a real pre-strain, not the identity
    ok = (np.abs(g - F64) <= 1e-6) | (np.abs(g - F32) <= 4 * 2.0 ** -23)
    assert ok.all(), int((~ok).sum())


def test_teleport_matches_oracle():
    """XPBD particles below the datum are deactivated, moved down by the
    teleport distance and stopped; nothing else changes (bit-exact)."""
    import torch

    from mpmwarpydw_b200.utils import mpmRoutines as M
    rng = np.random.default_rng(3)
    n = 50_000
    x = rng.uniform(-5, 5, (n, 3)).astype(np.float32)
    v = rng.normal(0, 1, (n, 3)).astype(np.float32)
    act = (rng.random(n) < 0.9).astype(np.int32)
    mat = rng.choice([0, 1, 2], n, p=[0.2, 0.4, 0.4]).astype(np.int32)
    xg, vg, ag, mg = _t(x), _t(v), _t(act), _t(mat)
    M.deactivate_and_teleport_xpbd_below_datum(xg, vg, ag, mg, -1.5, 20.0)
    torch.cuda.synchronize()
    o = oracle("f32")
    xo, vo, ao = x.copy(), v.copy(), act.copy()
    o.deactivate_and_teleport_xpbd_below_datum(xo, vo, ao, mat, -1.5, 20.0)
    assert int((ao != act).sum()) > 1000
    assert np.array_equal(ag.cpu().numpy(), ao)
    assert np.array_equal(xg.cpu().numpy(), xo)
    assert np.array_equal(vg.cpu().numpy(), vo)
    assert np.array_equal(mg.cpu().numpy(), mat)


def test_creep_matches_oracle():
    """Damage-driven creep of the yield stress of MPM particles: each within
    4 ulp of the FP32 oracle (powf may differ by an ulp) and never negative."""
    import torch

    from mpmwarpydw_b200.utils import mpmRoutines as M
    rng = np.random.default_rng(4)
    n = 50_000
    mat = rng.choice([0, 1, 2], n, p=[0.3, 0.5, 0.2]).astype(np.int32)
    D = rng.random(n).astype(np.float32)
    ys = (1e6 * rng.random(n)).astype(np.float32)
    base = (1e6 * rng.random(n)).astype(np.float32)
    ys[:100], base[:100] = 1.0, 1e6         # decays by more than it has: clamped at 0
    yg = _t(ys)
    M.creep_by_damage_with_baseline(_t(mat), _t(D), yg, _t(base), 1e-3, 0.05, 2.0, 3.0)
    torch.cuda.synchronize()
    yo = ys.copy()
    oracle("f32").creep_by_damage_with_baseline(mat, D, yo, base, 1e-3, 0.05, 2.0, 3.0)
    g = yg.cpu().numpy()
    assert (g >= 0).all() and (g[:100][mat[:100] <= 1] == 0).all()
    assert np.array_equal(g[mat > 1], ys[mat > 1])
    assert np.all(np.abs(g - yo) <= 4 * np.spacing(np.maximum(np.abs(yo), np.float32(1.0))))
    assert int((g != ys).sum()) > 10000


@pytest.mark.parametrize("n", [0, 1, 1000, 2_000_003])
def test_step_stats_match_oracle(n):
    """The per-step reductions (velocityConvergence, countActiveParticles,
    countParticlesByType, compute_mean_gpu's sum) in one GPU pass, accumulated
    in FP32: counts exact, sums within 1e-5 of the FP64 oracle (the
    reference itself sums these with FP32 atomics)."""
    import torch

    from mpmwarpydw_b200.utils import simulationRoutines as S
    rng = np.random.default_rng(5 + n)
    v = rng.normal(0, 2.0, (n, 3)).astype(np.float32)
    r = rng.uniform(0.05, 0.2, n).astype(np.float32)
    D = rng.random(n).astype(np.float32)
    act = (rng.random(n) < 0.8).astype(np.int32)
    mat = rng.choice([0, 1, 2], n, p=[0.2, 0.5, 0.3]).astype(np.int32)

    class _Sim:  # the storage attributes step_stats reads (as a SimState holds them)
        pass
    sim = _Sim()
    sim.device = torch.device("cuda:0")
    sim.nPoints = n
    sim._s_particle_v = _t(v.T.copy())
    sim._s_particle_radius, sim._s_activeLabel, sim._s_materialLabel = _t(r), _t(act, np.int32), _t(mat, np.int32)

    class _Mpm:
        pass
    mpm = _Mpm()
    mpm._s_particle_damage = _t(D)
    out = S.step_stats(sim, mpm).cpu().numpy()
    ref = oracle("f64").stats(act, mat, v.astype(np.float64), r.astype(np.float64), D.astype(np.float64))
    assert np.array_equal(out[[1, 3, 4, 5, 6]], ref[[1, 3, 4, 5, 6]])
    for k in (0, 2):
        assert abs(out[k] - ref[k]) <= 1e-5 * abs(ref[k]) + 1e-30, (k, out[k], ref[k])
