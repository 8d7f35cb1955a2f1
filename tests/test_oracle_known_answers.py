"""CPU checks of the oracle against known answers that follow from the
reference's formulas (no GPU).

  * SVD: reconstruction, proper rotations, ordering, sign convention;
  * elastic no-op: below yield the return map returns F_trial unchanged and
    the Kirchhoff stress of a diagonal F is 2 mu ln(F) + lam tr(ln F) I
    (utils/mpmRoutines.py:361,452-471);
  * geostatic F: the Kirchhoff stress of initialize_geostatic_F's F is the
    target geostatic stress (sigma_h, sigma_h, sigma_v) (mpmRoutines.py:51-124);
  * uniform translation through P2G -> grid -> G2P with no stress and no
    boundary contact is exact: v gains dt*g, C stays 0, F_trial = F
    (quadratic B-spline partition of unity and zero first moment);
  * P2G conserves mass.
"""
import numpy as np
import pytest

from oracle.oracle import OracleState
from tests.harness import oracle, rel_err


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_svd_properties(prec):
    o = oracle(prec)
    rng = np.random.default_rng(0)
    tol = 2e-6 if prec == "f32" else 1e-13
    for t in range(300):
        kind = t % 4
        if kind == 0:
            F = np.eye(3) + 1e-5 * rng.standard_normal((3, 3))
        elif kind == 1:
            F = rng.standard_normal((3, 3))
        elif kind == 2:
            Q, _ = np.linalg.qr(rng.standard_normal((3, 3)))
            F = Q @ np.diag(rng.uniform(0.5, 2.0, 3))
        else:
            F = np.diag(rng.uniform(0.5, 2.0, 3))
            F[2, 2] *= -1
        U, s, V = o.svd3(F.astype(o.dtype))
        U = U.astype(np.float64); V = V.astype(np.float64); s = s.astype(np.float64)
        assert np.abs(U @ np.diag(s) @ V.T - F).max() <= tol * max(1.0, np.abs(F).max()) * 10
        assert abs(np.linalg.det(U) - 1) < 1e-5 and abs(np.linalg.det(V) - 1) < 1e-5
        assert s[0] >= s[1] - tol and s[1] >= abs(s[2]) - tol
        assert np.sign(s[2]) == np.sign(np.linalg.det(F)) or abs(s[2]) < 1e-6


def _one_particle_state(o, F_trial, ys=1e20, mu=4e9, lam=4e9, damage=0.0, C=None):
    dt = o.dtype
    a = lambda v: np.ascontiguousarray(np.asarray(v, dt))  # noqa: E731
    s = OracleState()
    s.activeLabel = np.ones(1, np.int32); s.materialLabel = np.ones(1, np.int32)
    s.x = a(np.zeros((1, 3))); s.v = a(np.zeros((1, 3)))
    s.x_pc = a(np.zeros((1, 3))); s.v_pc = a(np.zeros((1, 3)))
    s.F = a(np.zeros((1, 3, 3))); s.Ft = a(np.asarray(F_trial).reshape(1, 3, 3))
    s.mu = a([mu]); s.lam = a([lam]); s.ys = a([ys]); s.H = a([0.0]); s.S = a([0.0]); s.rho = a([2650.0])
    s.sc = a([0.05]); s.eta_s = a([0.0]); s.eta_b = a([0.0]); s.C = a(np.zeros((1, 3, 3)) if C is None else C)
    s.stress = a(np.zeros((1, 3, 3))); s.acc = a([0.0]); s.D = a([damage]); s.alpha = a([0.2])
    return s


def _stress(o, s):
    o.compute_stress_from_F_trial(s.activeLabel, s.materialLabel, s.x, s.v, s.x_pc, s.v_pc, s.F, s.Ft, s.mu, s.lam,
                                  s.ys, s.H, s.S, s.rho, s.sc, 0.05, s.eta_s, s.eta_b, s.C, s.stress, s.acc, s.D, 1,
                                  s.alpha)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_elastic_noop_and_diagonal_kirchhoff(prec):
    o = oracle(prec)
    e = np.array([1e-3, -2e-3, 5e-4])
    s = _one_particle_state(o, np.diag(np.exp(e)))
    _stress(o, s)
    assert np.array_equal(s.F[0], s.Ft[0])                 # F_trial returned unchanged
    assert s.acc[0] == 0 and s.D[0] == 0 and s.materialLabel[0] == 1
    mu, lam = 4e9, 4e9
    expect = np.diag(2 * mu * e + lam * e.sum())
    tol = 1e-3 if prec == "f32" else 1e-10
    assert rel_err(s.stress[0], expect) < tol


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_geostatic_F_gives_target_stress(prec):
    o = oracle(prec)
    dt = o.dtype
    n = 5
    x = np.zeros((n, 3), dt); x[:, 2] = np.linspace(0, 40, n)
    F = np.zeros((n, 3, 3), dt)
    E, nu = 10e9, 0.25
    mu, lam, _ = o.mu_lam_bulk(np.full(n, E, dt), np.full(n, nu, dt))
    rho = np.full(n, 2600.0, dt)
    o.geostatic_F(x, F, mu, lam, rho, 9.81, 50.0, 0.5)
    depth = 50.0 - x[:, 2].astype(np.float64)
    sv = -2600.0 * 9.81 * depth
    sh = 0.5 * sv
    for p in range(n):
        s = _one_particle_state(o, F[p], mu=float(mu[p]), lam=float(lam[p]))
        _stress(o, s)
        expect = np.diag([sh[p], sh[p], sv[p]])
        tol = 2e-2 if prec == "f32" else 1e-9  # FP32: exp/log round trip of strains ~1e-4
        assert rel_err(s.stress[0], expect, floor=1e3) < tol, (p, s.stress[0], expect)


def _translation_state(o, n_side=4, spacing=0.25, dx=0.5, vel=(0.3, -0.2, 0.1)):
    dt = o.dtype
    rng = np.random.default_rng(3)
    g = (np.arange(n_side) + 0.5) * spacing + 3.0
    X = np.stack(np.meshgrid(g, g, g, indexing="ij"), -1).reshape(-1, 3) + rng.uniform(-0.05, 0.05, (n_side ** 3, 3))
    n = X.shape[0]
    s = OracleState()
    a = lambda v: np.ascontiguousarray(np.asarray(v, dt))  # noqa: E731
    s.activeLabel = np.ones(n, np.int32); s.materialLabel = np.ones(n, np.int32)
    s.particle_x = a(X); s.particle_v = a(np.tile(vel, (n, 1))); s.particle_C = a(np.zeros((n, 3, 3)))
    s.particle_stress = a(np.zeros((n, 3, 3))); s.particle_vol = a(np.full(n, spacing ** 3))
    s.particle_mass = a(np.full(n, 2650 * spacing ** 3))
    s.particle_F = a(np.tile(np.eye(3), (n, 1, 1))); s.particle_F_trial = a(np.zeros((n, 3, 3)))
    s.particle_cov = a(np.zeros(6 * n))
    dims = (20, 20, 20)
    s.grid_m = a(np.zeros(dims)); s.grid_v_in = a(np.zeros(dims + (3,))); s.grid_v_out = a(np.zeros(dims + (3,)))
    s.minBounds = a([0, 0, 0]); s.dx, s.invdx = dx, 1 / dx
    return s


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_uniform_translation_is_exact(prec):
    o = oracle(prec)
    s = _translation_state(o)
    g = np.array([0, 0, -9.81])
    dt = 1e-3
    st = o.p2g_apic_with_stress(s.activeLabel, s.materialLabel, s.particle_stress, s.particle_x, s.particle_v,
                                s.particle_C, s.particle_vol, s.particle_mass, s.dx, s.invdx, s.minBounds, 0.0,
                                s.grid_m, s.grid_v_in, dt)
    assert st == 0
    assert abs(s.grid_m.sum() - s.particle_mass.sum()) <= 1e-5 * s.particle_mass.sum()
    o.grid_normalization_and_gravity(s.grid_m, s.grid_v_in, s.grid_v_out, g.astype(o.dtype), dt)
    v0 = s.particle_v.copy()
    st = o.g2p(dt, s.activeLabel, s.materialLabel, s.particle_x, s.particle_v, s.particle_C, s.particle_F,
               s.particle_F_trial, s.particle_cov, s.invdx, s.grid_v_out, False, s.minBounds)
    assert st == 0
    tol = 1e-5 if prec == "f32" else 1e-12
    assert np.abs(s.particle_v - (v0 + dt * g)).max() < tol
    assert np.abs(s.particle_C).max() < tol * 10
    assert np.abs(s.particle_F_trial - np.eye(3)).max() < tol


def test_bc_last_face_wins_at_corners():
    """collideBounds writes from the entry velocity; at a corner node the later
    face (z after y after x) determines the result (mpmRoutines.py:956-993)."""
    o = oracle("f64")
    dims = (6, 6, 6)
    v = np.zeros(dims + (3,))
    v[0, 0, 0] = [-1.0, -2.0, -3.0]
    o.grid_bc(v, "friction", 0.0, 0.0, 1e-3, 9.81, 2)
    # z face wins: (coulomb(vx), coulomb(vy), 0) with mu = 0 -> (-1, -2, 0)
    assert np.allclose(v[0, 0, 0], [-1.0, -2.0, 0.0])


def test_hash_grid_restatement():
    """Cells, stable order and ranges of the restated wp.HashGrid."""
    o = oracle("f32")
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 8, (500, 3)).astype(np.float32)
    hg = o.hash_build(x, 1.0)
    cells = np.floor(x * np.float32(1.0)).astype(np.int64) + (1 << 20)
    h = (cells[:, 2] % 128) * 128 * 128 + (cells[:, 1] % 128) * 128 + cells[:, 0] % 128
    assert np.array_equal(hg.point_cells, h)
    assert np.array_equal(hg.point_ids, np.argsort(h, kind="stable"))
    for c in np.unique(h):
        ids = hg.point_ids[hg.cell_starts[c]:hg.cell_ends[c]]
        assert np.all(h[ids] == c) and np.all(np.diff(ids) > 0)


def test_surrogate_targets_encode_the_radial_return():
    """The network's targets (ln rho, ln(1 - rho), beta, sqrt(2/3)) decoded as
    the stress phase decodes them give the reference's principal-space return
    (utils/mpmRoutines.py:339-453) to FP64 rounding, over seeded plastic trials."""
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(7)
    checked = 0
    for _ in range(2000):
        mag = 10.0 ** rng.uniform(-6, -1)
        g = rng.standard_normal(3)
        e = np.sort(mag * g / np.linalg.norm(g))[::-1]
        E, nu = 1e9 * 50.0 ** rng.uniform(), rng.uniform(0.15, 0.35)
        mu, lam = E / (2 * (1 + nu)), E * nu / ((1 + nu) * (1 - 2 * nu))
        ys, D = 1e5 * 50.0 ** rng.uniform(), rng.uniform(0, 0.999)
        s = np.sin(np.radians(rng.uniform(20, 45)))
        alpha = 2 * s / (np.sqrt(3) * (3 - s))
        beta = 0.3 * alpha
        ref = M.dp_return_principal(e, mu, lam, ys, alpha, beta, D)
        tr = e.sum()
        if ref is None or (1 - D) * (ys - alpha * (2 * mu / 3 + lam) * tr) <= 0:
            continue
        y, e_ret, dacc = M.targets(e, mu, lam, ys, alpha, beta, D)
        if y[1] <= -12.0:
            continue
        assert np.allclose(e_ret, ref[0], rtol=0, atol=1e-12 * max(1.0, np.abs(e).max() / 1e-6) * 1e-6 + 1e-15)
        assert abs(dacc - ref[1]) <= 1e-9 * abs(ref[1]) + 1e-18
        assert y[2] == beta and abs(y[3] - np.sqrt(2 / 3)) == 0.0
        checked += 1
    assert checked > 500
