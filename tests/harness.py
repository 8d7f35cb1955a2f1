"""Shared helpers of the parity tests: seeded small scenes on the GPU and their
oracle twins (numpy, reference layout), plus error norms."""
from __future__ import annotations

import numpy as np

from oracle.oracle import Oracle, OracleState


def rel_err(a, b, floor=0.0):
    """max |a-b| / max(max|b|, floor) over the whole array."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, floor)
    if scale == 0.0:
        return float(np.max(np.abs(a - b))) if a.size else 0.0
    return float(np.max(np.abs(a - b))) / scale


def small_scene(seed=0, n_side=10, spacing=0.25, dx=0.5, plastic=True, labels=True, device="cuda:0", **over):
    """A perturbed block (n_side^3 particles) exercising elastic, plastic and
    phase-transition branches, mixed labels and nonzero v, C, F."""
    import torch

    from mpmwarpydw_b200 import domains

    d = domains.block_collapse(n_side=n_side, spacing=spacing, jitter=0.1 * spacing, seed=seed, dx=dx)
    d.overrides.update(dict(eta_shear=1e3, eta_bulk=2e3, rpic_damping=0.1, update_cov=1))
    d.overrides.update(over)
    sim, mpm, xpbd = domains.build(d, device=device)
    rng = np.random.default_rng(1000 + seed)
    n = sim.nPoints
    t = lambda a: torch.as_tensor(np.asarray(a, np.float32), device=device)  # noqa: E731
    sim.particle_v = t(rng.uniform(-0.2, 0.2, (n, 3)))
    mpm.particle_C = t(rng.normal(0, 0.05, (n, 3, 3)))
    Ft = np.eye(3)[None] + rng.normal(0, 2e-3 if plastic else 2e-5, (n, 3, 3))
    if plastic:
        # a few strongly deformed and a few inverted particles (clamp paths)
        k = max(1, n // 50)
        Ft[:k] = np.eye(3)[None] + rng.normal(0, 0.3, (k, 3, 3))
        Ft[k:2 * k, 2, 2] *= -1.0
    mpm.particle_F_trial = t(Ft)
    mpm.particle_F = t(np.eye(3)[None] + rng.normal(0, 1e-3, (n, 3, 3)))
    ys = rng.uniform(0.2e6, 20e6, n)
    if plastic:
        ys[rng.random(n) < 0.05] = -1.0
    mpm.ys = t(ys)
    mpm.particle_damage = t(np.where(rng.random(n) < 0.2, rng.uniform(0.9, 0.999, n), rng.uniform(0, 0.5, n)))
    mpm.strainCriteria = t(np.where(rng.random(n) < 0.1, 0.0, rng.uniform(1e-3, 0.05, n)))
    mpm.hardening = t(rng.uniform(0, 0.1, n))
    mpm.softening = t(rng.uniform(0, 0.1, n))
    mpm.particle_cov = t(rng.normal(0, 1e-3, 6 * n))
    if labels:
        ml = np.where(rng.random(n) < 0.15, 0, 1)
        ml[rng.random(n) < 0.05] = 2
        al = np.where(rng.random(n) < 0.05, 0, 1)
        sim.materialLabel = torch.as_tensor(ml.astype(np.int32), device=device)
        sim.activeLabel = torch.as_tensor(al.astype(np.int32), device=device)
    torch.cuda.synchronize()
    return sim, mpm, xpbd


def to_oracle(sim, mpm, xpbd, dtype=np.float32) -> OracleState:
    """Copy the GPU state into reference-layout numpy arrays for the oracle."""
    c = lambda t: np.ascontiguousarray(t.detach().cpu().numpy())  # noqa: E731
    f = lambda t: np.ascontiguousarray(c(t).astype(dtype))  # noqa: E731
    s = OracleState()
    s.particle_x, s.particle_v = f(sim.particle_x), f(sim.particle_v)
    s.particle_mass, s.particle_vol = f(sim.particle_mass), f(sim.particle_vol)
    s.particle_radius, s.particle_density = f(sim.particle_radius), f(sim.particle_density)
    s.materialLabel, s.activeLabel = c(sim.materialLabel).astype(np.int32), c(sim.activeLabel).astype(np.int32)
    s.particle_F, s.particle_F_trial = f(mpm.particle_F), f(mpm.particle_F_trial)
    s.particle_stress, s.particle_C = f(mpm.particle_stress), f(mpm.particle_C)
    s.particle_accumulated_strain, s.particle_damage = f(mpm.particle_accumulated_strain), f(mpm.particle_damage)
    s.particle_cov = f(mpm.particle_cov)
    for k in ("mu", "lam", "ys", "alpha", "hardening", "softening", "eta_shear", "eta_bulk", "strainCriteria"):
        setattr(s, k, f(getattr(mpm, k)))
    s.grid_m = f(mpm.grid_m)
    s.grid_v_in = f(mpm.grid_v_in)
    s.grid_v_out = f(mpm.grid_v_out)
    s.cell_div_v_weighted = f(mpm.cell_div_v_weighted)
    s.cell_vol_sum = f(mpm.cell_vol_sum)
    s.particle_x_initial_xpbd = f(xpbd.particle_x_initial_xpbd)
    s.particle_v_initial_xpbd = f(xpbd.particle_v_initial_xpbd)
    s.dx, s.invdx, s.dt = sim.dx, sim.invdx, sim.dt
    s.minBounds = np.asarray(sim.minBounds, dtype)
    s.gravity = np.asarray(sim.gravity, dtype)
    s.rpic_damping, s.grid_v_damping_scale = mpm.rpic_damping, mpm.grid_v_damping_scale
    s.boundaryCondition, s.boundFriction, s.boundRestitution = mpm.boundaryCondition, mpm.boundFriction, mpm.boundRestitution
    s.boundaryPadding = mpm.boundaryPadding
    s.update_cov, s.volumetric_locking_correction = mpm.update_cov, mpm.volumetric_locking_correction
    s.eff, s.constitutive_model = mpm.eff, mpm.constitutive_model
    # XPBD
    for k in ("particle_x_integrated", "particle_v_integrated", "particle_x_deltaInt", "particle_v_deltaInt",
              "particle_delta", "particle_v_before_contact"):
        setattr(s, k, f(getattr(xpbd, k)))
    s.particle_cumDist_xpbd = f(xpbd.particle_cumDist_xpbd)
    s.particleBaseRadius = f(xpbd.particleBaseRadius)
    s.particleMaxRadius = f(xpbd.particleMaxRadius)
    for k in ("xpbd_iterations", "xpbd_relaxation", "xpbd_mpm_coupling_strength", "mpm_contact_transition_lock",
              "dynamicParticleFriction", "staticParticleFriction", "staticVelocityThreshold", "particle_cohesion",
              "sleepThreshold", "particle_v_max", "swellingRatio", "swellingActivationFactor", "swellingMaxFactor",
              "max_radius"):
        setattr(s, k, getattr(xpbd, k))
    s.minBoundsXPBD = np.asarray(xpbd.minBoundsXPBD, dtype)
    s.maxBoundsXPBD = np.asarray(xpbd.maxBoundsXPBD, dtype)
    s.dtxpbd = sim.dtxpbd
    return s


def gpu_fields(sim, mpm, xpbd):
    c = lambda t: t.detach().cpu().numpy()  # noqa: E731
    return dict(particle_x=c(sim.particle_x), particle_v=c(sim.particle_v), particle_C=c(mpm.particle_C),
                particle_F=c(mpm.particle_F), particle_F_trial=c(mpm.particle_F_trial),
                particle_stress=c(mpm.particle_stress), particle_accumulated_strain=c(mpm.particle_accumulated_strain),
                particle_damage=c(mpm.particle_damage), materialLabel=c(sim.materialLabel), ys=c(mpm.ys),
                mu=c(mpm.mu), lam=c(mpm.lam), alpha=c(mpm.alpha), particle_cov=c(mpm.particle_cov),
                grid_m=c(mpm.grid_m), grid_v_in=c(mpm.grid_v_in), grid_v_out=c(mpm.grid_v_out),
                particle_x_initial_xpbd=c(xpbd.particle_x_initial_xpbd),
                particle_v_initial_xpbd=c(xpbd.particle_v_initial_xpbd),
                particle_x_integrated=c(xpbd.particle_x_integrated), particle_v_integrated=c(xpbd.particle_v_integrated),
                particle_x_deltaInt=c(xpbd.particle_x_deltaInt), particle_v_deltaInt=c(xpbd.particle_v_deltaInt),
                particle_delta=c(xpbd.particle_delta), particle_v_before_contact=c(xpbd.particle_v_before_contact),
                particle_cumDist_xpbd=c(xpbd.particle_cumDist_xpbd), particle_radius=c(sim.particle_radius),
                activeLabel=c(sim.activeLabel))


def xpbd_scene(seed=0, n_side=12, frac_xpbd=0.35, lock=1, device="cuda:0", **over):
    """A block where a fraction of particles are XPBD (label 2) with random
    velocities, some overlapping, plus MPM particles in contact with them."""
    import torch

    from mpmwarpydw_b200 import domains
    d = domains.block_collapse(n_side=n_side, spacing=0.25, jitter=0.05, seed=seed, dx=0.5)
    d.overrides.update(dict(dtxpbd=5e-4, mpm_contact_transition_lock=lock, particle_cohesion=0.02,
                            swellingRatio=0.2, staticVelocityThreshold=0.5, xpbd_iterations=4))
    d.overrides.update(over)
    sim, mpm, xpbd = domains.build(d, device=device)
    rng = np.random.default_rng(2000 + seed)
    n = sim.nPoints
    ml = np.ones(n, np.int32)
    ml[rng.random(n) < frac_xpbd] = 2
    ml[(ml == 1) & (rng.random(n) < 0.2)] = 0
    al = np.where(rng.random(n) < 0.03, 0, 1).astype(np.int32)
    sim.materialLabel = torch.as_tensor(ml, device=device)
    sim.activeLabel = torch.as_tensor(al, device=device)
    sim.particle_v = torch.as_tensor(rng.normal(0, 1.0, (n, 3)).astype(np.float32), device=device)
    r = sim.particle_radius.cpu().numpy() * rng.uniform(0.9, 1.6, n).astype(np.float32)
    sim.particle_radius = torch.as_tensor(r, device=device)
    # phase-change records of the XPBD particles (used by swelling)
    xin = sim.particle_x.cpu().numpy() - rng.normal(0, 0.05, (n, 3)).astype(np.float32)
    xpbd.particle_x_initial_xpbd = torch.as_tensor(np.where((ml == 2)[:, None], xin, 1e6).astype(np.float32), device=device)
    torch.cuda.synchronize()
    return sim, mpm, xpbd


ULP1 = 2.0 ** -23  # spacing of FP32 numbers just above 1


def stress_parity_violation(g, s32, s64, twomu):
    """Largest per-particle violation (<= 1 passes) of the stress parity rule.

    A particle passes if its stress matches
      * the FP64 oracle: |d| <= 1e-5 |tau| + 1 Pa (tensor path: same mathematics,
        evaluated without near-identity rounding), or
      * the FP32 oracle: |d| <= 1e-5 |tau| + 16 * 2mu * 2^-23 (SVD path: the FP32
        oracle performs the same operations; logf/expf may differ by an ulp, and
        an ulp of F near identity is worth 2mu * 2^-23 of stress).
    ``twomu`` is the per-particle 2*mu (array)."""
    n = len(g)
    g = np.asarray(g, np.float64).reshape(n, -1)
    a = np.asarray(s32, np.float64).reshape(n, -1)
    b = np.asarray(s64, np.float64).reshape(n, -1)
    tm = np.broadcast_to(np.asarray(twomu, np.float64), (n,))
    e64 = np.abs(g - b).max(1) / (1e-5 * np.abs(b).max(1) + 1.0)
    e32 = np.abs(g - a).max(1) / (1e-5 * np.abs(a).max(1) + 16.0 * tm * ULP1 + 1e-30)
    v = np.minimum(e64, e32)
    return float(v.max()) if v.size else 0.0


def close_to_either(g, a, b, rtol=1e-4, atol=1e-7):
    """Per-particle: g matches a (FP32 oracle) or b (FP64 oracle)."""
    n = len(g)
    g = np.asarray(g, np.float64).reshape(n, -1)
    a = np.asarray(a, np.float64).reshape(n, -1)
    b = np.asarray(b, np.float64).reshape(n, -1)
    ok_a = (np.abs(g - a) <= rtol * np.abs(a) + atol).all(1)
    ok_b = (np.abs(g - b) <= rtol * np.abs(b) + atol).all(1)
    return bool((ok_a | ok_b).all()), int((~(ok_a | ok_b)).sum())


ORACLES = {}


def oracle(prec="f32"):
    if prec not in ORACLES:
        ORACLES[prec] = Oracle(prec)
    return ORACLES[prec]
