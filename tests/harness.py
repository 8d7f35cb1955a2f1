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
                particle_v_initial_xpbd=c(xpbd.particle_v_initial_xpbd))


def stress_either_err(g, s32, s64, floor_frac=1e-4):
    """Per-particle stress error of the AUTO stress mode: each particle must
    match the FP32 oracle (SVD path, same operations) or the FP64 oracle (the
    SVD-free elastic path, which is closer to FP64 than an FP32 SVD).  Returns
    the largest min(err32, err64) / scale over particles, scale = max(|s64_p|,
    floor_frac * max|s64|)."""
    g = np.asarray(g, np.float64).reshape(len(g), -1)
    a = np.asarray(s32, np.float64).reshape(len(g), -1)
    b = np.asarray(s64, np.float64).reshape(len(g), -1)
    scale = np.maximum(np.abs(b).max(1), floor_frac * np.abs(b).max())
    scale = np.where(scale > 0, scale, 1.0)
    e = np.minimum(np.abs(g - a).max(1), np.abs(g - b).max(1)) / scale
    return float(e.max()) if e.size else 0.0


ORACLES = {}


def oracle(prec="f32"):
    if prec not in ORACLES:
        ORACLES[prec] = Oracle(prec)
    return ORACLES[prec]
