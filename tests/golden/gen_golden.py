#!/usr/bin/env python
"""Generate the golden fixtures in tests/golden/ by executing the reference's own
kernel and orchestration source (MPMWarpYDW utils/simulationRoutines.py,
utils/mpmRoutines.py, utils/xpbdRoutines.py, utils/simStates.py) in float64 on
the CPU, through the Warp stand-in in fakewarp.py.

    python tests/golden/gen_golden.py --reference PATH     (or MPMW_REFERENCE=PATH)

Needs a checkout of the reference project (no default location); the fixtures it
writes are committed, so the tests never read the reference.  Each fixture is
one seeded scene: every input array (``in/<state>.<attribute>``), then the
arrays that one ``mpmSimulationStep`` or ``xpbdSimulationStep`` changed
(``out/<state>.<attribute>``).

Scenes (small: 216 particles, 10^3 grid nodes):
  mpm_friction    getArgs defaults: volumetric locking correction and
                  covariance update on, Coulomb-friction boundary, rpic 0.2;
                  elastic, plastic, transitioning, inverted and inactive particles
  mpm_restitution restitution boundary, grid damping 0.98, no VLC, no cov
  mpm_planestrain plane_strain_y boundary, rpic 0 (APIC)
  xpbd_lock       XPBD step with the contact-transition lock, 35 % XPBD particles
  xpbd_free       XPBD step without the lock, swelling active
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def load_reference(path):
    sys.path.insert(0, HERE)
    import fakewarp
    wp = fakewarp.install()
    sys.dont_write_bytecode = True  # the reference checkout may be read-only
    sys.path.insert(0, path)
    from utils import mpmRoutines, simStates, simulationRoutines, xpbdRoutines  # noqa: F401
    return wp, simStates, simulationRoutines, mpmRoutines


def default_args(**over):
    sys.path.insert(0, ROOT)
    from mpmwarpydw_b200.utils.getArgs import defaults
    a = defaults()
    for k, v in over.items():
        setattr(a, k, v)
    return a


def friction_alpha(phi):
    s = np.sin(np.radians(phi))
    return 2.0 * s / (np.sqrt(3.0) * (3.0 - s))


def build_scene(wp, SS, RM, seed, args, n_side=6, spacing=0.25, dx=0.5, xpbd_frac=0.0, lock_labels=False):
    rng = np.random.default_rng(seed)
    n = n_side ** 3
    ii = np.arange(n_side) + 0.5
    zz, yy, xx = np.meshgrid(ii, ii, ii, indexing="ij")
    x = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1) * spacing + 0.75
    x += rng.uniform(-0.1 * spacing, 0.1 * spacing, x.shape)
    minB = np.array([-1.0, -1.0, -1.0])
    dims = (10, 10, 10)  # grid spans [-1, 4) with dx 0.5
    sim = SS.SimState(args, n, device="cpu")
    mpm = SS.MPMState(args, n, dims, device="cpu")
    xp = SS.XPBDState(args, n, device="cpu")
    sim.particle_x = wp.array(x, dtype=wp.vec3)
    sim.particle_v = wp.array(rng.uniform(-0.2, 0.2, (n, 3)), dtype=wp.vec3)
    vol = np.full(n, spacing ** 3)
    sim.particle_vol = wp.array(vol, dtype=float)
    sim.particle_density = wp.array(np.full(n, args.density), dtype=float)
    sim.particle_mass = wp.array(vol * args.density, dtype=float)
    radius = np.full(n, spacing * 0.5) * rng.uniform(0.9, 1.4, n)
    sim.particle_radius = wp.array(radius, dtype=float)
    sim.minBounds = wp.vec3(*minB)
    sim.maxBounds = wp.vec3(*(minB + np.array(dims) * dx))
    sim.dx = dx
    sim.invdx = 1.0 / dx
    if xpbd_frac > 0:
        ml = np.ones(n, np.int64)
        ml[rng.random(n) < xpbd_frac] = 2
        ml[(ml == 1) & (rng.random(n) < 0.2)] = 0 if lock_labels else 1
    else:
        ml = np.where(rng.random(n) < 0.15, 0, 1)
        ml[rng.random(n) < 0.05] = 2
    al = np.where(rng.random(n) < 0.04, 0, 1)
    sim.materialLabel = wp.array(ml, dtype=wp.int32)
    sim.activeLabel = wp.array(al, dtype=wp.int32)
    # material (E, nu through the reference's own kernel)
    E = rng.uniform(0.5e9, 2e9, n)
    nu = np.full(n, 0.25)
    mpm.mu = wp.zeros(shape=n, dtype=float)
    mpm.lam = wp.zeros(shape=n, dtype=float)
    mpm.bulk = wp.zeros(shape=n, dtype=float)
    wp.launch(RM.compute_mu_lam_bulk_from_E_nu, dim=n,
              inputs=[wp.array(E, dtype=float), wp.array(nu, dtype=float), mpm.mu, mpm.lam, mpm.bulk])
    ys = rng.uniform(0.2e6, 20e6, n)
    ys[rng.random(n) < 0.05] = -1.0
    mpm.ys = wp.array(ys, dtype=float)
    mpm.ys_base = wp.array(ys.copy(), dtype=float)
    mpm.alpha = wp.array(np.full(n, friction_alpha(30.0)), dtype=float)
    mpm.hardening = wp.array(rng.uniform(0, 0.1, n), dtype=float)
    mpm.softening = wp.array(rng.uniform(0, 0.1, n), dtype=float)
    mpm.eta_shear = wp.array(np.full(n, 1e3), dtype=float)
    mpm.eta_bulk = wp.array(np.full(n, 2e3), dtype=float)
    mpm.strainCriteria = wp.array(np.where(rng.random(n) < 0.1, 0.0, rng.uniform(1e-3, 0.05, n)), dtype=float)
    mpm.boundaryPadding = 2
    # deformation state: mostly near identity, some strongly deformed, some inverted
    Ft = np.eye(3)[None] + rng.normal(0, 2e-3, (n, 3, 3))
    k = n // 40
    Ft[:k] = np.eye(3)[None] + rng.normal(0, 0.3, (k, 3, 3))
    Ft[k:2 * k, 2, 2] *= -1.0
    mpm.particle_F_trial = wp.array(Ft, dtype=wp.mat33)
    mpm.particle_F = wp.array(np.eye(3)[None] + rng.normal(0, 1e-3, (n, 3, 3)), dtype=wp.mat33)
    mpm.particle_C = wp.array(rng.normal(0, 0.05, (n, 3, 3)), dtype=wp.mat33)
    mpm.particle_damage = wp.array(np.where(rng.random(n) < 0.2, rng.uniform(0.9, 0.999, n),
                                            rng.uniform(0, 0.5, n)), dtype=float)
    mpm.particle_cov = wp.array(rng.normal(0, 1e-3, 6 * n), dtype=float)
    # XPBD fields
    xp.particleBaseRadius = wp.array(radius.copy(), dtype=float)
    rmax = radius * (1 + xp.swellingRatio) ** (1 / 3)
    xp.particleMaxRadius = wp.array(rmax, dtype=float)
    xp.max_radius = float(np.max(rmax))
    pad = -xp.max_radius * 1.5 - (mpm.boundaryPadding - 1) * dx
    xp.minBoundsXPBD = wp.vec3(*(minB - pad))
    xp.maxBoundsXPBD = wp.vec3(*(minB + np.array(dims) * dx + pad))
    xin = x - rng.normal(0, 0.05, (n, 3))
    xp.particle_x_initial_xpbd = wp.array(np.where((ml == 2)[:, None], xin, 1e6), dtype=wp.vec3)
    return sim, mpm, xp


SCALARS = {"sim": ("dt", "dtxpbd", "dx", "invdx"),
           "mpm": ("rpic_damping", "grid_v_damping_scale", "boundFriction", "boundRestitution",
                   "boundaryPadding", "eff", "update_cov", "volumetric_locking_correction", "constitutive_model"),
           "xpbd": ("xpbd_iterations", "xpbd_relaxation", "xpbd_mpm_coupling_strength", "mpm_contact_transition_lock",
                    "dynamicParticleFriction", "staticParticleFriction", "staticVelocityThreshold",
                    "particle_cohesion", "sleepThreshold", "particle_v_max", "swellingRatio",
                    "swellingActivationFactor", "swellingMaxFactor", "max_radius")}


def snapshot(wp, objs, prefix):
    out = {}
    for tag, o in objs.items():
        for k, v in vars(o).items():
            if isinstance(v, wp.array) and v.data is not None:
                out[f"{prefix}{tag}.{k}"] = np.array(v.data)
            elif isinstance(v, wp.vec3):
                out[f"{prefix}{tag}.{k}"] = v.a.copy()
        for k in SCALARS[tag]:
            if hasattr(o, k):
                out[f"{prefix}{tag}.{k}"] = np.asarray(getattr(o, k))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("MPMW_REFERENCE"),
                    help="checkout of the reference project (or set MPMW_REFERENCE)")
    a = ap.parse_args()
    if not a.reference:
        ap.error("give the reference checkout with --reference PATH or MPMW_REFERENCE")
    wp, SS, RS, RM = load_reference(a.reference)
    scenes = [
        ("mpm_friction", 101, dict(dt=1e-4), "mpm", {}),
        ("mpm_restitution", 102, dict(dt=1e-4, boundaryCondition="restitution", boundRestitution=0.3,
                                      grid_v_damping_scale=0.98, volumetric_locking_correction=0, update_cov=0), "mpm", {}),
        ("mpm_planestrain", 103, dict(dt=1e-4, boundaryCondition="plane_strain_y", rpic_damping=0.0), "mpm", {}),
        ("xpbd_lock", 201, dict(dt=1e-4, dtxpbd=5e-4, mpm_contact_transition_lock=1, particle_cohesion=0.02,
                                staticVelocityThreshold=0.5, xpbd_iterations=4), "xpbd", dict(xpbd_frac=0.35, lock_labels=True)),
        ("xpbd_free", 202, dict(dt=1e-4, dtxpbd=5e-4, mpm_contact_transition_lock=0, particle_cohesion=0.0,
                                swellingRatio=0.3, xpbd_iterations=3), "xpbd", dict(xpbd_frac=0.35)),
    ]
    for name, seed, over, kind, kw in scenes:
        args = default_args(**over)
        sim, mpm, xp = build_scene(wp, SS, RM, seed, args, **kw)
        objs = {"sim": sim, "mpm": mpm, "xpbd": xp}
        data = snapshot(wp, objs, "in/")
        if kind == "mpm":
            RS.mpmSimulationStep(sim, mpm, xp, "cpu")
        else:
            RS.xpbdSimulationStep(sim, mpm, xp, "cpu")
        # outputs: only the arrays the step changed (a missing out/ key means unchanged)
        for k, v in snapshot(wp, objs, "out/").items():
            kin = "in/" + k[4:]
            if kin not in data or data[kin].shape != v.shape or not np.array_equal(data[kin], v):
                data[k] = v
        data["meta/boundaryCondition"] = np.asarray(args.boundaryCondition)
        data["meta/gravity"] = sim.gravity.a.copy()
        path = os.path.join(HERE, f"{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{name}: {sim.nPoints} particles, {len(data)} arrays -> {os.path.relpath(path, ROOT)}")


if __name__ == "__main__":
    main()
