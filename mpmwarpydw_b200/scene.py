"""Scene set-up: from particle positions/volumes + args to the three state objects.

Restates the driver's set-up stage (runMPMYDW.py:17-489): grid spacing from
the mean particle volume, padded bounds from the 6-digit padding mask, CFL
auto-dt and the integer XPBD ratio, material arrays (per-particle arrays from
``props`` override the scalar args, as HDF5 arrays do in the driver), Lame
constants, mass, geostatic (or identity) F, radii and XPBD bounds.  File I/O
and printing are left to the caller.
"""
from __future__ import annotations

import math
from types import SimpleNamespace

import numpy as np
import torch

from .utils import mpmRoutines
from .utils.simStates import MPMState, SimState, XPBDState, vec3

MPM_PADDING = 2  # runMPMYDW.py:35 (grid cells; also mpm.boundaryPadding)

PROP_NAMES = ["density", "E", "nu", "ys", "alpha", "hardening", "softening", "eta_shear", "eta_bulk",
              "strainCriteria", "damage"]


def grid_geometry(args, x, particle_volume, dx=None, minBounds=None, gridDims=None):
    """runMPMYDW.py:21-65: dx, minBounds, maxBounds, gridDims (numpy float64)."""
    if dx is None:
        diameter = float(np.mean(particle_volume)) ** 0.33
        dx = diameter * args.grid_particle_spacing_scale
    pmin, pmax = x.min(0).astype(np.float64), x.max(0).astype(np.float64)
    mask = args.boundary_padding_mask
    if len(mask) != 6 or any(c not in "01" for c in mask):
        raise ValueError(f"boundary_padding_mask must be 6-digit binary string, got: {mask}")
    f = [int(c) for c in mask]
    pad = lambda flag: args.grid_padding * dx if flag else MPM_PADDING * dx  # noqa: E731
    if minBounds is None:
        minBounds = np.array([pmin[0] - pad(f[0]), pmin[1] - pad(f[2]), pmin[2] - pad(f[4])])
    maxBounds = np.array([pmax[0] + pad(f[1]), pmax[1] + pad(f[3]), pmax[2] + pad(f[5])])
    if gridDims is None:
        gridDims = np.ceil((maxBounds - np.asarray(minBounds)) / dx).astype(int)
    else:
        maxBounds = np.asarray(minBounds) + np.asarray(gridDims) * dx
    return float(dx), np.asarray(minBounds, np.float64), maxBounds, tuple(int(g) for g in gridDims)


def auto_dt(args, dx, E, nu, density):
    """runMPMYDW.py:84-169: CFL-based dt when args.dt <= 0, then snap dt so that
    dtxpbd/dt is an integer.  Returns (dt, mpmStepsPerXpbdStep)."""
    E_mean, nu_mean, rho_mean = float(np.mean(E)), float(np.mean(nu)), float(np.mean(density))
    K = E_mean / (3 * (1 - 2 * nu_mean))
    G = E_mean / (2 * (1 + nu_mean))
    c_p = math.sqrt((K + 4 * G / 3) / rho_mean)
    dt = args.dt
    if dt <= 0:
        sf = 0.1
        if nu_mean > 0.45:
            sf *= math.exp(-10 * (nu_mean - 0.45))
        if E_mean < 1e9:
            sf *= float(np.clip((E_mean / 1e9) ** 0.3, 0.1, 1.0))
        sf = float(np.clip(sf, 0.005, 0.2))
        dt = sf * dx / c_p
    ratio = int(np.round(args.dtxpbd / dt))
    ratio = max(ratio, 1)
    return args.dtxpbd / ratio, ratio


def build_states(args, x, particle_volume, props=None, device="cuda:0", dx=None, minBounds=None, gridDims=None,
                 adjust_dt=True):
    """Construct (sim, mpm, xpbd) as the driver does (runMPMYDW.py:180-489)."""
    props = props or {}
    x = np.asarray(x, dtype=np.float32)
    vol = np.asarray(particle_volume, dtype=np.float32).reshape(-1)
    n = x.shape[0]
    dx, minB, maxB, dims = grid_geometry(args, x, vol, dx, minBounds, gridDims)

    def prop(name, default):
        if name in props and props[name] is not None:
            return np.asarray(props[name], dtype=np.float32).reshape(-1)
        return np.full(n, default, dtype=np.float32)

    density, E, nu = prop("density", args.density), prop("E", args.E), prop("nu", args.nu)
    if adjust_dt:
        args.dt, _ = auto_dt(args, dx, E, nu, density)
    sim = SimState(args, n, device=device)
    mpm = MPMState(args, n, dims, device=device)
    xpbd = XPBDState(args, n, device=device)
    sim.minBounds = vec3(*minB)
    sim.maxBounds = vec3(*maxB)
    sim.dx = dx
    sim.invdx = 1.0 / dx
    mpm.boundaryPadding = MPM_PADDING

    d = torch.device(device)
    t = lambda a: torch.as_tensor(a, device=d)  # noqa: E731
    mpm.mu = torch.zeros(n, device=d)
    mpm.lam = torch.zeros(n, device=d)
    mpm.bulk = torch.zeros(n, device=d)
    mpmRoutines.compute_mu_lam_bulk_from_E_nu(t(E), t(nu), mpm.mu, mpm.lam, mpm.bulk)
    mpm.alpha = t(prop("alpha", args.alpha))
    mpm.strainCriteria = t(prop("strainCriteria", args.strainCriteria))
    ys = prop("ys", args.ys)
    mpm.ys_base = t(ys.copy())
    mpm.ys = t(ys)
    mpm.hardening = t(prop("hardening", args.hardening))
    mpm.softening = t(prop("softening", args.softening))
    mpm.eta_shear = t(prop("eta_shear", args.eta_shear))
    mpm.eta_bulk = t(prop("eta_bulk", args.eta_bulk))

    sim.materialLabel = torch.ones(n, dtype=torch.int32, device=d)
    sim.activeLabel = torch.ones(n, dtype=torch.int32, device=d)
    sim.particle_density = t(density)
    sim.particle_x = t(x)
    sim.particle_v = torch.zeros(n, 3, device=d)
    sim.particle_vol = t(vol)
    sim.particle_mass = torch.zeros(n, device=d)
    sim.particleBCMask = torch.zeros(n, dtype=torch.int32, device=d)
    mpmRoutines.get_float_array_product(sim.particle_density, sim.particle_vol, sim.particle_mass)

    z_top = float(np.max(x[:, 2])) if args.z_top is None else float(args.z_top)
    g_mag = abs(args.gravity)
    if args.initialise_geostatic:
        if args.boundaryCondition == "plane_strain_y_global":
            mpmRoutines.initialize_geostatic_F_planestrain(sim.particle_x, mpm.particle_F, mpm.mu, mpm.lam,
                                                           sim.particle_density, g_mag, z_top, mpm.K0)
        else:
            mpmRoutines.initialize_geostatic_F(sim.particle_x, mpm.particle_F, mpm.mu, mpm.lam,
                                               sim.particle_density, g_mag, z_top, mpm.K0)
    else:
        mpmRoutines.set_mat33_to_identity(mpm.particle_F)
    mpmRoutines.set_mat33_to_copy(mpm.particle_F, mpm.particle_F_trial)
    mpm.particle_damage = t(prop("damage", 0.0))

    radius = vol ** (1 / 3) * np.pi / 6  # float32 arithmetic, as runMPMYDW.py:464 on a float32 array
    sim.particle_radius = t(radius.astype(np.float32))
    xpbd.particleBaseRadius = t(radius.astype(np.float32))
    max_r = radius * (1 + xpbd.swellingRatio) ** (1 / 3)
    xpbd.particleMaxRadius = t(max_r.astype(np.float32))
    xpbd.max_radius = float(np.max(max_r)) if n else 0.0
    pd = -xpbd.max_radius * 1.5 - (mpm.boundaryPadding - 1) * sim.dx
    xpbd.minBoundsXPBD = vec3(*(np.asarray(sim.minBounds) - pd))
    xpbd.maxBoundsXPBD = vec3(*(np.asarray(sim.maxBounds) + pd))
    sim.z_top = z_top
    return sim, mpm, xpbd


def clone_args(args, **over):
    a = SimpleNamespace(**vars(args))
    for k, v in over.items():
        setattr(a, k, v)
    return a
