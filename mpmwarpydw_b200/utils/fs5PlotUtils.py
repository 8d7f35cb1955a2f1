"""Output and restart files with the reference's names, arrays and file
layout (utils/fs5PlotUtils.py of the reference), written and read by
:mod:`mpmwarpydw_b200.vtkio` instead of the vtk package:

  save_grid_and_particles_vti_vtp  (:433-645)  <prefix>_grid.vti + <prefix>_particles.vtp
  save_mpm                         (:785-881)  one save of the simulation state
  load_restart_from_vtp            (:253-431)  the restart dictionary of a checkpoint

The renderers of that module (OpenGL, USD) are not provided: no graphics
stack is available.  Particle arrays are taken in the order given; the driver
passes them in input order, as the reference writes them.
"""
from __future__ import annotations

import os

import numpy as np

from .. import vtkio

MATERIAL_PROPERTIES = ("mu", "lam", "bulk", "alpha", "hardening", "softening", "eta_shear", "eta_bulk",
                       "strainCriteria")


def _np(a):
    if a is None:
        return None
    if hasattr(a, "detach"):
        return a.detach().cpu().numpy()
    return np.asarray(a)


def save_grid_and_particles_vti_vtp(output_prefix, grid_mass, minBounds, dx, particle_positions, particle_radius=0.5,
                                    particle_velocity=None, particle_ys=None, particle_effective_ys=None,
                                    particle_damage=None, particle_mean_stress=None, particle_von_mises=None,
                                    particle_stress_tensor=None, particle_active_label=None,
                                    particle_material_label=None, restart_data=None):
    """The grid mass as <prefix>_grid.vti and the particles as
    <prefix>_particles.vtp, with the reference's array names; restart_data
    (a checkpoint) adds F, C, the plastic state, material and physical
    properties, the XPBD fields and the sim_time / bigStep / dx field data."""
    d = os.path.dirname(output_prefix)
    if d:
        os.makedirs(d, exist_ok=True)
    gm = np.asarray(_np(grid_mass), np.float32)
    vtkio.write_vti(f"{output_prefix}_grid.vti", gm.shape, np.asarray(minBounds, np.float64), float(dx),
                    {"grid_mass": gm})
    pos = np.asarray(_np(particle_positions), np.float32).reshape(-1, 3)
    n = pos.shape[0]
    pd = {}
    r = _np(particle_radius)
    pd["radius"] = np.full(n, float(r), np.float32) if np.ndim(r) == 0 else np.asarray(r, np.float32)
    f32 = lambda a: np.asarray(_np(a), np.float32)  # noqa: E731
    if particle_velocity is not None:
        pd["velocity"] = f32(particle_velocity).reshape(n, 3)
    for name, a in (("yield_stress", particle_ys), ("effective_yield_stress", particle_effective_ys),
                    ("damage", particle_damage), ("mean_stress", particle_mean_stress),
                    ("von_mises_stress", particle_von_mises)):
        if a is not None:
            pd[name] = f32(a).reshape(n)
    if particle_stress_tensor is not None:
        s = f32(particle_stress_tensor)
        if s.ndim == 3:
            s = np.stack([s[:, 0, 0], s[:, 1, 1], s[:, 2, 2], s[:, 0, 1], s[:, 0, 2], s[:, 1, 2]], 1)
        pd["stress_tensor"] = np.ascontiguousarray(s.reshape(n, -1))
    if particle_active_label is not None:
        pd["active_label"] = np.asarray(_np(particle_active_label), np.int32)
    if particle_material_label is not None:
        pd["material_label"] = np.asarray(_np(particle_material_label), np.int32)
    fd = None
    if restart_data is not None:
        fd = {k: np.array([float(restart_data[k])], np.float32) for k in ("sim_time", "bigStep", "dx")
              if k in restart_data}
        rd = restart_data
        if "particle_F" in rd:
            pd["deformation_gradient_F"] = f32(rd["particle_F"]).reshape(n, 9)
        if "particle_C" in rd:
            pd["apic_C"] = f32(rd["particle_C"]).reshape(n, 9)
        if "particle_accumulated_strain" in rd:
            pd["accumulated_strain"] = f32(rd["particle_accumulated_strain"]).reshape(n)
        if "ys_base" in rd and rd["ys_base"] is not None:
            pd["yield_stress_base"] = f32(rd["ys_base"]).reshape(n)
        for p in MATERIAL_PROPERTIES:
            if p in rd and rd[p] is not None:
                pd[f"mpm_{p}"] = f32(rd[p]).reshape(n)
        for key, name in (("particle_vol", "particle_volume"), ("particle_mass", "particle_mass"),
                          ("particle_density", "particle_density"), ("particle_cumDist_xpbd",
                                                                     "xpbd_cumulative_distance")):
            if key in rd and rd[key] is not None:
                pd[name] = f32(rd[key]).reshape(n)
        if "particle_x_initial_xpbd" in rd and rd["particle_x_initial_xpbd"] is not None:
            pd["xpbd_initial_position"] = f32(rd["particle_x_initial_xpbd"]).reshape(n, 3)
    vtkio.write_vtp(f"{output_prefix}_particles.vtp", pos, pd, fd)
    return f"{output_prefix}_particles.vtp"


def save_mpm(sim, mpm, bigStep, counter, include_restart_data=False, xpbd=None, order=None):
    """One save of the simulation state with the reference's derived arrays:
    mean stress tr(sigma)/3, von Mises sqrt(3/2 |dev sigma|^2) and the
    Drucker-Prager effective yield stress (ys - alpha p)(1 - D), p the mean
    stress.  ``order`` (a callable) maps each per-particle array to the
    order to write (the driver passes the input order); include_restart_data
    makes the save a checkpoint.  Returns the .vtp path."""
    o = order or (lambda t: t)
    c = lambda t: None if t is None else _np(o(t))  # noqa: E731
    sigma = c(mpm.particle_stress).astype(np.float64)
    mean_stress = np.trace(sigma, axis1=1, axis2=2) / 3.0
    s = sigma - mean_stress[:, None, None] * np.eye(3)
    von_mises = np.sqrt(1.5 * np.sum(s ** 2, axis=(1, 2)))
    ys, alpha, damage = c(mpm.ys), c(mpm.alpha), c(mpm.particle_damage)
    effective_ys = (ys - alpha * mean_stress) * (1.0 - damage)
    restart = None
    if include_restart_data:
        restart = {"sim_time": sim.t, "bigStep": bigStep, "dx": sim.dx, "particle_F": c(mpm.particle_F),
                   "particle_C": c(mpm.particle_C), "particle_accumulated_strain": c(mpm.particle_accumulated_strain),
                   "ys_base": c(getattr(mpm, "ys_base", None)), "particle_vol": c(sim.particle_vol),
                   "particle_mass": c(sim.particle_mass), "particle_density": c(sim.particle_density)}
        for p in MATERIAL_PROPERTIES:
            restart[p] = c(getattr(mpm, p, None))
        if xpbd is not None:
            restart["particle_x_initial_xpbd"] = c(xpbd.particle_x_initial_xpbd)
            restart["particle_cumDist_xpbd"] = c(xpbd.particle_cumDist_xpbd)
    prefix = f"{sim.outputFolder}/sim_step_{bigStep:04d}{counter:06d}{int(np.ceil(sim.t * 1e8)):016d}"
    return save_grid_and_particles_vti_vtp(
        prefix, grid_mass=_np(mpm.grid_m), minBounds=sim.minBounds, dx=sim.dx,
        particle_positions=c(sim.particle_x), particle_radius=c(sim.particle_radius),
        particle_velocity=c(sim.particle_v), particle_ys=ys, particle_effective_ys=effective_ys,
        particle_damage=damage, particle_mean_stress=mean_stress, particle_von_mises=von_mises,
        particle_stress_tensor=sigma, particle_active_label=c(sim.activeLabel),
        particle_material_label=c(sim.materialLabel), restart_data=restart)


def load_restart_from_vtp(vtp_path):
    """The restart dictionary of a checkpoint .vtp, with the reference's keys
    and defaults: F identity and C zero when absent, ys_base = ys when absent,
    zero velocity and accumulated strain when absent, sim_time / bigStep / dx
    from the field data."""
    f = vtkio.read_vtp(vtp_path)
    pts = np.asarray(f["points"], np.float32)
    n = pts.shape[0]
    if n == 0:
        raise ValueError(f"Failed to read VTP file or file is empty: {vtp_path}")
    pd, fd = f["point_data"], f["field_data"]
    get = lambda k: pd.get(k)  # noqa: E731
    if "radius" not in pd:
        raise ValueError(f"Required array 'radius' not found in VTP file")
    r = {"particle_x": pts, "particle_radius": get("radius")}
    r["particle_v"] = get("velocity") if get("velocity") is not None else np.zeros((n, 3), np.float32)
    r["ys"], r["particle_damage"] = get("yield_stress"), get("damage")
    r["materialLabel"], r["activeLabel"] = get("material_label"), get("active_label")
    s6 = get("stress_tensor")
    if s6 is not None:
        s = np.zeros((n, 3, 3), np.float32)
        s[:, 0, 0], s[:, 1, 1], s[:, 2, 2] = s6[:, 0], s6[:, 1], s6[:, 2]
        s[:, 0, 1] = s[:, 1, 0] = s6[:, 3]
        s[:, 0, 2] = s[:, 2, 0] = s6[:, 4]
        s[:, 1, 2] = s[:, 2, 1] = s6[:, 5]
        r["particle_stress"] = s
    F = get("deformation_gradient_F")
    r["particle_F"] = F.reshape(-1, 3, 3) if F is not None else np.tile(np.eye(3, dtype=np.float32), (n, 1, 1))
    C = get("apic_C")
    r["particle_C"] = C.reshape(-1, 3, 3) if C is not None else np.zeros((n, 3, 3), np.float32)
    acc = get("accumulated_strain")
    r["particle_accumulated_strain"] = acc if acc is not None else np.zeros(n, np.float32)
    r["ys_base"] = get("yield_stress_base")
    if r["ys_base"] is None and r["ys"] is not None:
        r["ys_base"] = r["ys"].copy()
    for p in MATERIAL_PROPERTIES:
        if get(f"mpm_{p}") is not None:
            r[p] = get(f"mpm_{p}")
    r["particle_vol"], r["particle_mass"] = get("particle_volume"), get("particle_mass")
    r["particle_density"] = get("particle_density")
    if get("xpbd_initial_position") is not None:
        r["particle_x_initial_xpbd"] = get("xpbd_initial_position")
    r["particle_cumDist_xpbd"] = get("xpbd_cumulative_distance")
    scalar = lambda k, d: float(fd[k].reshape(-1)[0]) if k in fd else d  # noqa: E731
    r["sim_time"] = scalar("sim_time", 0.0)
    r["bigStep"] = int(scalar("bigStep", 0))
    r["dx"] = scalar("dx", None)
    return r
