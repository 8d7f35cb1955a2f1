"""The reference's XPBD kernel surface (utils/xpbdRoutines.py), backed by libmpmw.

Each reference kernel is a callable with the same name and positional
arguments (CUDA tensors in the reference shapes, or state attributes).
``HashGrid`` stands in for ``wp.HashGrid``: same constructor dims, same
``build(points, radius)``, and its object is what the reference passes as
``grid`` (``particle_grid.id``).  :func:`xpbd_step` is the whole
``xpbdSimulationStep`` (utils/simulationRoutines.py:295-526) in one library call.
"""
from __future__ import annotations

import ctypes

import torch

from .. import _lib
from ..bind import Marshal, particles_from_states, particles_struct, ptr, status_word, stream_handle
from ..state import F32, I32

__all__ = ["HashGrid", "reset_mpm_contact_labels", "integrateParticlesXPBD", "my_solve_particle_bound_contacts",
           "my_solve_particle_particle_contacts", "my_apply_particle_deltas", "apply_mpm_contact_impulses",
           "sleepParticles", "clipParticleVelocitiesOnPhaseChange", "swellParticlesType2", "xpbd_step"]


class HashGrid:
    """Spatial hash with the interface of ``wp.HashGrid(dim_x, dim_y, dim_z)``.

    ``build(points, radius)`` hashes (N, 3) CUDA points into cubic cells of
    width ``radius``; the sorted point order (``point_ids``) and per-hash ranges
    (``cell_starts``/``cell_ends``, 0/0 for empty hashes) stay on the device."""

    def __init__(self, dim_x, dim_y, dim_z, device="cuda:0"):
        self.dims = (int(dim_x), int(dim_y), int(dim_z))
        self.device = torch.device(device)
        self.cell_width = None
        self.n = 0
        self.point_ids = None
        self.point_cells = None
        self.cell_starts = None
        self.cell_ends = None
        self._ws = None
        self.id = self  # the reference passes grid.id into its kernels

    def _ensure(self, n):
        nc = self.dims[0] * self.dims[1] * self.dims[2]
        if self.cell_starts is None:
            self.cell_starts = torch.zeros(nc, dtype=I32, device=self.device)
            self.cell_ends = torch.zeros(nc, dtype=I32, device=self.device)
        if self.point_ids is None or self.point_ids.numel() < n:
            self.point_ids = torch.zeros(max(n, 1), dtype=I32, device=self.device)
            self.point_cells = torch.zeros(max(n, 1), dtype=I32, device=self.device)
        # room for the XPBD step's contact records as well (the hash build alone
        # needs less)
        dims = (ctypes.c_int32 * 3)(*[int(d) for d in self.dims])
        need = int(_lib.lib().mpmw_xpbd_step_workspace_bytes(n, dims))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.empty(max(need, 256), dtype=torch.uint8, device=self.device)

    def struct(self) -> _lib.Hash:
        h = _lib.Hash()
        for i in range(3):
            h.dims[i] = self.dims[i]
        h.cell_width = float(self.cell_width or 1.0)
        h.point_ids = ptr(self.point_ids)
        h.cell_starts = ptr(self.cell_starts)
        h.cell_ends = ptr(self.cell_ends)
        h.point_cells = ptr(self.point_cells)
        return h

    def workspace(self):
        return self._ws

    def build(self, points, radius):
        m = Marshal()
        x = m.vec3(points)
        n = x.shape[1]
        self.cell_width = float(radius)
        self._ensure(n)
        self.n = n
        _lib.check(_lib.lib().mpmw_hash_build(x.data_ptr(), n, self.struct(), self._ws.data_ptr(), self._ws.numel(),
                                              stream_handle()), "HashGrid.build")


def _params(**kw) -> _lib.XPBDParams:
    q = _lib.XPBDParams()
    g = kw.get("gravity", (0.0, 0.0, 0.0))
    for i in range(3):
        q.gravity[i] = float(g[i])
        q.bmin[i] = float(kw.get("bmin", (0, 0, 0))[i])
        q.bmax[i] = float(kw.get("bmax", (0, 0, 0))[i])
    for name in ("dt", "v_max", "relaxation", "coupling", "dyn_friction", "static_friction", "static_thr", "cohesion",
                 "max_radius", "sleep_thr", "swelling_ratio", "swell_act", "swell_max"):
        setattr(q, name, float(kw.get(name, 0.0)))
    q.iterations = int(kw.get("iterations", 0))
    q.lock = int(kw.get("lock", 0))
    q.xpbd_only = int(kw.get("xpbd_only", 0))
    if q.dt == 0.0:
        q.dt = 1.0  # kernels that do not use dt still pass the argument check
    return q


def _xstruct(**kw) -> _lib.XPBD:
    X = _lib.XPBD()
    for name, _ in X._fields_:
        t = kw.get(name)
        setattr(X, name, ptr(t) if t is not None else None)
    return X


def _run(which, P, X, q, flag=0, H=None, what=""):
    _lib.check(_lib.lib().mpmw_xpbd_kernel(_lib.XK[which], P, X, H, q, int(flag), stream_handle()), what or which)


def _n(t):
    return t.shape[0]


# ---------------------------------------------------------------------------
# reference kernels
# ---------------------------------------------------------------------------
def reset_mpm_contact_labels(activeLabel, materialLabel):
    """xpbdRoutines.py:3-21."""
    m = Marshal()
    P = particles_struct(_n(activeLabel), active=m.labels(activeLabel), material=m.labels(materialLabel, out=True))
    dummy = torch.zeros(3, _n(activeLabel), dtype=F32, device=activeLabel.device)
    P.x = P.v = P.mass = P.radius = dummy.data_ptr()
    X = _xstruct(x_int=dummy, v_int=dummy, delta=dummy)
    _run("RESET_LABELS", P, X, _params(dt=1.0), what="reset_mpm_contact_labels")
    m.finish()


def integrateParticlesXPBD(activeLabel, materialLabel, x, v, gravity, dt, x_new, v_new, v_max):
    """xpbdRoutines.py:23-48 (writes x_new/v_new of active XPBD particles only)."""
    m = Marshal()
    n = _n(activeLabel)
    xi, vi = m.vec3(x), m.vec3(v)
    xo, vo = m.vec3(x_new, out=True), m.vec3(v_new, out=True)
    ones = torch.ones(n, dtype=F32, device=activeLabel.device)
    P = particles_struct(n, active=m.labels(activeLabel), material=m.labels(materialLabel), x=xi, v=vi, mass=ones,
                         radius=ones)
    X = _xstruct(x_int=xo, v_int=vo, delta=xo)
    _run("INTEGRATE", P, X, _params(gravity=gravity, dt=dt, v_max=v_max), flag=1, what="integrateParticlesXPBD")
    m.finish()


def my_solve_particle_bound_contacts(activeLabel, materialLabel, particle_x, particle_v, mass, particle_radius, mu,
                                     staticGroundVelocityThresholdRatio, staticGroundFriction, minbounds, maxbounds,
                                     dt, relaxation, delta):
    """xpbdRoutines.py:49-136 (adds into delta)."""
    m = Marshal()
    n = _n(activeLabel)
    xi, vi = m.vec3(particle_x), m.vec3(particle_v)
    P = particles_struct(n, active=m.labels(activeLabel), material=m.labels(materialLabel), x=xi, v=vi,
                         mass=m.scalar(mass), radius=m.scalar(particle_radius))
    X = _xstruct(x_int=xi, v_int=vi, delta=m.vec3(delta, out=True))
    q = _params(dt=dt, relaxation=relaxation, dyn_friction=mu, static_thr=staticGroundVelocityThresholdRatio,
                static_friction=staticGroundFriction, bmin=minbounds, bmax=maxbounds)
    _run("BOUND", P, X, q, flag=1, what="my_solve_particle_bound_contacts")
    m.finish()


def my_solve_particle_particle_contacts(activeLabel, materialLabel, grid, particle_x, particle_v, particle_mass,
                                        particle_radius, k_mu, staticParticleVelocityThresholdRatio,
                                        staticParticleFriction, k_cohesion, max_radius, dt, relaxation,
                                        mpm_contact_transition_lock, deltas):
    """xpbdRoutines.py:138-219 (adds into deltas; may set materialLabel to 0)."""
    m = Marshal()
    n = _n(activeLabel)
    xi, vi = m.vec3(particle_x), m.vec3(particle_v)
    P = particles_struct(n, active=m.labels(activeLabel), material=m.labels(materialLabel, out=True), x=xi, v=vi,
                         mass=m.scalar(particle_mass), radius=m.scalar(particle_radius))
    X = _xstruct(x_int=xi, v_int=vi, delta=m.vec3(deltas, out=True))
    q = _params(dt=dt, relaxation=relaxation, dyn_friction=k_mu, static_thr=staticParticleVelocityThresholdRatio,
                static_friction=staticParticleFriction, cohesion=k_cohesion, max_radius=max_radius,
                lock=mpm_contact_transition_lock)
    g = grid.id if hasattr(grid, "id") else grid
    _run("PARTICLE", P, X, q, H=g.struct(), what="my_solve_particle_particle_contacts")
    m.finish()


def my_apply_particle_deltas(activeLabel, materialLabel, x_orig, x_pred, delta, dt, v_max, x_out, v_out):
    """xpbdRoutines.py:221-257 (writes x_out/v_out of active particles)."""
    m = Marshal()
    n = _n(activeLabel)
    ones = torch.ones(n, dtype=F32, device=activeLabel.device)
    P = particles_struct(n, active=m.labels(activeLabel), material=m.labels(materialLabel), x=m.vec3(x_orig),
                         v=m.vec3(x_orig), mass=ones, radius=ones)
    xp = m.vec3(x_pred)
    X = _xstruct(x_int=xp, v_int=xp, delta=m.vec3(delta), x_dI=m.vec3(x_out, out=True), v_dI=m.vec3(v_out, out=True))
    _run("APPLY", P, X, _params(dt=dt, v_max=v_max), flag=2, what="my_apply_particle_deltas")
    m.finish()


def apply_mpm_contact_impulses(activeLabel, materialLabel, x_orig, v_orig, x_final, v_final, dt, v_max,
                               coupling_strength, xpbd_only, v_out):
    """xpbdRoutines.py:259-310 (x_final reset for MPM particles; v_out written
    for MPM particles unless xpbd_only)."""
    m = Marshal()
    n = _n(activeLabel)
    ones = torch.ones(n, dtype=F32, device=activeLabel.device)
    P = particles_struct(n, active=m.labels(activeLabel), material=m.labels(materialLabel), x=m.vec3(x_orig),
                         v=m.vec3(v_orig), mass=ones, radius=ones)
    xf = m.vec3(x_final, out=True)
    vo = m.vec3(v_out, out=True)
    X = _xstruct(x_int=xf, v_int=vo, delta=xf)
    q = _params(dt=dt, v_max=v_max, coupling=coupling_strength, xpbd_only=xpbd_only)
    _run("IMPULSES", P, X, q, flag=0, what="apply_mpm_contact_impulses")
    m.finish()


def sleepParticles(activeLabel, materialLabel, sleepThreshold, radius, particle_positions_prev,
                   particle_positions_after, particle_distance_total, dt, total_xpbd, sleeping_xpbd):
    """xpbdRoutines.py:312-334 (adds into total_xpbd[0] / sleeping_xpbd[0])."""
    m = Marshal()
    n = _n(activeLabel)
    ones = torch.ones(n, dtype=F32, device=activeLabel.device)
    P = particles_struct(n, active=m.labels(activeLabel), material=m.labels(materialLabel),
                         x=m.vec3(particle_positions_prev), v=m.vec3(particle_positions_prev), mass=ones,
                         radius=m.scalar(radius))
    xa = m.vec3(particle_positions_after, out=True)
    counts = torch.zeros(2, dtype=I32, device=activeLabel.device)
    X = _xstruct(x_int=xa, v_int=xa, delta=xa, cum_dist=m.scalar(particle_distance_total, out=True), counts=counts)
    _run("SLEEP", P, X, _params(dt=dt, sleep_thr=sleepThreshold), flag=0, what="sleepParticles")
    m.finish()
    total_xpbd[0] += counts[0].to(total_xpbd.dtype)
    sleeping_xpbd[0] += counts[1].to(sleeping_xpbd.dtype)


def clipParticleVelocitiesOnPhaseChange(activeLabel, materialLabel, particle_distance_total,
                                        particleInitialXPBDVelocity, particle_v, radius):
    """xpbdRoutines.py:336-351 (its launch is commented out in the reference):
    active XPBD particles that travelled less than two radii keep at most their
    phase-change velocity."""
    sel = (activeLabel == 1) & (materialLabel == 2) & (particle_distance_total < radius * 2.0)
    sel = sel & (torch.linalg.vector_norm(particle_v, dim=1) > torch.linalg.vector_norm(particleInitialXPBDVelocity, dim=1))
    particle_v[sel] = particleInitialXPBDVelocity[sel]


def swellParticlesType2(activeLabel, materialLabel, particle_initial_position, particle_position, particle_radius,
                        factor, factor_max, swellRadius, baseRadius):
    """xpbdRoutines.py:354-375."""
    m = Marshal()
    n = _n(activeLabel)
    xp = m.vec3(particle_position)
    P = particles_struct(n, active=m.labels(activeLabel), material=m.labels(materialLabel), x=xp, v=xp,
                         x_pc=m.vec3(particle_initial_position), mass=m.scalar(particle_radius),
                         radius=m.scalar(particle_radius, out=True))
    X = _xstruct(x_int=xp, v_int=xp, delta=xp, base_radius=m.scalar(baseRadius), max_radius=m.scalar(swellRadius))
    _run("SWELL", P, X, _params(swell_act=factor, swell_max=factor_max), what="swellParticlesType2")
    m.finish()


# ---------------------------------------------------------------------------
# whole step
# ---------------------------------------------------------------------------
def _counts_view(sim):
    c = getattr(sim, "_xpbd_counts", None)
    if c is None:
        c = torch.zeros(2, dtype=I32, device=sim.device)
        sim._xpbd_counts = c
        sim.numTotalXPBD = c[0:1]
        sim.numSleepingXPBD = c[1:2]
    return c


def xpbd_structs(sim, mpm, xpbd, xpbd_only=False):
    g = lambda o, a: getattr(o, "_s_" + a, None)  # noqa: E731
    P = particles_from_states(sim, mpm, xpbd)
    X = _xstruct(x_int=g(xpbd, "particle_x_integrated"), v_int=g(xpbd, "particle_v_integrated"),
                 x_dI=g(xpbd, "particle_x_deltaInt"), v_dI=g(xpbd, "particle_v_deltaInt"),
                 delta=g(xpbd, "particle_delta"), v_before=g(xpbd, "particle_v_before_contact"),
                 cum_dist=g(xpbd, "particle_cumDist_xpbd"), base_radius=g(xpbd, "particleBaseRadius"),
                 max_radius=g(xpbd, "particleMaxRadius"), counts=_counts_view(sim))
    q = _params(gravity=sim.gravity, dt=sim.dtxpbd, v_max=xpbd.particle_v_max, iterations=xpbd.xpbd_iterations,
                relaxation=xpbd.xpbd_relaxation, coupling=xpbd.xpbd_mpm_coupling_strength,
                lock=xpbd.mpm_contact_transition_lock, dyn_friction=xpbd.dynamicParticleFriction,
                static_friction=xpbd.staticParticleFriction, static_thr=xpbd.staticVelocityThreshold,
                cohesion=xpbd.particle_cohesion, max_radius=xpbd.max_radius or 0.0, sleep_thr=xpbd.sleepThreshold,
                bmin=xpbd.minBoundsXPBD or (0, 0, 0), bmax=xpbd.maxBoundsXPBD or (0, 0, 0),
                swelling_ratio=xpbd.swellingRatio, swell_act=xpbd.swellingActivationFactor,
                swell_max=xpbd.swellingMaxFactor, xpbd_only=xpbd_only)
    return P, X, q


def xpbd_step(sim, mpm, xpbd, xpbd_only=False):
    """utils/simulationRoutines.py:295-526 as one library call."""
    P, X, q = xpbd_structs(sim, mpm, xpbd, xpbd_only)
    hg = xpbd.particle_grid
    hg.cell_width = float(sim.dx)
    hg._ensure(sim.nPoints)
    hg.n = sim.nPoints
    ws = hg.workspace()
    _lib.check(_lib.lib().mpmw_xpbd_step(P, X, hg.struct(), q, status_word(sim.device).data_ptr(), ws.data_ptr(),
                                         ws.numel(), stream_handle()),
               "xpbdSimulationStep")
