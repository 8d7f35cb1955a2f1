"""State containers under the reference's names (utils/simStates.py:10-179).

``SimState``, ``MPMState`` and ``XPBDState`` keep every attribute name,
constructor signature and default of the reference.  Arrays are CUDA tensors
held in SoA storage (see ``mpmwarpydw_b200.state``) and read back under the
reference shapes: ``particle_x`` is (N, 3), ``particle_F`` is (N, 3, 3),
``grid_v_out`` is (nx, ny, nz, 3), and so on.  ``device`` defaults to
"cuda:0" as in the reference.

Differences a caller may notice:
  * scalar "vectors" (gravity, minBounds, ...) are tuples of 3 floats instead
    of ``wp.vec3``; indexing works the same;
  * ``particle_stress`` is stored as its 6 symmetric components; reading it
    returns a freshly built (N, 3, 3) tensor, assigning it stores a copy;
  * ``XPBDState.particle_grid`` is a :class:`mpmwarpydw_b200.utils.xpbdRoutines.HashGrid`
    (same dims, same ``build(points, cell_width)`` call).
"""
from __future__ import annotations

import torch

from ..state import F32, I32, GridField, GridPacked, Mat33Field, ScalarField, Sym33Field, Vec3Field


def vec3(x, y, z):
    """Stand-in for ``wp.vec3`` scalars: a tuple of three Python floats."""
    return (float(x), float(y), float(z))


def _zeros(n, device, dtype=F32):
    return torch.zeros(n, dtype=dtype, device=device)


class SimState:
    particle_x = Vec3Field()
    particle_v = Vec3Field()
    particle_mass = ScalarField()
    particle_vol = ScalarField()
    particle_radius = ScalarField()
    particle_density = ScalarField()
    materialLabel = ScalarField(I32)
    activeLabel = ScalarField(I32)
    particleBCMask = ScalarField(I32)

    def __init__(self, args, nPoints, device="cuda:0"):
        """Initialize simulation state (utils/simStates.py:11-71)."""
        self.device = torch.device(device)
        self.nPoints = int(nPoints)
        self.dt = args.dt
        self.dtxpbd = args.dtxpbd
        self.bigStepDuration = args.bigStepDuration
        self.xpbdOnlyDuration = args.xpbdOnlyDuration
        self.bigSteps = args.bigSteps
        self.nSteps = int(self.bigStepDuration / self.dt) if self.dt else 0
        self.xpbdOnlySteps = int(self.xpbdOnlyDuration / self.dtxpbd) if self.xpbdOnlyDuration > 0 else 0
        self.mpmStepsPerXpbdStep = int(self.dtxpbd / self.dt) if self.dt else 1
        self.t = 0.0
        self.residualThreshold = args.residualThreshold
        self.damage_stall_threshold = args.damage_stall_threshold
        self.damage_stall_duration = args.damage_stall_duration
        self.xpbd_sleep_termination_ratio = args.xpbd_sleep_termination_ratio
        self.render = args.render
        self.saveFlag = args.saveFlag
        self.color_mode = args.color_mode
        self.outputFolder = args.outputFolder
        self.gravity = vec3(0.0, 0.0, args.gravity)
        self.particle_x = None
        self.particle_v = None
        self.particle_mass = None
        self.particle_vol = None
        self.particle_radius = None
        self.particle_density = None
        self.materialLabel = None
        self.activeLabel = None
        self.particleBCMask = None
        self.minBounds = None
        self.maxBounds = None
        self.dx = None
        self.invdx = None
        d = self.device
        self.residual = torch.tensor([1e10], dtype=F32, device=d)
        self.numActiveParticles = _zeros(1, d, I32)
        self.numTotalXPBD = _zeros(1, d, I32)
        self.numSleepingXPBD = _zeros(1, d, I32)
        self.numActiveMPM = _zeros(1, d, I32)
        self.numActiveXPBD = _zeros(1, d, I32)
        self.numInactiveMPM = _zeros(1, d, I32)
        self.numInactiveXPBD = _zeros(1, d, I32)
        self.scratchFloat = _zeros(1, d)
        self.scratchInt = _zeros(1, d, I32)


class MPMState:
    """MPM-specific state variables (utils/simStates.py:74-130)."""

    mu = ScalarField()
    lam = ScalarField()
    bulk = ScalarField()
    ys = ScalarField()
    ys_base = ScalarField()
    alpha = ScalarField()
    hardening = ScalarField()
    softening = ScalarField()
    eta_shear = ScalarField()
    eta_bulk = ScalarField()
    strainCriteria = ScalarField()
    particle_F = Mat33Field()
    particle_F_trial = Mat33Field()
    particle_stress = Sym33Field()
    particle_accumulated_strain = ScalarField()
    particle_damage = ScalarField()
    particle_C = Mat33Field()
    particle_init_cov = ScalarField()
    particle_cov = ScalarField()
    particle_x_initial = Vec3Field()
    cell_div_v_weighted = GridField()
    cell_vol_sum = GridField()

    def __init__(self, args, nPoints, gridDims, device="cuda:0"):
        self.device = torch.device(device)
        d = self.device
        self.nPoints = int(nPoints)
        self.gridDims = tuple(int(g) for g in gridDims)
        self.rpic_damping = args.rpic_damping
        self.grid_v_damping_scale = args.grid_v_damping_scale
        self.update_cov = args.update_cov
        self.constitutive_model = args.constitutive_model
        self.K0 = args.K0
        self.boundaryCondition = args.boundaryCondition
        self.boundFriction = args.boundFriction
        self.boundRestitution = args.boundRestitution
        self.boundaryPadding = None
        for name in ("mu", "lam", "bulk", "ys", "ys_base", "alpha", "hardening", "softening", "eta_shear",
                     "eta_bulk", "strainCriteria"):
            setattr(self, name, None)
        n = self.nPoints
        eye = torch.zeros(n, 3, 3, dtype=F32, device=d)
        self.particle_F = eye
        self.particle_F_trial = eye
        self.particle_stress = eye
        self.particle_accumulated_strain = _zeros(n, d)
        self.particle_damage = _zeros(n, d)
        self.particle_C = eye
        self.particle_init_cov = _zeros(n * 6, d)
        self.particle_cov = _zeros(n * 6, d)
        self._grid_mv = GridPacked(self.gridDims, d)     # (m, m*v): P2G accumulators
        self._grid_v = GridPacked(self.gridDims, d)      # (v, pad): grid velocity
        self.gridBCIndex = torch.zeros(self.gridDims, dtype=I32, device=d)
        self.volumetric_locking_correction = args.volumetric_locking_correction
        self.cell_div_v_weighted = torch.zeros(self.gridDims, dtype=F32, device=d)
        self.cell_vol_sum = torch.zeros(self.gridDims, dtype=F32, device=d)
        self.particle_x_initial = torch.zeros(n, 3, dtype=F32, device=d)
        self.eff = args.eff
        # 0 (default): clearly elastic particles take the SVD-free log-strain path,
        # all others the SVD return map; 1: SVD return map for every particle
        self.stress_mode = int(getattr(args, "stress_mode", 0))

    @property
    def grid_m(self):
        return self._grid_mv.comp(0)

    @property
    def grid_v_in(self):
        return self._grid_mv.comp(slice(1, 4))

    @property
    def grid_v_out(self):
        return self._grid_v.comp(slice(0, 3))


class XPBDState:
    """XPBD-specific state variables (utils/simStates.py:133-179)."""

    particle_x_initial_xpbd = Vec3Field()
    particle_v_initial_xpbd = Vec3Field()
    particle_cumDist_xpbd = ScalarField()
    particle_distance_total = ScalarField()
    particle_x_integrated = Vec3Field()
    particle_v_integrated = Vec3Field()
    particle_x_deltaInt = Vec3Field()
    particle_v_deltaInt = Vec3Field()
    particle_delta = Vec3Field()
    particle_v_before_contact = Vec3Field()
    particleBaseRadius = ScalarField()
    particleMaxRadius = ScalarField()

    def __init__(self, args, nPoints, device="cuda:0"):
        from .xpbdRoutines import HashGrid

        self.device = torch.device(device)
        d = self.device
        self.nPoints = n = int(nPoints)
        self.xpbd_iterations = args.xpbd_iterations
        self.xpbd_relaxation = args.xpbd_relaxation
        self.xpbd_mpm_coupling_strength = args.xpbd_mpm_coupling_strength
        self.mpm_contact_transition_lock = args.mpm_contact_transition_lock
        self.dynamicParticleFriction = args.dynamicParticleFriction
        self.staticParticleFriction = args.staticParticleFriction
        self.staticVelocityThreshold = args.staticVelocityThreshold
        self.particle_cohesion = args.particle_cohesion
        self.sleepThreshold = args.sleepThreshold
        self.particle_v_max = args.particle_v_max
        self.swellingRatio = args.swellingRatio
        self.swellingActivationFactor = args.swellingActivationFactor
        self.swellingMaxFactor = args.swellingMaxFactor
        self.particleBaseRadius = None
        self.particleMaxRadius = None
        z3 = torch.zeros(n, 3, dtype=F32, device=d)
        self.particle_x_initial_xpbd = torch.full((n, 3), 1e6, dtype=F32, device=d)
        self.particle_v_initial_xpbd = z3
        self.particle_cumDist_xpbd = _zeros(n, d)
        self.particle_distance_total = _zeros(n, d)
        self.particle_x_integrated = z3
        self.particle_v_integrated = z3
        self.particle_x_deltaInt = z3
        self.particle_v_deltaInt = z3
        self.particle_delta = z3
        self.particle_v_before_contact = z3
        self.particle_grid = HashGrid(128, 128, 128, device=d)
        self.minBoundsXPBD = None
        self.maxBoundsXPBD = None
        self.max_radius = None
