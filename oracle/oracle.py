"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loaded only by tests/, ``__graft_entry__.smoke()`` and ``bench.py``'s
CPU-baseline leg.  The product package never imports this module.

``Oracle(prec)`` wraps ``oracle/_build/libmpm_oracle_<prec>.so`` (built by
``oracle/Makefile``) with numpy-array entry points named after the reference
kernels, and restates the launch order of
``utils/simulationRoutines.py:6-293`` (mpmSimulationStep) and ``:295-526``
(xpbdSimulationStep) in :func:`mpm_step` / :func:`xpbd_step`.

State objects are duck-typed: any object with the reference attribute names
(``particle_x`` (N,3), ``particle_F`` (N,3,3), ``grid_m`` (nx,ny,nz), ...)
holding contiguous numpy arrays of the oracle's dtype works; see
:class:`OracleState`.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import types

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_BUILD = os.path.join(_HERE, "_build")

BC_CODES = {
    "friction": 0,
    "friction_gradual": 1,
    "restitution": 2,
    "absorbing": 3,
    "plane_strain_y": 4,
    "plane_strain_y_global": 5,
}

HASH_DIMS = (128, 128, 128)  # wp.HashGrid(128, 128, 128) at utils/simStates.py:174


def build():
    """Compile the oracle libraries (gcc only)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_I = ctypes.c_int


class Oracle:
    """One precision of the oracle: 'f32', 'f64', 'f32_omp' or 'f64_omp' (OpenMP)."""

    def __init__(self, prec: str = "f64"):
        path = os.path.join(_BUILD, f"libmpm_oracle_{prec}.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        self.prec = prec
        self.dtype = np.float64 if prec.startswith("f64") else np.float32
        self.R = ctypes.c_double if prec.startswith("f64") else ctypes.c_float
        assert self.lib.orc_real_bytes() == np.dtype(self.dtype).itemsize

    # -- argument helpers ---------------------------------------------------
    def _a(self, arr, dtype=None):
        dtype = dtype or self.dtype
        if not (isinstance(arr, np.ndarray) and arr.dtype == dtype and arr.flags["C_CONTIGUOUS"]):
            raise TypeError(f"expected C-contiguous {np.dtype(dtype).name} array, got "
                            f"{getattr(arr, 'dtype', type(arr))}")
        return arr.ctypes.data_as(_P)

    def _i(self, arr):
        return self._a(arr, np.int32)

    def _v3(self, v):
        a = np.ascontiguousarray(np.asarray(v, dtype=self.dtype).reshape(3))
        self._keep = getattr(self, "_keep", [])
        self._keep.append(a)
        return a.ctypes.data_as(_P)

    @staticmethod
    def _dims(d):
        a = (ctypes.c_int * 3)(*[int(v) for v in d])
        return a

    # -- kernels ------------------------------------------------------------
    def svd3(self, F):
        F = np.ascontiguousarray(F, dtype=self.dtype).reshape(3, 3)
        U = np.zeros((3, 3), self.dtype); s = np.zeros(3, self.dtype); V = np.zeros((3, 3), self.dtype)
        self.lib.orc_svd3(self._a(F), self._a(U), self._a(s), self._a(V))
        return U, s, V

    def mu_lam_bulk(self, E, nu):
        n = E.shape[0]
        mu = np.zeros(n, self.dtype); lam = np.zeros(n, self.dtype); bulk = np.zeros(n, self.dtype)
        self.lib.orc_mu_lam_bulk(_I64(n), self._a(E), self._a(nu), self._a(mu), self._a(lam), self._a(bulk))
        return mu, lam, bulk

    def geostatic_F(self, x, F, mu, lam, density, gravity, z_top, K0, planestrain=False):
        fn = self.lib.orc_geostatic_F_planestrain if planestrain else self.lib.orc_geostatic_F
        fn(_I64(x.shape[0]), self._a(x), self._a(F), self._a(mu), self._a(lam), self._a(density),
           self.R(gravity), self.R(z_top), self.R(K0))

    def compute_stress_from_F_trial(self, activeLabel, materialLabel, particlePosition, particleVelocity,
                                    initialPhaseChangePosition, initialPhaseChangeVelocity, particle_F,
                                    particle_F_trial, mu, lam, yield_stress, hardening, softening,
                                    particle_density, strainCriteria, efficiency, eta_shear, eta_bulk,
                                    particle_C, particle_stress, particle_accumulated_strain,
                                    particle_damage, constitutive_model, alpha):
        """mpmRoutines.py:229-312 (argument order of the reference kernel)."""
        self.lib.orc_compute_stress(
            _I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel),
            self._a(particlePosition), self._a(particleVelocity), self._a(initialPhaseChangePosition),
            self._a(initialPhaseChangeVelocity), self._a(particle_F), self._a(particle_F_trial),
            self._a(mu), self._a(lam), self._a(yield_stress), self._a(hardening), self._a(softening),
            self._a(particle_density), self._a(strainCriteria), self.R(efficiency), self._a(eta_shear),
            self._a(eta_bulk), self._a(particle_C), self._a(particle_stress),
            self._a(particle_accumulated_strain), self._a(particle_damage), _I(int(constitutive_model)),
            self._a(alpha))

    def p2g_apic_with_stress(self, activeLabel, materialLabel, particle_stress, particle_x, particle_v,
                             particle_C, particle_vol, particle_mass, dx, inv_dx, minBounds, rpic_damping,
                             grid_m, grid_v_in, dt):
        """mpmRoutines.py:485-569; returns the status bits (1 = out-of-grid node skipped)."""
        return self.lib.orc_p2g(
            _I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel), self._a(particle_stress),
            self._a(particle_x), self._a(particle_v), self._a(particle_C), self._a(particle_vol),
            self._a(particle_mass), self.R(dx), self.R(inv_dx), self._v3(minBounds), self.R(rpic_damping),
            self._dims(grid_m.shape), self._a(grid_m), self._a(grid_v_in), self.R(dt))

    def grid_normalization_and_gravity(self, grid_m, grid_v_in, grid_v_out, gravity, dt):
        self.lib.orc_grid_normalize(_I64(grid_m.size), self._a(grid_m), self._a(grid_v_in),
                                    self._a(grid_v_out), self._v3(gravity), self.R(dt))

    def add_damping_via_grid(self, grid_v_out, scale):
        self.lib.orc_grid_damping(_I64(grid_v_out.size // 3), self._a(grid_v_out), self.R(scale))

    def grid_bc(self, grid_v_out, bc, friction, restitution, dt, gmag, pad):
        code = BC_CODES[bc] if isinstance(bc, str) else int(bc)
        self.lib.orc_grid_bc(self._dims(grid_v_out.shape[:3]), self._a(grid_v_out), _I(code),
                             self.R(friction), self.R(restitution), self.R(dt), self.R(gmag), _I(int(pad)))

    def g2p(self, dt, activeLabel, materialLabel, particle_x, particle_v, particle_C, particle_F,
            particle_F_trial, particle_cov, inv_dx, grid_v_out, update_cov_with_F, minBounds):
        """mpmRoutines.py:715-802."""
        return self.lib.orc_g2p(
            _I64(activeLabel.shape[0]), self.R(dt), self._i(activeLabel), self._i(materialLabel),
            self._a(particle_x), self._a(particle_v), self._a(particle_C), self._a(particle_F),
            self._a(particle_F_trial), self._a(particle_cov), self.R(inv_dx),
            self._dims(grid_v_out.shape[:3]), self._a(grid_v_out), _I(int(bool(update_cov_with_F))),
            self._v3(minBounds))

    def accumulate_cell_divergence(self, activeLabel, materialLabel, particle_x, particle_C, particle_vol,
                                   inv_dx, minBounds, cell_div_v_weighted, cell_vol_sum):
        return self.lib.orc_vlc_accumulate(
            _I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel), self._a(particle_x),
            self._a(particle_C), self._a(particle_vol), self.R(inv_dx), self._v3(minBounds),
            self._dims(cell_vol_sum.shape), self._a(cell_div_v_weighted), self._a(cell_vol_sum))

    def apply_volumetric_locking_correction(self, activeLabel, materialLabel, particle_x, particle_C, inv_dx,
                                            minBounds, cell_div_v_weighted, cell_vol_sum):
        return self.lib.orc_vlc_apply(
            _I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel), self._a(particle_x),
            self._a(particle_C), self.R(inv_dx), self._v3(minBounds), self._dims(cell_vol_sum.shape),
            self._a(cell_div_v_weighted), self._a(cell_vol_sum))

    def deactivate_and_teleport_xpbd_below_datum(self, particle_x, particle_v, activeLabel, materialLabel,
                                                 z_datum, teleport_distance):
        self.lib.orc_teleport(_I64(activeLabel.shape[0]), self._a(particle_x), self._a(particle_v),
                              self._i(activeLabel), self._i(materialLabel), self.R(z_datum),
                              self.R(teleport_distance))

    def creep_by_damage_with_baseline(self, materialLabel, damage, ys, ys_base, dt, base_creep, damage_creep,
                                      damage_exponent):
        self.lib.orc_creep(_I64(materialLabel.shape[0]), self._i(materialLabel), self._a(damage), self._a(ys),
                           self._a(ys_base), self.R(dt), self.R(base_creep), self.R(damage_creep),
                           self.R(damage_exponent))

    # -- XPBD -----------------------------------------------------------------
    def hash_build(self, x, cell_width, dims=HASH_DIMS):
        """Restated wp.HashGrid.build; positions are hashed in float32 as in Warp."""
        x32 = np.ascontiguousarray(x, dtype=np.float32)
        n = x32.shape[0]
        nc = int(np.prod(dims))
        hg = types.SimpleNamespace(
            dims=tuple(int(d) for d in dims), cell_width=float(np.float32(cell_width)),
            point_cells=np.zeros(n, np.int32), point_ids=np.zeros(n, np.int32),
            cell_starts=np.zeros(nc, np.int32), cell_ends=np.zeros(nc, np.int32))
        self.lib.orc_hash_build(_I64(n), x32.ctypes.data_as(_P), ctypes.c_float(cell_width),
                                self._dims(dims), self._i(hg.point_cells), self._i(hg.point_ids),
                                self._i(hg.cell_starts), self._i(hg.cell_ends))
        return hg

    def reset_mpm_contact_labels(self, activeLabel, materialLabel):
        self.lib.orc_reset_labels(_I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel))

    def integrateParticlesXPBD(self, activeLabel, materialLabel, x, v, gravity, dt, v_max):
        self.lib.orc_integrate_xpbd(_I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel),
                                    self._a(x), self._a(v), self._v3(gravity), self.R(dt), self.R(v_max))

    def my_solve_particle_bound_contacts(self, activeLabel, materialLabel, particle_x, particle_v, mass,
                                         particle_radius, mu, thr, static_mu, minbounds, maxbounds, dt,
                                         relaxation, delta):
        self.lib.orc_bound_contacts(
            _I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel), self._a(particle_x),
            self._a(particle_v), self._a(mass), self._a(particle_radius), self.R(mu), self.R(thr),
            self.R(static_mu), self._v3(minbounds), self._v3(maxbounds), self.R(dt), self.R(relaxation),
            self._a(delta))

    def my_solve_particle_particle_contacts(self, activeLabel, materialLabel, hg, particle_x, particle_v,
                                            particle_mass, particle_radius, k_mu, thr, static_mu, k_cohesion,
                                            max_radius, dt, relaxation, lock, deltas):
        self.lib.orc_particle_contacts(
            _I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel), self._dims(hg.dims),
            self._i(hg.cell_starts), self._i(hg.cell_ends), self._i(hg.point_ids), ctypes.c_float(hg.cell_width),
            self._a(particle_x), self._a(particle_v), self._a(particle_mass), self._a(particle_radius),
            self.R(k_mu), self.R(thr), self.R(static_mu), self.R(k_cohesion), self.R(max_radius), self.R(dt),
            self.R(relaxation), _I(int(lock)), self._a(deltas))

    def my_apply_particle_deltas(self, activeLabel, materialLabel, x_orig, x_pred, delta, dt, v_max, x_out, v_out):
        self.lib.orc_apply_deltas(_I64(activeLabel.shape[0]), self._i(activeLabel), self._a(x_orig),
                                  self._a(x_pred), self._a(delta), self.R(dt), self.R(v_max), self._a(x_out),
                                  self._a(v_out))

    def apply_mpm_contact_impulses(self, activeLabel, materialLabel, x_orig, v_orig, x_final, v_final, dt,
                                   v_max, coupling_strength, xpbd_only, v_out):
        self.lib.orc_mpm_impulses(_I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel),
                                  self._a(x_orig), self._a(v_orig), self._a(x_final), self.R(dt), self.R(v_max),
                                  self.R(coupling_strength), _I(int(xpbd_only)), self._a(v_out))

    def sleepParticles(self, activeLabel, materialLabel, sleepThreshold, radius, prev, after, dist, dt):
        counts = np.zeros(2, np.int32)
        self.lib.orc_sleep(_I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel),
                           self.R(sleepThreshold), self._a(radius), self._a(prev), self._a(after),
                           self._a(dist), self.R(dt), self._i(counts))
        return int(counts[0]), int(counts[1])

    def swellParticlesType2(self, activeLabel, materialLabel, x_init, x, radius, factor, factor_max, swellR, baseR):
        self.lib.orc_swell(_I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel),
                           self._a(x_init), self._a(x), self._a(radius), self.R(factor), self.R(factor_max),
                           self._a(swellR), self._a(baseR))

    def stats(self, activeLabel, materialLabel, v, radius, damage):
        out = np.zeros(7, np.float64)
        self.lib.orc_stats(_I64(activeLabel.shape[0]), self._i(activeLabel), self._i(materialLabel),
                           self._a(v), self._a(radius), self._a(damage), out.ctypes.data_as(_P))
        return out


# --------------------------------------------------------------------------
# state container + launch-order restatement
# --------------------------------------------------------------------------
class OracleState(types.SimpleNamespace):
    """Flat bag of reference-named numpy arrays + scalars for the oracle."""

    def copy(self):
        out = OracleState()
        for k, v in self.__dict__.items():
            setattr(out, k, v.copy() if isinstance(v, np.ndarray) else v)
        return out

    def astype(self, dtype):
        out = OracleState()
        for k, v in self.__dict__.items():
            if isinstance(v, np.ndarray) and v.dtype.kind == "f":
                v = np.ascontiguousarray(v.astype(dtype))
            elif isinstance(v, np.ndarray):
                v = v.copy()
            setattr(out, k, v)
        return out


def build_state(o: Oracle, x, vol, args, dx, minBounds, gridDims, props=None, limit=None) -> OracleState:
    """Restates the driver's set-up (runMPMYDW.py:194-489) on the CPU for the
    oracle: materials from args (or per-particle ``props``), Lame constants,
    mass, geostatic or identity F, radii.  ``limit`` keeps the first particles."""
    props = props or {}
    dt_ = o.dtype
    x = np.ascontiguousarray(np.asarray(x, dt_)[:limit])
    n = x.shape[0]
    vol = np.ascontiguousarray(np.asarray(vol, dt_)[:n])
    arr = lambda name, default: np.ascontiguousarray(  # noqa: E731
        (np.asarray(props[name], dt_)[:n] if name in props else np.full(n, default, dt_)))
    s = OracleState()
    s.particle_x = x
    s.particle_v = np.zeros((n, 3), dt_)
    s.particle_vol = vol
    s.particle_density = arr("density", args.density)
    s.particle_mass = np.ascontiguousarray((s.particle_density * vol).astype(dt_))
    s.particle_radius = np.ascontiguousarray((vol.astype(np.float32) ** (1 / 3) * np.pi / 6).astype(dt_))
    s.activeLabel = np.ones(n, np.int32)
    s.materialLabel = np.ones(n, np.int32)
    s.mu, s.lam, _ = o.mu_lam_bulk(arr("E", args.E), arr("nu", args.nu))
    for name, key in (("ys", "ys"), ("alpha", "alpha"), ("hardening", "hardening"), ("softening", "softening"),
                      ("eta_shear", "eta_shear"), ("eta_bulk", "eta_bulk"), ("strainCriteria", "strainCriteria")):
        setattr(s, name, arr(key, getattr(args, key)))
    s.particle_F = np.zeros((n, 3, 3), dt_)
    if args.initialise_geostatic:
        z_top = float(np.max(x[:, 2])) if args.z_top is None else float(args.z_top)
        o.geostatic_F(x, s.particle_F, s.mu, s.lam, s.particle_density, abs(args.gravity), z_top, args.K0,
                      planestrain=args.boundaryCondition == "plane_strain_y_global")
    else:
        s.particle_F[:] = np.eye(3, dtype=dt_)
    s.particle_F_trial = s.particle_F.copy()
    s.particle_stress = np.zeros((n, 3, 3), dt_)
    s.particle_C = np.zeros((n, 3, 3), dt_)
    s.particle_cov = np.zeros(6 * n, dt_)
    s.particle_accumulated_strain = np.zeros(n, dt_)
    s.particle_damage = arr("damage", 0.0)
    s.particle_x_initial_xpbd = np.full((n, 3), 1e6, dt_)
    s.particle_v_initial_xpbd = np.zeros((n, 3), dt_)
    dims = tuple(int(g) for g in gridDims)
    s.grid_m = np.zeros(dims, dt_)
    s.grid_v_in = np.zeros(dims + (3,), dt_)
    s.grid_v_out = np.zeros(dims + (3,), dt_)
    s.cell_div_v_weighted = np.zeros(dims, dt_)
    s.cell_vol_sum = np.zeros(dims, dt_)
    s.dx, s.invdx, s.dt = float(dx), 1.0 / float(dx), float(args.dt)
    s.minBounds = np.asarray(minBounds, dt_)
    s.gravity = np.asarray([0.0, 0.0, args.gravity], dt_)
    s.rpic_damping, s.grid_v_damping_scale = args.rpic_damping, args.grid_v_damping_scale
    s.boundaryCondition, s.boundFriction, s.boundRestitution = args.boundaryCondition, args.boundFriction, args.boundRestitution
    s.boundaryPadding = 2
    s.update_cov, s.volumetric_locking_correction = args.update_cov, args.volumetric_locking_correction
    s.eff, s.constitutive_model = args.eff, args.constitutive_model
    return s


def mpm_step(o: Oracle, s: OracleState):
    """utils/simulationRoutines.py:6-293 mpmSimulationStep, in launch order."""
    s.grid_m[...] = 0
    s.grid_v_in[...] = 0
    s.grid_v_out[...] = 0
    o.compute_stress_from_F_trial(
        s.activeLabel, s.materialLabel, s.particle_x, s.particle_v, s.particle_x_initial_xpbd,
        s.particle_v_initial_xpbd, s.particle_F, s.particle_F_trial, s.mu, s.lam, s.ys, s.hardening,
        s.softening, s.particle_density, s.strainCriteria, s.eff, s.eta_shear, s.eta_bulk, s.particle_C,
        s.particle_stress, s.particle_accumulated_strain, s.particle_damage, s.constitutive_model, s.alpha)
    st = o.p2g_apic_with_stress(s.activeLabel, s.materialLabel, s.particle_stress, s.particle_x, s.particle_v,
                                s.particle_C, s.particle_vol, s.particle_mass, s.dx, s.invdx, s.minBounds,
                                s.rpic_damping, s.grid_m, s.grid_v_in, s.dt)
    o.grid_normalization_and_gravity(s.grid_m, s.grid_v_in, s.grid_v_out, s.gravity, s.dt)
    if s.grid_v_damping_scale < 1.0:
        o.add_damping_via_grid(s.grid_v_out, s.grid_v_damping_scale)
    if s.boundaryCondition in BC_CODES:
        o.grid_bc(s.grid_v_out, s.boundaryCondition, s.boundFriction, s.boundRestitution, s.dt,
                  abs(float(s.gravity[2])), s.boundaryPadding)
    st |= o.g2p(s.dt, s.activeLabel, s.materialLabel, s.particle_x, s.particle_v, s.particle_C, s.particle_F,
                s.particle_F_trial, s.particle_cov, s.invdx, s.grid_v_out, s.update_cov, s.minBounds)
    if s.volumetric_locking_correction:
        s.cell_div_v_weighted[...] = 0
        s.cell_vol_sum[...] = 0
        st |= o.accumulate_cell_divergence(s.activeLabel, s.materialLabel, s.particle_x, s.particle_C,
                                           s.particle_vol, s.invdx, s.minBounds, s.cell_div_v_weighted,
                                           s.cell_vol_sum)
        st |= o.apply_volumetric_locking_correction(s.activeLabel, s.materialLabel, s.particle_x, s.particle_C,
                                                    s.invdx, s.minBounds, s.cell_div_v_weighted, s.cell_vol_sum)
    return st


def xpbd_step(o: Oracle, s: OracleState, xpbd_only: bool = False):
    """utils/simulationRoutines.py:295-526 xpbdSimulationStep, in launch order."""
    hg = o.hash_build(s.particle_x, s.dx)
    s.particle_x_integrated[...] = s.particle_x
    s.particle_v_integrated[...] = s.particle_v
    o.integrateParticlesXPBD(s.activeLabel, s.materialLabel, s.particle_x_integrated, s.particle_v_integrated,
                             s.gravity, s.dtxpbd, s.particle_v_max)
    if s.mpm_contact_transition_lock and not xpbd_only:
        o.reset_mpm_contact_labels(s.activeLabel, s.materialLabel)
    for _ in range(int(s.xpbd_iterations)):
        s.particle_delta[...] = 0
        o.my_solve_particle_bound_contacts(
            s.activeLabel, s.materialLabel, s.particle_x_integrated, s.particle_v_integrated, s.particle_mass,
            s.particle_radius, s.dynamicParticleFriction, s.staticVelocityThreshold, s.staticParticleFriction,
            s.minBoundsXPBD, s.maxBoundsXPBD, s.dtxpbd, s.xpbd_relaxation, s.particle_delta)
        lock = s.mpm_contact_transition_lock if not xpbd_only else 0
        o.my_solve_particle_particle_contacts(
            s.activeLabel, s.materialLabel, hg, s.particle_x_integrated, s.particle_v_integrated,
            s.particle_mass, s.particle_radius, s.dynamicParticleFriction, s.staticVelocityThreshold,
            s.staticParticleFriction, s.particle_cohesion, s.max_radius, s.dtxpbd, s.xpbd_relaxation, lock,
            s.particle_delta)
        s.particle_v_deltaInt[...] = s.particle_v_integrated
        s.particle_x_deltaInt[...] = s.particle_x_integrated
        o.my_apply_particle_deltas(s.activeLabel, s.materialLabel, s.particle_x, s.particle_x_integrated,
                                   s.particle_delta, s.dtxpbd, s.particle_v_max, s.particle_x_deltaInt,
                                   s.particle_v_deltaInt)
        s.particle_v_integrated[...] = s.particle_v_deltaInt
        s.particle_x_integrated[...] = s.particle_x_deltaInt
    tot, slp = o.sleepParticles(s.activeLabel, s.materialLabel, s.sleepThreshold, s.particle_radius, s.particle_x,
                                s.particle_x_integrated, s.particle_cumDist_xpbd, s.dtxpbd)
    s.numTotalXPBD, s.numSleepingXPBD = tot, slp
    s.particle_v_before_contact[...] = s.particle_v
    o.apply_mpm_contact_impulses(s.activeLabel, s.materialLabel, s.particle_x, s.particle_v,
                                 s.particle_x_integrated, s.particle_v_integrated, s.dtxpbd, s.particle_v_max,
                                 s.xpbd_mpm_coupling_strength, 1 if xpbd_only else 0, s.particle_v_integrated)
    s.particle_x[...] = s.particle_x_integrated
    s.particle_v[...] = s.particle_v_integrated
    if s.swellingRatio > 0:
        o.swellParticlesType2(s.activeLabel, s.materialLabel, s.particle_x_initial_xpbd, s.particle_x,
                              s.particle_radius, s.swellingActivationFactor, s.swellingMaxFactor,
                              s.particleMaxRadius, s.particleBaseRadius)
    return hg
