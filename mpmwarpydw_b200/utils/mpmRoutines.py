"""The reference's MPM kernel surface (utils/mpmRoutines.py), backed by libmpmw.

Every kernel of the reference is a module-level callable here with the same
name and the same positional argument order, so a reference call site

    wp.launch(kernel=mpmRoutines.g2p, dim=sim.nPoints, inputs=[...], device=device)

becomes ``launch(mpmRoutines.g2p, sim.nPoints, inputs=[...])`` (see
:func:`launch`) or a direct call ``mpmRoutines.g2p(*inputs)``.  Arguments are
CUDA tensors in the reference shapes ((N, 3) vec3, (N, 3, 3) mat33, (nx, ny,
nz[, 3]) grids) or the state objects' attributes, which are passed to the
library without copies.  Scalars are Python numbers / 3-tuples.  Mutation is
in place, exactly as the reference kernels mutate their wp.array arguments.

All compute runs in libmpmw.so; nothing here falls back to the CPU.
"""
from __future__ import annotations

import torch

from .. import _lib
from ..bind import Marshal, grid_struct, params_struct, particles_struct, status_word, stream_handle
from ..state import F32, I32

__all__ = [
    "launch", "compute_mu_lam_bulk_from_E_nu", "initialize_geostatic_F", "initialize_geostatic_F_planestrain",
    "compute_stress_from_F_trial", "drucker_prager_return_mapping", "kirchoff_stress", "p2g_apic_with_stress",
    "grid_normalization_and_gravity", "add_damping_via_grid", "collideBounds", "collideBoundsPlaneStrainY",
    "collideBoundsPlaneStrainYGlobal", "collideBoundsAbsorbing", "collideBoundsRestitution",
    "collideBoundsGradualFriction", "g2p", "accumulate_cell_divergence", "apply_volumetric_locking_correction",
    "deactivate_and_teleport_xpbd_below_datum", "creep_by_damage_with_baseline", "set_mat33_to_identity",
    "set_mat33_to_copy", "add_identity_to_mat33", "subtract_identity_to_mat33", "add_vec3_to_vec3",
    "set_value_to_float_array", "set_value_to_int_array", "get_float_array_product",
]


def launch(kernel, dim=None, inputs=(), outputs=(), device=None, stream=None):
    """``wp.launch`` stand-in: calls ``kernel(*inputs, *outputs)``.

    ``dim`` is implied by the array arguments (the library launches one thread
    per particle / node) and is accepted for call-site compatibility."""
    return kernel(*inputs, *outputs)


def _dev(*ts):
    for t in ts:
        if isinstance(t, torch.Tensor):
            return t.device
    return torch.device("cuda", torch.cuda.current_device())


def _call(fn, *args, what):
    _lib.check(fn(*args), what)


# ---------------------------------------------------------------------------
# set-up kernels
# ---------------------------------------------------------------------------
def compute_mu_lam_bulk_from_E_nu(E, nu, mu, lam, bulk):
    """utils/mpmRoutines.py:206-226."""
    m = Marshal()
    e, v = m.scalar(E), m.scalar(nu)
    mo, lo, bo = m.scalar(mu, out=True), m.scalar(lam, out=True), m.scalar(bulk, out=True)
    _call(_lib.lib().mpmw_mu_lam_bulk, e.numel(), e.data_ptr(), v.data_ptr(), mo.data_ptr(), lo.data_ptr(),
          bo.data_ptr(), stream_handle(), what="compute_mu_lam_bulk_from_E_nu")
    m.finish()


def _geostatic(particle_x, particle_F, mu, lam, density, gravity, z_top, K0, planestrain):
    m = Marshal()
    x = m.vec3(particle_x)
    F = m.mat33(particle_F, out=True)
    mu_, lam_, rho = m.scalar(mu), m.scalar(lam), m.scalar(density)
    _call(_lib.lib().mpmw_geostatic_F, x.shape[1], x.data_ptr(), F.data_ptr(), mu_.data_ptr(), lam_.data_ptr(),
          rho.data_ptr(), float(gravity), float(z_top), float(K0), int(planestrain), stream_handle(),
          what="initialize_geostatic_F")
    m.finish()


def initialize_geostatic_F(particle_x, particle_F, mu, lam, density, gravity, z_top, K0):
    """utils/mpmRoutines.py:51-124."""
    _geostatic(particle_x, particle_F, mu, lam, density, gravity, z_top, K0, 0)


def initialize_geostatic_F_planestrain(particle_x, particle_F, mu, lam, density, g, z_top, K0):
    """utils/mpmRoutines.py:127-203."""
    _geostatic(particle_x, particle_F, mu, lam, density, g, z_top, K0, 1)


# ---------------------------------------------------------------------------
# substep kernels
# ---------------------------------------------------------------------------
def compute_stress_from_F_trial(activeLabel, materialLabel, particlePosition, particleVelocity,
                                initialPhaseChangePosition, initialPhaseChangeVelocity, particle_F,
                                particle_F_trial, mu, lam, yield_stress, hardening, softening, particle_density,
                                strainCriteria, efficiency, eta_shear, eta_bulk, particle_C, particle_stress,
                                particle_accumulated_strain, particle_damage, constitutive_model, alpha,
                                stress_mode=0):
    """utils/mpmRoutines.py:229-312 (return map :314-453, Kirchhoff :456-471).

    ``stress_mode`` (not in the reference): 0 lets clearly elastic particles
    take the SVD-free log-strain path (same stress, less FP32 rounding), 1
    runs the SVD return map for every particle."""
    m = Marshal()
    P = particles_struct(
        activeLabel.numel(), active=m.labels(activeLabel), material=m.labels(materialLabel, out=True),
        x=m.vec3(particlePosition), v=m.vec3(particleVelocity, out=True),
        x_pc=m.vec3(initialPhaseChangePosition, out=True), v_pc=m.vec3(initialPhaseChangeVelocity, out=True),
        F=m.mat33(particle_F, out=True), F_trial=m.mat33(particle_F_trial), mu=m.scalar(mu, out=True),
        lam=m.scalar(lam, out=True), ys=m.scalar(yield_stress, out=True), hardening=m.scalar(hardening),
        softening=m.scalar(softening), density=m.scalar(particle_density), strain_criteria=m.scalar(strainCriteria),
        eta_shear=m.scalar(eta_shear), eta_bulk=m.scalar(eta_bulk), C=m.mat33(particle_C),
        stress=m.sym33(particle_stress, out=True), acc_strain=m.scalar(particle_accumulated_strain, out=True),
        damage=m.scalar(particle_damage, out=True), alpha=m.scalar(alpha, out=True))
    prm = params_struct(eff=efficiency, constitutive_model=constitutive_model, stress_mode=stress_mode)
    dev = _dev(activeLabel)
    _call(_lib.lib().mpmw_stress, P, prm, status_word(dev).data_ptr(), stream_handle(),
          what="compute_stress_from_F_trial")
    m.finish()


def drucker_prager_return_mapping(*args, **kw):
    """utils/mpmRoutines.py:314-453 is a @wp.func inlined into
    compute_stress_from_F_trial; it has no launchable form of its own.  The
    library runs it inside the stress kernels (mpmw_stress, mpmw_g2p_stress)."""
    raise TypeError("drucker_prager_return_mapping is a device function; call compute_stress_from_F_trial")


def kirchoff_stress(*args, **kw):
    """utils/mpmRoutines.py:456-471 is a @wp.func inlined into the stress kernel."""
    raise TypeError("kirchoff_stress is a device function; call compute_stress_from_F_trial")


def p2g_apic_with_stress(activeLabel, materialLabel, particle_stress, particle_x, particle_v, particle_C,
                         particle_vol, particle_mass, dx, inv_dx, minBounds, rpic_damping, grid_m, grid_v_in, dt):
    """utils/mpmRoutines.py:485-569 (accumulates into grid_m / grid_v_in)."""
    m = Marshal()
    dev = _dev(grid_m, particle_x)
    dims = tuple(grid_m.shape[:3])
    mv = m.grid_packed([(grid_m, 0), (grid_v_in, slice(1, 4))], dims, dev, out=True)
    P = particles_struct(activeLabel.numel(), active=m.labels(activeLabel), material=m.labels(materialLabel),
                         stress=m.sym33(particle_stress), x=m.vec3(particle_x), v=m.vec3(particle_v),
                         C=m.mat33(particle_C), F=m.mat33(particle_C), vol=m.scalar(particle_vol),
                         mass=m.scalar(particle_mass))
    G = grid_struct(dims, mv=mv, v=mv)
    prm = params_struct(minBounds=minBounds, dx=dx, inv_dx=inv_dx, dt=dt, rpic_damping=rpic_damping)
    _call(_lib.lib().mpmw_p2g, P, G, prm, status_word(dev).data_ptr(), stream_handle(), what="p2g_apic_with_stress")
    m.finish()


def _grid_op(op, grid_m, grid_v_in, grid_v_out, prm):
    m = Marshal()
    dev = _dev(grid_v_out)
    dims = tuple(grid_v_out.shape[:3])
    mv = m.grid_packed([(grid_m, 0), (grid_v_in, slice(1, 4))], dims, dev) if grid_m is not None else None
    v = m.grid_packed([(grid_v_out, slice(0, 3))], dims, dev, out=True)
    G = grid_struct(dims, mv=mv if mv is not None else v, v=v)
    _call(_lib.lib().mpmw_grid_op, G, prm, op, stream_handle(), what="grid op")
    m.finish()


def grid_normalization_and_gravity(grid_m, grid_v_in, grid_v_out, gravity, dt):
    """utils/mpmRoutines.py:690-704."""
    _grid_op(0, grid_m, grid_v_in, grid_v_out, params_struct(gravity=gravity, dt=dt))


def add_damping_via_grid(grid_v_out, scale):
    """utils/mpmRoutines.py:706-711."""
    _grid_op(1, None, None, grid_v_out, params_struct(grid_v_damping_scale=scale))


def _bc(code, grid_v_out, friction=0.0, restitution=0.0, dt=0.0, gmag=0.0, pad=0):
    prm = params_struct(boundary_condition=code, bound_friction=friction, bound_restitution=restitution, dt=dt,
                        gravity=(0.0, 0.0, gmag), boundary_padding=pad)
    _grid_op(2, None, None, grid_v_out, prm)


def collideBounds(grid_v_out, grid_dim_x, grid_dim_y, grid_dim_z, friction_coefficient, dt, gravity_magnitude,
                  boundary_padding):
    """utils/mpmRoutines.py:942-993."""
    _bc("friction", grid_v_out, friction_coefficient, 0.0, dt, gravity_magnitude, boundary_padding)


def collideBoundsPlaneStrainY(grid_v_out, grid_dim_x, grid_dim_y, grid_dim_z, friction_coefficient, dt,
                              gravity_magnitude, boundary_padding):
    """utils/mpmRoutines.py:996-1063."""
    _bc("plane_strain_y", grid_v_out, friction_coefficient, 0.0, dt, gravity_magnitude, boundary_padding)


def collideBoundsPlaneStrainYGlobal(grid_v_out, grid_dim_x, grid_dim_y, grid_dim_z, friction_coefficient, dt,
                                    gravity_magnitude, boundary_padding):
    """utils/mpmRoutines.py:1066-1125."""
    _bc("plane_strain_y_global", grid_v_out, friction_coefficient, 0.0, dt, gravity_magnitude, boundary_padding)


def collideBoundsAbsorbing(grid_v_out, grid_dim_x, grid_dim_y, grid_dim_z, boundary_padding):
    """utils/mpmRoutines.py:1128-1178."""
    _bc("absorbing", grid_v_out, pad=boundary_padding)


def collideBoundsRestitution(grid_v_out, grid_dim_x, grid_dim_y, grid_dim_z, restitution, friction_coefficient, dt,
                             gravity_magnitude, boundary_padding):
    """utils/mpmRoutines.py:1181-1261."""
    _bc("restitution", grid_v_out, friction_coefficient, restitution, dt, gravity_magnitude, boundary_padding)


def collideBoundsGradualFriction(grid_v_out, grid_dim_x, grid_dim_y, grid_dim_z, friction_coefficient, dt,
                                 gravity_magnitude, boundary_padding):
    """utils/mpmRoutines.py:1263-1362."""
    _bc("friction_gradual", grid_v_out, friction_coefficient, 0.0, dt, gravity_magnitude, boundary_padding)


def g2p(dt, activeLabel, materialLabel, particle_x, particle_v, particle_C, particle_F, particle_F_trial,
        particle_cov, inv_dx, grid_v_out, update_cov_with_F, minBounds):
    """utils/mpmRoutines.py:715-802."""
    m = Marshal()
    dev = _dev(grid_v_out, particle_x)
    dims = tuple(grid_v_out.shape[:3])
    v4 = m.grid_packed([(grid_v_out, slice(0, 3))], dims, dev)
    P = particles_struct(activeLabel.numel(), active=m.labels(activeLabel), material=m.labels(materialLabel),
                         x=m.vec3(particle_x, out=True), v=m.vec3(particle_v, out=True),
                         C=m.mat33(particle_C, out=True), F=m.mat33(particle_F),
                         F_trial=m.mat33(particle_F_trial, out=True),
                         cov=m.scalar(particle_cov, out=True) if update_cov_with_F else None)
    G = grid_struct(dims, mv=v4, v=v4)
    prm = params_struct(dt=dt, inv_dx=inv_dx, minBounds=minBounds, update_cov=update_cov_with_F)
    _call(_lib.lib().mpmw_g2p, P, G, prm, status_word(dev).data_ptr(), stream_handle(), what="g2p")
    m.finish()


def accumulate_cell_divergence(activeLabel, materialLabel, particle_x, particle_C, particle_vol, inv_dx,
                               minBounds, cell_div_v_weighted, cell_vol_sum):
    """utils/mpmRoutines.py:817-856 (accumulates into the cell arrays)."""
    m = Marshal()
    dev = _dev(particle_x)
    dims = tuple(cell_vol_sum.shape[:3])
    P = particles_struct(activeLabel.numel(), active=m.labels(activeLabel), material=m.labels(materialLabel),
                         x=m.vec3(particle_x), C=m.mat33(particle_C), vol=m.scalar(particle_vol))
    cd, cv = m.scalar(cell_div_v_weighted, out=True), m.scalar(cell_vol_sum, out=True)
    G = grid_struct(dims, cell_div=cd, cell_vol=cv)
    prm = params_struct(inv_dx=inv_dx, minBounds=minBounds)
    _call(_lib.lib().mpmw_vlc_phase, P, G, prm, 0,
          status_word(dev).data_ptr(), stream_handle(), what="accumulate_cell_divergence")
    m.finish()


def apply_volumetric_locking_correction(activeLabel, materialLabel, particle_x, particle_C, inv_dx, minBounds,
                                        cell_div_v_weighted, cell_vol_sum):
    """utils/mpmRoutines.py:859-911."""
    m = Marshal()
    dev = _dev(particle_x)
    dims = tuple(cell_vol_sum.shape[:3])
    P = particles_struct(activeLabel.numel(), active=m.labels(activeLabel), material=m.labels(materialLabel),
                         x=m.vec3(particle_x), C=m.mat33(particle_C, out=True))
    cd, cv = m.scalar(cell_div_v_weighted), m.scalar(cell_vol_sum)
    G = grid_struct(dims, cell_div=cd, cell_vol=cv)
    prm = params_struct(inv_dx=inv_dx, minBounds=minBounds)
    _call(_lib.lib().mpmw_vlc_phase, P, G, prm, 1,
          status_word(dev).data_ptr(), stream_handle(), what="apply_volumetric_locking_correction")
    m.finish()


def deactivate_and_teleport_xpbd_below_datum(particle_x, particle_v, activeLabel, materialLabel, z_datum,
                                             teleport_distance):
    """utils/mpmRoutines.py:1446-1475."""
    m = Marshal()
    P = particles_struct(activeLabel.numel(), x=m.vec3(particle_x, out=True), v=m.vec3(particle_v, out=True),
                         active=m.labels(activeLabel, out=True), material=m.labels(materialLabel))
    _call(_lib.lib().mpmw_teleport, P, float(z_datum), float(teleport_distance), stream_handle(),
          what="deactivate_and_teleport_xpbd_below_datum")
    m.finish()


def creep_by_damage_with_baseline(materialLabel, damage, ys, ys_base, dt, base_creep, damage_creep,
                                  damage_exponent):
    """utils/mpmRoutines.py:3-21."""
    m = Marshal()
    P = particles_struct(materialLabel.numel(), material=m.labels(materialLabel), damage=m.scalar(damage),
                         ys=m.scalar(ys, out=True))
    yb = m.scalar(ys_base)
    _call(_lib.lib().mpmw_creep, P, yb.data_ptr(), float(dt), float(base_creep), float(damage_creep),
          float(damage_exponent), stream_handle(), what="creep_by_damage_with_baseline")
    m.finish()


# ---------------------------------------------------------------------------
# array utilities (utils/mpmRoutines.py:635-688): plain tensor operations
# ---------------------------------------------------------------------------
def set_mat33_to_identity(target_array):
    target_array.copy_(torch.eye(3, dtype=target_array.dtype, device=target_array.device).expand_as(target_array))


def set_mat33_to_copy(source_array, target_array):
    target_array.copy_(source_array)


def add_identity_to_mat33(target_array):
    target_array.add_(torch.eye(3, dtype=target_array.dtype, device=target_array.device))


def subtract_identity_to_mat33(target_array):
    target_array.sub_(torch.eye(3, dtype=target_array.dtype, device=target_array.device))


def add_vec3_to_vec3(first_array, second_array):
    first_array.add_(second_array)


def set_value_to_float_array(target_array, value):
    target_array.fill_(float(value))


def set_value_to_int_array(target_array, value):
    target_array.fill_(int(value))


def get_float_array_product(arrayA, arrayB, arrayC):
    torch.mul(arrayA, arrayB, out=arrayC)
