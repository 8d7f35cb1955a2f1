"""Substep orchestration under the reference's names (utils/simulationRoutines.py).

``mpmSimulationStep(sim, mpm, xpbd, device)`` and
``xpbdSimulationStep(sim, mpm, xpbd, device, xpbd_only=False)`` keep the
reference signatures and launch order; each kernel launch goes to libmpmw on
the current CUDA stream without host synchronisation.  The per-step
reductions of the reference driver are here too, computed on the device; the
ones that return Python numbers (``compute_mean_gpu``) synchronise, as the
reference's ``.numpy()`` reads do.

``run_mpm_substeps(sim, mpm, xpbd, nsteps)`` is the fast path for a run of
substeps with no XPBD step in between: one library call that fuses each
step's return map into the previous G2P (identical results to calling
``mpmSimulationStep`` ``nsteps`` times).
"""
from __future__ import annotations

import torch

from .. import _lib
from ..bind import grid_from_state, params_from_states, particles_from_states, status_word, stream_handle, workspace
from ..state import F32, I32

__all__ = ["mpmSimulationStep", "xpbdSimulationStep", "run_mpm_substeps", "arrayScalarMultiply",
           "velocityConvergence", "countActiveParticles", "countParticlesByType", "sum_float_array",
           "sum_float_array_active", "sum_float_array_by_material", "compute_mean_gpu", "step_stats"]


def _structs(sim, mpm, xpbd):
    return particles_from_states(sim, mpm, xpbd), grid_from_state(mpm), params_from_states(sim, mpm)


def mpmSimulationStep(sim, mpm, xpbd, device=None):
    """utils/simulationRoutines.py:6-293: zero grid, stress, P2G, grid update
    (normalise + gravity, damping if < 1, boundary condition), G2P, optional
    volumetric locking correction.  The stress and the P2G run as one kernel
    (the workspace, cached on ``mpm``, holds its SVD-path worklist)."""
    P, G, prm = _structs(sim, mpm, xpbd)
    st = status_word(sim.device)
    ws = workspace(mpm, sim.nPoints, sim.device)
    _lib.check(_lib.lib().mpmw_run_substeps(P, G, prm, 1, st.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle()),
               "mpmSimulationStep")


def run_mpm_substeps(sim, mpm, xpbd, nsteps, device=None):
    """``nsteps`` consecutive ``mpmSimulationStep`` calls as one library call."""
    P, G, prm = _structs(sim, mpm, xpbd)
    st = status_word(sim.device)
    ws = workspace(mpm, sim.nPoints, sim.device)
    _lib.check(_lib.lib().mpmw_run_substeps(P, G, prm, int(nsteps), st.data_ptr(), ws.data_ptr(), ws.numel(),
                                            stream_handle()), "run_mpm_substeps")


def xpbdSimulationStep(sim, mpm, xpbd, device=None, xpbd_only=False):
    """utils/simulationRoutines.py:295-526."""
    from .xpbdRoutines import xpbd_step
    xpbd_step(sim, mpm, xpbd, xpbd_only=xpbd_only)


# ---------------------------------------------------------------------------
# reductions (utils/simulationRoutines.py:529-675)
# ---------------------------------------------------------------------------
_STATS = {}


def step_stats(sim, mpm=None, out=None):
    """All per-step reductions in one device pass (no host sync).

    Returns a (7,) float64 CUDA tensor: [sum |v|/r over active, active count,
    sum damage over active, active MPM, active XPBD, inactive MPM,
    inactive XPBD]."""
    if out is None:
        key = sim.device
        out = _STATS.get(key)
        if out is None:
            out = torch.zeros(7, dtype=torch.float64, device=sim.device)
            _STATS[key] = out
    P = particles_from_states(sim, mpm, None)
    _lib.check(_lib.lib().mpmw_stats(P, out.data_ptr(), stream_handle()), "step_stats")
    return out


def arrayScalarMultiply(grid_A, scalar):
    """utils/simulationRoutines.py:530-535."""
    grid_A.mul_(float(scalar))


def _stats_for(activeLabel, materialLabel, particle_v=None, particle_radius=None, damage=None):
    from ..bind import Marshal, particles_struct
    n = activeLabel.numel()
    m = Marshal()
    dev = activeLabel.device
    z = torch.zeros(n, dtype=F32, device=dev)
    ones = torch.ones(n, dtype=F32, device=dev)
    P = particles_struct(n, active=m.labels(activeLabel), material=m.labels(materialLabel),
                         v=m.vec3(particle_v) if particle_v is not None else torch.zeros(3, n, dtype=F32, device=dev),
                         radius=m.scalar(particle_radius) if particle_radius is not None else ones,
                         damage=m.scalar(damage) if damage is not None else z)
    out = torch.zeros(7, dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().mpmw_stats(P, out.data_ptr(), stream_handle()), "stats")
    return out


def velocityConvergence(activeLabel, materialLabel, particle_v, particle_radius, residual):
    """utils/simulationRoutines.py:538-549: residual[0] += sum |v|/r over active."""
    out = _stats_for(activeLabel, materialLabel, particle_v, particle_radius)
    residual[0] += out[0].to(residual.dtype)


def countActiveParticles(activeLabel, sum):  # noqa: A002 - reference argument name
    """utils/simulationRoutines.py:551-558."""
    sum[0] += (activeLabel == 1).sum().to(sum.dtype)


def countParticlesByType(activeLabel, materialLabel, numActiveMPM, numActiveXPBD, numInactiveMPM,
                         numInactiveXPBD):
    """utils/simulationRoutines.py:560-587."""
    out = _stats_for(activeLabel, materialLabel)
    numActiveMPM[0] += out[3].to(numActiveMPM.dtype)
    numActiveXPBD[0] += out[4].to(numActiveXPBD.dtype)
    numInactiveMPM[0] += out[5].to(numInactiveMPM.dtype)
    numInactiveXPBD[0] += out[6].to(numInactiveXPBD.dtype)


def sum_float_array(arr, result):
    """utils/simulationRoutines.py:590-597."""
    result[0] += arr.sum(dtype=torch.float64).to(result.dtype)


def sum_float_array_active(arr, activeLabel, result, count):
    """utils/simulationRoutines.py:600-611."""
    act = activeLabel == 1
    result[0] += torch.where(act, arr, torch.zeros_like(arr)).sum(dtype=torch.float64).to(result.dtype)
    count[0] += act.sum().to(count.dtype)


def sum_float_array_by_material(arr, materialLabel, result_mpm, result_xpbd, count_mpm, count_xpbd):
    """utils/simulationRoutines.py:614-630."""
    xp = materialLabel == 2
    z = torch.zeros_like(arr)
    result_xpbd[0] += torch.where(xp, arr, z).sum(dtype=torch.float64).to(result_xpbd.dtype)
    result_mpm[0] += torch.where(~xp, arr, z).sum(dtype=torch.float64).to(result_mpm.dtype)
    count_xpbd[0] += xp.sum().to(count_xpbd.dtype)
    count_mpm[0] += (~xp).sum().to(count_mpm.dtype)


def compute_mean_gpu(arr, sim, device=None, filtered=True):
    """utils/simulationRoutines.py:633-675: mean of arr over active particles
    (filtered) or all particles; returns a Python float (synchronises)."""
    if filtered:
        act = sim.activeLabel == 1
        cnt = int(act.sum().item())
        total = float(torch.where(act, arr, torch.zeros_like(arr)).sum(dtype=torch.float64).item())
    else:
        cnt = sim.nPoints
        total = float(arr.sum(dtype=torch.float64).item())
    return total / cnt if cnt > 0 else 0.0
