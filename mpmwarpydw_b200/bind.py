"""Marshalling between torch tensors / state objects and the libmpmw C ABI.

Two ways in:
  * state objects (SimState/MPMState/XPBDState): their SoA storage is passed
    to the library by pointer, no copies (:func:`particles_from_states`);
  * arbitrary reference-shaped tensors (the per-kernel surface in
    ``utils.mpmRoutines``): each is mapped to SoA storage, zero-copy when it
    already is a view of SoA storage (every state attribute is), otherwise via
    a temporary that is copied back after the call (:class:`Marshal`).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .state import F32, I32, full_to_sym6, sym6_to_full

_STATUS = {}


def stream_handle(stream=None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def status_word(device) -> torch.Tensor:
    """Per-device uint32 status word (as int32 tensor) that kernels OR bits into."""
    device = torch.device(device)
    key = (device.type, device.index if device.index is not None else torch.cuda.current_device())
    t = _STATUS.get(key)
    if t is None:
        t = torch.zeros(1, dtype=I32, device=device)
        _STATUS[key] = t
    return t


def read_status(device, clear=True) -> int:
    t = status_word(device)
    v = int(t.item()) & 0xFFFFFFFF
    if clear:
        t.zero_()
    return v


STATUS_BITS = {1: "OOB", 2: "NAN", 4: "TIMEOUT"}  # MPMW_ST_* of mpmw.h


def status_names(word: int):
    """Names of the MPMW_ST_* bits set in a status word."""
    return [name for bit, name in STATUS_BITS.items() if word & bit]


class DeviceFault(RuntimeError):
    """A kernel reported a non-finite particle position (MPMW_ST_NAN)."""


def check_status(device, where: str, log=print) -> int:
    """Read and clear the device status word after a stretch of GPU work.

    A non-finite position (MPMW_ST_NAN) ends the run with DeviceFault; stencil
    nodes outside the grid (MPMW_ST_OOB, the access was skipped) and bounded
    waits that gave up (MPMW_ST_TIMEOUT, the kernel took its fallback) are
    logged.  Returns the word."""
    w = read_status(device)
    if w & 2:
        raise DeviceFault(f"{where}: a particle position became non-finite (status {status_names(w)})")
    if w:
        log(f"    warning: {where}: device status {status_names(w)}")
    return w


def ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


def _require_cuda(t, name):
    if t is not None and not t.is_cuda:
        raise ValueError(f"{name} must be a CUDA tensor (libmpmw has no CPU path)")


class Marshal:
    """Maps reference-shaped tensors onto SoA buffers for one library call."""

    def __init__(self):
        self._writebacks = []
        self.keep = []

    def _tensor(self, v, dtype, device=None):
        if isinstance(v, torch.Tensor):
            return v
        return torch.as_tensor(v, dtype=dtype, device=device or "cuda")

    def vec3(self, t, out=False):
        """(N, 3) -> (3, N) contiguous float32."""
        if t is None:
            return None
        t = self._tensor(t, F32)
        _require_cuda(t, "vec3 array")
        s = t.t() if t.dim() == 2 else t.reshape(-1, 3).t()
        if s.dtype == F32 and s.is_contiguous():
            return s
        c = s.to(F32).contiguous()
        if out:
            self._writebacks.append(lambda: t.copy_(c.t().reshape(t.shape)))
        self.keep.append(c)
        return c

    def mat33(self, t, out=False):
        """(N, 3, 3) -> (9, N) contiguous float32."""
        if t is None:
            return None
        t = self._tensor(t, F32)
        _require_cuda(t, "mat33 array")
        s = t.reshape(-1, 3, 3).permute(1, 2, 0)
        if s.dtype == F32 and s.is_contiguous():
            return s.reshape(9, -1)
        c = s.to(F32).contiguous().reshape(9, -1)
        if out:
            self._writebacks.append(lambda: t.copy_(c.reshape(3, 3, -1).permute(2, 0, 1).reshape(t.shape)))
        self.keep.append(c)
        return c

    def sym33(self, t, out=False):
        """(N, 3, 3) stress -> (6, N) symmetric storage."""
        if t is None:
            return None
        s6 = getattr(t, "_mpmw_sym6", None)
        if s6 is not None:
            if out:
                self._writebacks.append(lambda: t.copy_(sym6_to_full(s6)))
            return s6
        t = self._tensor(t, F32)
        _require_cuda(t, "stress array")
        c = full_to_sym6(t.to(F32)).contiguous()
        if out:
            self._writebacks.append(lambda: t.copy_(sym6_to_full(c).reshape(t.shape)))
        self.keep.append(c)
        return c

    def scalar(self, t, dtype=F32, out=False):
        if t is None:
            return None
        t = self._tensor(t, dtype)
        _require_cuda(t, "array")
        if t.dtype == dtype and t.is_contiguous():
            return t.reshape(-1)
        c = t.to(dtype).contiguous().reshape(-1)
        if out:
            self._writebacks.append(lambda: t.copy_(c.reshape(t.shape)))
        self.keep.append(c)
        return c

    def labels(self, t, out=False):
        return self.scalar(t, I32, out)

    def grid_packed(self, comps, dims, device, out=False):
        """comps: list of (tensor, slice) to pack into a (G, 4) float buffer.

        Zero-copy when every tensor is a component view of the same packed
        storage (MPMState.grid_m / grid_v_in / grid_v_out)."""
        bases = {id(getattr(t, "_mpmw_packed", None)) for t, _ in comps}
        base = getattr(comps[0][0], "_mpmw_packed", None)
        if base is not None and len(bases) == 1:
            return base
        buf = torch.zeros(*dims, 4, dtype=F32, device=device)
        for t, sl in comps:
            if t is None:
                continue
            buf[..., sl].copy_(torch.as_tensor(t, device=device).reshape(buf[..., sl].shape))
        if out:
            def wb():
                for t, sl in comps:
                    if t is not None:
                        t.copy_(buf[..., sl].reshape(t.shape))
            self._writebacks.append(wb)
        self.keep.append(buf)
        return buf

    def finish(self):
        for wb in self._writebacks:
            wb()
        self._writebacks.clear()


def particles_struct(n, **f) -> _lib.Particles:
    P = _lib.Particles()
    P.n = int(n)
    for name in ("x", "v", "C", "F", "F_trial", "stress", "cov", "vol", "mass", "density", "radius", "mu", "lam",
                 "ys", "alpha", "hardening", "softening", "strain_criteria", "eta_shear", "eta_bulk",
                 "acc_strain", "damage", "active", "material", "x_pc", "v_pc"):
        t = f.get(name)
        setattr(P, name, ptr(t) if t is not None else None)
    return P


# mpmw_particles_t field -> (state object: 0 sim, 1 mpm, 2 xpbd; its attribute)
PARTICLE_FIELDS = (
    ("x", 0, "particle_x"), ("v", 0, "particle_v"),
    ("C", 1, "particle_C"), ("F", 1, "particle_F"), ("F_trial", 1, "particle_F_trial"),
    ("stress", 1, "particle_stress"), ("cov", 1, "particle_cov"),
    ("vol", 0, "particle_vol"), ("mass", 0, "particle_mass"), ("density", 0, "particle_density"),
    ("radius", 0, "particle_radius"),
    ("mu", 1, "mu"), ("lam", 1, "lam"), ("ys", 1, "ys"), ("alpha", 1, "alpha"),
    ("hardening", 1, "hardening"), ("softening", 1, "softening"), ("strain_criteria", 1, "strainCriteria"),
    ("eta_shear", 1, "eta_shear"), ("eta_bulk", 1, "eta_bulk"),
    ("acc_strain", 1, "particle_accumulated_strain"), ("damage", 1, "particle_damage"),
    ("active", 0, "activeLabel"), ("material", 0, "materialLabel"),
    ("x_pc", 2, "particle_x_initial_xpbd"), ("v_pc", 2, "particle_v_initial_xpbd"),
)


def particle_storage(sim, mpm=None, xpbd=None) -> dict:
    """The state objects' SoA storage tensors by mpmw_particles_t field name
    (None where the state object or the array is absent)."""
    objs = (sim, mpm, xpbd)
    return {name: (getattr(objs[w], "_s_" + attr, None) if objs[w] is not None else None)
            for name, w, attr in PARTICLE_FIELDS}


def particles_from_states(sim, mpm=None, xpbd=None) -> _lib.Particles:
    """Zero-copy C view of the state objects' SoA storage."""
    return particles_struct(sim.nPoints, **particle_storage(sim, mpm, xpbd))


def grid_struct(dims, mv=None, v=None, cell_div=None, cell_vol=None) -> _lib.Grid:
    G = _lib.Grid()
    for i in range(3):
        G.dims[i] = int(dims[i])
    G.mv = ptr(mv) if mv is not None else None
    G.v = ptr(v) if v is not None else None
    G.cell_div = ptr(cell_div) if cell_div is not None else None
    G.cell_vol = ptr(cell_vol) if cell_vol is not None else None
    return G


def grid_from_state(mpm) -> _lib.Grid:
    return grid_struct(mpm.gridDims, mpm._grid_mv.t, mpm._grid_v.t, mpm.cell_div_v_weighted, mpm.cell_vol_sum)


def params_struct(*, minBounds=(0, 0, 0), dx=1.0, inv_dx=None, dt=0.0, gravity=(0, 0, 0), rpic_damping=0.0,
                  grid_v_damping_scale=1.1, bound_friction=0.0, bound_restitution=0.0, boundary_condition=-1,
                  boundary_padding=0, eff=0.0, update_cov=0, vlc=0, constitutive_model=1,
                  stress_mode=0) -> _lib.Params:
    P = _lib.Params()
    for i in range(3):
        P.min_bounds[i] = float(minBounds[i])
        P.gravity[i] = float(gravity[i])
    P.dx = float(dx)
    P.inv_dx = float(inv_dx if inv_dx is not None else 1.0 / dx)
    P.dt = float(dt)
    P.rpic_damping = float(rpic_damping)
    P.grid_v_damping_scale = float(grid_v_damping_scale)
    P.bound_friction = float(bound_friction)
    P.bound_restitution = float(bound_restitution)
    bc = boundary_condition
    P.boundary_condition = _lib.BC_CODES[bc] if isinstance(bc, str) else int(bc)
    P.boundary_padding = int(boundary_padding)
    P.eff = float(eff)
    P.update_cov = int(bool(update_cov))
    P.vlc = int(bool(vlc))
    P.constitutive_model = int(constitutive_model)
    P.stress_mode = int(stress_mode)
    return P


def params_from_states(sim, mpm) -> _lib.Params:
    bc = mpm.boundaryCondition
    code = _lib.BC_CODES.get(bc, -1) if isinstance(bc, str) else int(bc)
    return params_struct(minBounds=sim.minBounds, dx=sim.dx, inv_dx=sim.invdx, dt=sim.dt, gravity=sim.gravity,
                         rpic_damping=mpm.rpic_damping, grid_v_damping_scale=mpm.grid_v_damping_scale,
                         bound_friction=mpm.boundFriction, bound_restitution=mpm.boundRestitution,
                         boundary_condition=code, boundary_padding=mpm.boundaryPadding or 0, eff=mpm.eff,
                         update_cov=mpm.update_cov, vlc=mpm.volumetric_locking_correction,
                         constitutive_model=mpm.constitutive_model,
                         stress_mode=getattr(mpm, "stress_mode", 0))


def byref(x):
    return ctypes.byref(x)


def workspace(owner, n: int, device) -> torch.Tensor:
    """Device workspace for the fused substep (mpmw_workspace_bytes(n)), cached on ``owner``."""
    need = int(_lib.lib().mpmw_workspace_bytes(int(n)))
    ws = getattr(owner, "_mpmw_ws", None)
    if ws is None or ws.numel() < need:
        ws = torch.empty(max(need, 256), dtype=torch.uint8, device=device)
        owner._mpmw_ws = ws
    return ws
