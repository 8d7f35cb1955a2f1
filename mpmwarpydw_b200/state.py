"""Device storage of particle and grid state.

Every per-particle field is a CUDA tensor in component-major (SoA) layout so
that a warp reads 128 contiguous bytes per component.  The reference exposes
the same fields as array-of-structure ``wp.array`` objects
(utils/simStates.py:10-179); the descriptors below present them under the
reference names and shapes as *views* of the SoA storage:

    vec3  field  -> (N, 3)    view of a (3, N) tensor      (writes propagate)
    mat33 field  -> (N, 3, 3) view of a (9, N) tensor      (writes propagate)
    stress       -> (N, 3, 3) tensor rebuilt from the (6, N) symmetric storage on
                   every read; assigning a (N, 3, 3) array stores it (the
                   reference only ever assigns or reads it)
    scalar/label -> (N,) tensor
    grid_m / grid_v_in -> views of one (nx, ny, nz, 4) float tensor (m, m*v)
    grid_v_out         -> view of one (nx, ny, nz, 4) float tensor (v, pad)

Assigning a numpy array / tensor / list to any of these attributes copies it
into the storage, which mirrors the reference driver's ``x = wp.array(...)``.
"""
from __future__ import annotations

import numpy as np
import torch

F32 = torch.float32
I32 = torch.int32


def _to_tensor(value, dtype, device):
    if isinstance(value, torch.Tensor):
        return value.to(device=device, dtype=dtype)
    return torch.as_tensor(np.asarray(value), dtype=dtype, device=device)


def mat_view(store: torch.Tensor) -> torch.Tensor:
    """(9, N) SoA storage -> (N, 3, 3) view."""
    n = store.shape[1]
    return store.as_strided((n, 3, 3), (1, 3 * n, n), store.storage_offset())


def sym6_to_full(s6: torch.Tensor) -> torch.Tensor:
    """(6, N) xx yy zz xy xz yz -> (N, 3, 3)."""
    xx, yy, zz, xy, xz, yz = s6
    return torch.stack([torch.stack([xx, xy, xz], -1), torch.stack([xy, yy, yz], -1),
                        torch.stack([xz, yz, zz], -1)], -2)


def full_to_sym6(t: torch.Tensor) -> torch.Tensor:
    t = t.reshape(-1, 3, 3)
    return torch.stack([t[:, 0, 0], t[:, 1, 1], t[:, 2, 2], t[:, 0, 1], t[:, 0, 2], t[:, 1, 2]])


class _Field:
    kind = "scalar"

    def __set_name__(self, owner, name):
        self.name = name
        self.store = "_s_" + name

    def storage(self, obj):
        return getattr(obj, self.store, None)


class ScalarField(_Field):
    def __init__(self, dtype=F32):
        self.dtype = dtype

    def __get__(self, obj, cls=None):
        if obj is None:
            return self
        return self.storage(obj)

    def __set__(self, obj, value):
        if value is None:
            setattr(obj, self.store, None)
            return
        t = _to_tensor(value, self.dtype, obj.device).reshape(-1)
        # a contiguous device tensor of the right dtype is stored as is (aliased,
        # like assigning a wp.array); anything else is converted into a new tensor
        setattr(obj, self.store, t if t.is_contiguous() else t.contiguous())


class Vec3Field(_Field):
    kind = "vec3"

    def __get__(self, obj, cls=None):
        if obj is None:
            return self
        s = self.storage(obj)
        return None if s is None else s.t()

    def __set__(self, obj, value):
        if value is None:
            setattr(obj, self.store, None)
            return
        t = _to_tensor(value, F32, obj.device).reshape(-1, 3)
        cur = self.storage(obj)
        if cur is None or cur.shape[1] != t.shape[0]:
            cur = torch.empty(3, t.shape[0], dtype=F32, device=obj.device)
            setattr(obj, self.store, cur)
        cur.copy_(t.t())


class Mat33Field(_Field):
    kind = "mat33"

    def __get__(self, obj, cls=None):
        if obj is None:
            return self
        s = self.storage(obj)
        return None if s is None else mat_view(s)

    def __set__(self, obj, value):
        if value is None:
            setattr(obj, self.store, None)
            return
        t = _to_tensor(value, F32, obj.device).reshape(-1, 3, 3)
        cur = self.storage(obj)
        if cur is None or cur.shape[1] != t.shape[0]:
            cur = torch.empty(9, t.shape[0], dtype=F32, device=obj.device)
            setattr(obj, self.store, cur)
        cur.copy_(t.permute(1, 2, 0).reshape(9, -1))


class Sym33Field(_Field):
    kind = "sym33"

    def __get__(self, obj, cls=None):
        if obj is None:
            return self
        s = self.storage(obj)
        if s is None:
            return None
        full = sym6_to_full(s)
        full._mpmw_sym6 = s  # lets the kernel wrappers write straight into the storage
        return full

    def __set__(self, obj, value):
        if value is None:
            setattr(obj, self.store, None)
            return
        t = _to_tensor(value, F32, obj.device).reshape(-1, 3, 3)
        cur = self.storage(obj)
        if cur is None or cur.shape[1] != t.shape[0]:
            cur = torch.empty(6, t.shape[0], dtype=F32, device=obj.device)
            setattr(obj, self.store, cur)
        cur.copy_(full_to_sym6(t))


class GridField(_Field):
    """A grid-shaped float array stored as given (contiguous, on the device)."""

    def __get__(self, obj, cls=None):
        if obj is None:
            return self
        return self.storage(obj)

    def __set__(self, obj, value):
        if value is None:
            setattr(obj, self.store, None)
            return
        t = _to_tensor(value, F32, obj.device)
        setattr(obj, self.store, t if t.is_contiguous() else t.contiguous())


class GridPacked:
    """(nx, ny, nz, 4) float storage with named component views."""

    def __init__(self, dims, device):
        self.dims = tuple(int(d) for d in dims)
        self.t = torch.zeros(*self.dims, 4, dtype=F32, device=device)

    def comp(self, sl):
        v = self.t[..., sl]
        v._mpmw_packed = self.t
        return v
