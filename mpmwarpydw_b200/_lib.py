"""ctypes binding of libmpmw.so (declarations in include/mpmw.h).

The CUDA library is the only compute path: if it is missing or cannot be
loaded, :func:`lib` raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

from .build import LIB, build

_P = ctypes.c_void_p
_F = ctypes.c_float
_I = ctypes.c_int
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64

MPMW_OK = 0
ST_OOB, ST_NAN, ST_TIMEOUT = 1, 2, 4
BC_CODES = {
    "none": -1,
    "friction": 0,
    "friction_gradual": 1,
    "restitution": 2,
    "absorbing": 3,
    "plane_strain_y": 4,
    "plane_strain_y_global": 5,
}


class Particles(ctypes.Structure):
    _fields_ = [("n", _I64),
                ("x", _P), ("v", _P),
                ("C", _P), ("F", _P), ("F_trial", _P),
                ("stress", _P), ("cov", _P),
                ("vol", _P), ("mass", _P), ("density", _P), ("radius", _P),
                ("mu", _P), ("lam", _P), ("ys", _P), ("alpha", _P), ("hardening", _P), ("softening", _P),
                ("strain_criteria", _P), ("eta_shear", _P), ("eta_bulk", _P),
                ("acc_strain", _P), ("damage", _P),
                ("active", _P), ("material", _P),
                ("x_pc", _P), ("v_pc", _P)]


class Grid(ctypes.Structure):
    _fields_ = [("dims", _I32 * 3), ("mv", _P), ("v", _P), ("cell_div", _P), ("cell_vol", _P)]


class Params(ctypes.Structure):
    _fields_ = [("min_bounds", _F * 3), ("dx", _F), ("inv_dx", _F), ("dt", _F), ("gravity", _F * 3),
                ("rpic_damping", _F), ("grid_v_damping_scale", _F), ("bound_friction", _F),
                ("bound_restitution", _F), ("boundary_condition", _I32), ("boundary_padding", _I32),
                ("eff", _F), ("update_cov", _I32), ("vlc", _I32), ("constitutive_model", _I32),
                ("stress_mode", _I32)]


STRESS_AUTO, STRESS_SVD = 0, 1

MLP_IN, MLP_HID, MLP_OUT, MLP_NPARAM, MLP_PACKED_BYTES = 8, 64, 4, 9156, 20480
SURR_NSTATS = 8          # MPMW_SURR_NSTATS
SURR_D_MAX = 0.999       # MPMW_SURR_D_MAX


class XPBD(ctypes.Structure):
    _fields_ = [("x_int", _P), ("v_int", _P), ("x_dI", _P), ("v_dI", _P), ("delta", _P), ("v_before", _P),
                ("cum_dist", _P), ("base_radius", _P), ("max_radius", _P), ("counts", _P)]


class Hash(ctypes.Structure):
    _fields_ = [("dims", _I32 * 3), ("cell_width", _F), ("point_ids", _P), ("cell_starts", _P),
                ("cell_ends", _P), ("point_cells", _P)]


class XPBDParams(ctypes.Structure):
    _fields_ = [("gravity", _F * 3), ("dt", _F), ("v_max", _F), ("iterations", _I32), ("relaxation", _F),
                ("coupling", _F), ("lock", _I32), ("dyn_friction", _F), ("static_friction", _F),
                ("static_thr", _F), ("cohesion", _F), ("max_radius", _F), ("sleep_thr", _F),
                ("bmin", _F * 3), ("bmax", _F * 3), ("swelling_ratio", _F), ("swell_act", _F),
                ("swell_max", _F), ("xpbd_only", _I32)]


XK = dict(INTEGRATE=0, RESET_LABELS=1, BOUND=2, PARTICLE=3, APPLY=4, SLEEP=5, IMPULSES=6, SWELL=7)


class LoopState(ctypes.Structure):
    """mpmw_loop_state_t (include/mpmw.h)."""
    _fields_ = [("counter", ctypes.c_int), ("stall", ctypes.c_int), ("stopped_early", ctypes.c_int),
                ("segment_left", ctypes.c_int), ("residual", ctypes.c_double), ("prev_damage", ctypes.c_double),
                ("stats", ctypes.c_double * 7)]


class LoopParams(ctypes.Structure):
    """mpmw_loop_params_t (include/mpmw.h)."""
    _fields_ = [("chunk", ctypes.c_int), ("n_steps", ctypes.c_int), ("min_steps", ctypes.c_int),
                ("stall_steps", ctypes.c_int), ("residual_threshold", ctypes.c_double),
                ("stall_threshold", ctypes.c_double)]


class PhaseParams(ctypes.Structure):
    """mpmw_phase_params_t"""
    _fields_ = [("loop", LoopParams), ("xpbd_ratio", ctypes.c_int32), ("pulse_steps", ctypes.c_int32),
                ("phase", ctypes.c_int32)]


_SIGS = {
    "mpmw_last_error": (ctypes.c_char_p, []),
    "mpmw_version": (_I, []),
    "mpmw_mu_lam_bulk": (_I, [_I64, _P, _P, _P, _P, _P, _P]),
    "mpmw_geostatic_F": (_I, [_I64, _P, _P, _P, _P, _P, _F, _F, _F, _I, _P]),
    "mpmw_stress": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Params), _P, _P]),
    "mpmw_p2g": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _P, _P]),
    "mpmw_grid_update": (_I, [ctypes.POINTER(Grid), ctypes.POINTER(Params), _P]),
    "mpmw_grid_op": (_I, [ctypes.POINTER(Grid), ctypes.POINTER(Params), _I, _P]),
    "mpmw_g2p": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _P, _P]),
    "mpmw_g2p_stress": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _P, _P,
                             ctypes.c_size_t, _P]),
    "mpmw_workspace_bytes": (ctypes.c_size_t, [_I64]),
    "mpmw_stress_p2g": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _P, _P,
                             ctypes.c_size_t, _P]),
    "mpmw_g2p2g": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _I, _P, _P,
                        ctypes.c_size_t, _P]),
    "mpmw_vlc": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _P, _P]),
    "mpmw_vlc_phase": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _I, _P, _P]),
    "mpmw_substep": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _P, _P]),
    "mpmw_run_substeps": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params), _I, _P,
                               _P, ctypes.c_size_t, _P]),
    "mpmw_batch_workspace_bytes": (ctypes.c_size_t, [ctypes.POINTER(Grid), _I, _I64]),
    "mpmw_batch_prepare": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params),
                                ctypes.POINTER(_I64), _I, _P, ctypes.c_size_t, _P]),
    "mpmw_batch_run_substeps": (_I, [ctypes.POINTER(Particles), _I, _P, _P, ctypes.c_size_t, _P]),
    "mpmw_batch_run_range": (_I, [ctypes.POINTER(Particles), _I, _I, _I, _P, _P, ctypes.c_size_t, _P]),
    "mpmw_batch_set_options": (_I, [_P, _I, _I]),
    "mpmw_loop_create": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params),
                              ctypes.POINTER(LoopParams), _P, _P, _P, ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p),
                              _P]),
    "mpmw_phase_loop_create": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Grid), ctypes.POINTER(Params),
                                    ctypes.POINTER(Params), ctypes.POINTER(XPBD), ctypes.POINTER(Hash),
                                    ctypes.POINTER(XPBDParams), ctypes.POINTER(XPBDParams), ctypes.POINTER(PhaseParams),
                                    _P, _P, _P, ctypes.c_size_t, _P, ctypes.c_size_t,
                                    ctypes.POINTER(ctypes.c_void_p), _P]),
    "mpmw_xpbd_loop_create": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(XPBD), ctypes.POINTER(Hash),
                                   ctypes.POINTER(XPBDParams), _I, ctypes.c_double, _P, _P, _P, ctypes.c_size_t,
                                   ctypes.POINTER(ctypes.c_void_p), _P]),
    "mpmw_loop_launch": (_I, [_P, _P]),
    "mpmw_loop_destroy": (None, [_P]),
    "mpmw_teleport": (_I, [ctypes.POINTER(Particles), _F, _F, _P]),
    "mpmw_creep": (_I, [ctypes.POINTER(Particles), _P, _F, _F, _F, _F, _P]),
    "mpmw_stats": (_I, [ctypes.POINTER(Particles), _P, _P]),
    "mpmw_dp_samples": (_I, [_I64, ctypes.c_uint64, _P, _P, _P]),
    "mpmw_mlp_forward": (_I, [_P, _P, _I64, _P, _P]),
    "mpmw_mlp_grad": (_I, [_P, _P, _P, _I64, _P, _P, _P]),
    "mpmw_mlp_grad_tc": (_I, [_P, _P, _P, _I64, _P, _P, _P, _P]),
    "mpmw_mlp_adam": (_I, [_P, _P, _P, _P, _I, _F, _P]),
    "mpmw_mlp_pack": (_I, [_P, _P, _P]),
    "mpmw_mlp_infer_tc": (_I, [_P, _P, _P, _I64, _P, _P, _P]),
    "mpmw_surrogate_workspace_bytes": (ctypes.c_size_t, [_I64]),
    "mpmw_stress_surrogate": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(Params), _P, _P, _F, _I,
                                   ctypes.c_uint64, _P, _P, _P, ctypes.c_size_t, _P]),
    "mpmw_block_sort_workspace_bytes": (ctypes.c_size_t, [_I64]),
    "mpmw_block_sort": (_I, [_P, _I64, ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_int32), _I, _P, _P,
                             ctypes.c_size_t, _P]),
    "mpmw_hash_workspace_bytes": (ctypes.c_size_t, [_I64]),
    "mpmw_xpbd_step_workspace_bytes": (ctypes.c_size_t, [_I64, ctypes.POINTER(ctypes.c_int32)]),
    "mpmw_hash_build": (_I, [_P, _I64, ctypes.POINTER(Hash), _P, ctypes.c_size_t, _P]),
    "mpmw_hash_build_noalloc": (_I, [_P, _I64, ctypes.POINTER(Hash), _P]),
    "mpmw_xpbd_kernel": (_I, [_I, ctypes.POINTER(Particles), ctypes.POINTER(XPBD), ctypes.POINTER(Hash),
                              ctypes.POINTER(XPBDParams), _I, _P]),
    "mpmw_xpbd_step": (_I, [ctypes.POINTER(Particles), ctypes.POINTER(XPBD), ctypes.POINTER(Hash),
                            ctypes.POINTER(XPBDParams), _P, _P, ctypes.c_size_t, _P]),
    "mpmw_xpbd_set_options": (_I, [_I]),
    "mpmw_batch_run_persistent": (_I, [ctypes.POINTER(Particles), _I, _P, _P, ctypes.c_size_t, _P]),
    "mpmw_batch_persistent_launches": (_I64, []),
    "mpmw_xpbd_persistent_launches": (_I64, []),
}

_LIB = None


def lib(rebuild: bool = True):
    """Load (building first if stale) libmpmw.so; raises if it cannot be loaded."""
    global _LIB
    if _LIB is not None:
        return _LIB
    path = LIB
    if rebuild:
        try:
            path = build()
        except Exception:
            if not os.path.exists(LIB):
                raise
    if not os.path.exists(path):
        raise RuntimeError(f"libmpmw.so not found at {path}; run python -m mpmwarpydw_b200.build")
    h = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(h, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _LIB = h
    return h


class MPMWError(RuntimeError):
    pass


def check(rc: int, what: str = ""):
    if rc != MPMW_OK:
        msg = lib().mpmw_last_error().decode(errors="replace")
        raise MPMWError(f"{what}: libmpmw error {rc}: {msg}")


def exported_symbols(header: str | None = None):
    """Names of every function declared in include/*.h (for symbol checks)."""
    import glob
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    names = []
    files = [header] if header else sorted(glob.glob(os.path.join(root, "include", "*.h")))
    for f in files:
        src = open(f).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"\b(mpmw_[a-z0-9_]+)\s*\(", src)
    return sorted(set(names))
