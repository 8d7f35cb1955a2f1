"""Loading of the golden fixtures in tests/golden/ (written by
tests/golden/gen_golden.py from the reference's own kernel source executed in
float64).  A fixture holds ``in/<state>.<attribute>`` inputs and the
``out/<state>.<attribute>`` arrays that one reference step changed."""
from __future__ import annotations

import os

import numpy as np

from oracle.oracle import OracleState

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
MPM_FIXTURES = ("mpm_friction", "mpm_restitution", "mpm_planestrain")
XPBD_FIXTURES = ("xpbd_lock", "xpbd_free")


def _attr(key):
    return key.split("/", 1)[1].split(".", 1)[1]


def load(name, dtype=np.float64):
    """(inputs as an OracleState in ``dtype``, expected state after the step as a dict)."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    s = OracleState()
    expected = {}
    for k in z.files:
        if not k.startswith("in/"):
            continue
        a = z[k]
        if a.ndim == 0:
            v = a.item()
        elif a.dtype.kind in "iu":
            v = np.ascontiguousarray(a.astype(np.int32))
        else:
            v = np.ascontiguousarray(a.astype(dtype))
        setattr(s, _attr(k), v)
        expected[_attr(k)] = a
    for k in z.files:
        if k.startswith("out/"):
            expected[_attr(k)] = z[k]
    s.boundaryCondition = str(z["meta/boundaryCondition"])
    s.gravity = np.ascontiguousarray(z["meta/gravity"].astype(dtype))
    s.minBounds = np.ascontiguousarray(np.asarray(s.minBounds, dtype))
    return s, expected


def array_rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-300)) if a.size else 0.0


def gpu_states(name, device="cuda:0"):
    """(sim, mpm, xpbd) of this package on ``device`` holding a fixture's inputs."""
    import torch

    from mpmwarpydw_b200.utils.getArgs import defaults
    from mpmwarpydw_b200.utils.simStates import MPMState, SimState, XPBDState, vec3
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    ins = {k[3:]: z[k] for k in z.files if k.startswith("in/")}
    args = defaults()
    for key, a in ins.items():
        attr = key.split(".", 1)[1]
        if a.ndim == 0 and hasattr(args, attr):
            setattr(args, attr, a.item())
    args.boundaryCondition = str(z["meta/boundaryCondition"])
    args.gravity = float(z["meta/gravity"][2])
    n = ins["sim.particle_x"].shape[0]
    dims = tuple(int(d) for d in ins["mpm.grid_m"].shape)
    sim, mpm, xpbd = SimState(args, n, device), MPMState(args, n, dims, device), XPBDState(args, n, device)
    objs = {"sim": sim, "mpm": mpm, "xpbd": xpbd}
    arrays = {
        "sim": ("particle_x", "particle_v", "particle_mass", "particle_vol", "particle_radius", "particle_density",
                "materialLabel", "activeLabel"),
        "mpm": ("mu", "lam", "ys", "alpha", "hardening", "softening", "eta_shear", "eta_bulk", "strainCriteria",
                "particle_F", "particle_F_trial", "particle_stress", "particle_C", "particle_accumulated_strain",
                "particle_damage", "particle_cov"),
        "xpbd": ("particle_x_initial_xpbd", "particle_v_initial_xpbd", "particle_cumDist_xpbd", "particleBaseRadius",
                 "particleMaxRadius"),
    }
    for tag, names in arrays.items():
        for attr in names:
            a = ins[f"{tag}.{attr}"]
            dt = torch.int32 if a.dtype.kind in "iu" else torch.float32
            setattr(objs[tag], attr, torch.as_tensor(a, dtype=dt, device=device))
    sim.dx = float(ins["sim.dx"])
    sim.invdx = float(ins["sim.invdx"])
    sim.dt = float(ins["sim.dt"])
    sim.dtxpbd = float(ins["sim.dtxpbd"])
    sim.minBounds = vec3(*[float(v) for v in ins["sim.minBounds"]])
    mpm.boundaryPadding = int(ins["mpm.boundaryPadding"])
    xpbd.max_radius = float(ins["xpbd.max_radius"])
    xpbd.minBoundsXPBD = vec3(*[float(v) for v in ins["xpbd.minBoundsXPBD"]])
    xpbd.maxBoundsXPBD = vec3(*[float(v) for v in ins["xpbd.maxBoundsXPBD"]])
    torch.cuda.synchronize(device)
    return sim, mpm, xpbd
