"""Command-line / JSON configuration of the driver (reference: utils/getArgs.py:13-153).

The flag names, types and defaults are the reference's (they are the drop-in
interface: the reference's benchmark JSON files must load unchanged).  The
merge rule is also the reference's: a JSON file given with ``--config``
overrides the defaults, a flag given on the command line overrides the JSON,
and JSON keys that are not flags are ignored.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

# (name, type, default)  -- utils/getArgs.py:22-123
FLAGS = [
    ("dt", float, 0.0), ("dtxpbd", float, 1e-2), ("bigStepDuration", float, 10.0), ("xpbdOnlyDuration", float, 0.0),
    ("bigSteps", int, 100),
    ("residualThreshold", float, 1e-8), ("damage_stall_threshold", float, 1e-9), ("damage_stall_duration", float, 0.1),
    ("xpbd_sleep_termination_ratio", float, 0.95),
    ("rpic_damping", float, 0.2), ("grid_v_damping_scale", float, 1.1), ("update_cov", int, 1),
    ("render", int, 0), ("render_interval", float, 0.1), ("color_mode", str, "effective_ys"), ("saveFlag", int, 0),
    ("outputFolder", str, "./output/"), ("restart", str, None), ("open_paraview", int, 0),
    ("domainFile", str, "./exampleDomains/annular_arch_particles.h5"), ("grid_padding", float, 25.0),
    ("grid_particle_spacing_scale", float, 2.0), ("boundary_padding_mask", str, "111101"),
    ("density", float, 3000.0), ("E", float, 1e8), ("nu", float, 0.2), ("constitutive_model", int, 1),
    ("ys", float, 3e8), ("alpha", float, 0.3), ("hardening", float, 0.0), ("softening", float, 0.0),
    ("eta_shear", float, 1e5), ("eta_bulk", float, 1e5), ("volumetric_locking_correction", int, 1),
    ("gravity", float, -9.81), ("K0", float, 0.5), ("z_top", float, None), ("initialise_geostatic", int, 1),
    ("gravity_pulse_factor", float, 1.0), ("gravity_pulse_duration", float, 0.0),
    ("boundFriction", float, 0.2), ("boundaryCondition", str, "friction"), ("boundRestitution", float, 0.0),
    ("eff", float, 0.05), ("strainCriteria", float, 0.05),
    ("xpbd_relaxation", float, 1.0), ("xpbd_mpm_coupling_strength", float, 0.25),
    ("xpbd_deactivation_z_datum", float, None), ("mpm_contact_transition_lock", int, 0),
    ("dynamicParticleFriction", float, 0.05), ("staticVelocityThreshold", float, 1e-5),
    ("staticParticleFriction", float, 0.1), ("xpbd_iterations", int, 4), ("particle_cohesion", float, 0.0),
    ("sleepThreshold", float, 0.5),
    ("swellingRatio", float, 0.2), ("swellingActivationFactor", float, 1.0), ("swellingMaxFactor", float, 2.0),
    ("particle_v_max", float, 1000.0),
]

# the reference restricts the CLI choice to these four; JSON may set the plane-strain kinds too
BC_CHOICES = ["friction", "friction_gradual", "restitution", "absorbing"]


def make_parser():
    pre = argparse.ArgumentParser(add_help=False)
    pre.add_argument("--config", type=str, help="Path to JSON config file")
    p = argparse.ArgumentParser(description="MPM-XPBD Simulation Parameters", parents=[pre])
    for name, typ, default in FLAGS:
        kw = dict(type=typ, default=default)
        if name == "boundaryCondition":
            kw["choices"] = BC_CHOICES
        p.add_argument("--" + name, **kw)
    return pre, p


def defaults():
    """An argparse.Namespace holding every default (no CLI, no JSON)."""
    _, p = make_parser()
    return p.parse_args([])


def get_args(argv=None, verbose=True):
    """Parse ``argv`` (default sys.argv[1:]) merged with ``--config`` JSON."""
    argv = sys.argv[1:] if argv is None else list(argv)
    pre, p = make_parser()
    pre_args, _ = pre.parse_known_args(argv)
    config = {}
    if pre_args.config and os.path.exists(pre_args.config):
        with open(pre_args.config) as f:
            config = json.load(f)
    args, _unknown = p.parse_known_args(argv)
    on_cli = {a.lstrip("-").replace("-", "_").split("=")[0] for a in argv if a.startswith("--")}
    for k, v in config.items():
        if k not in on_cli and hasattr(args, k):
            setattr(args, k, v)
    if verbose:
        print("\n===== Loaded Simulation Parameters =====")
        for name, _, _ in [("config", str, None)] + FLAGS:
            if hasattr(args, name):
                print(f"{name}: {getattr(args, name)}")
        print("=======================================\n")
    return args
