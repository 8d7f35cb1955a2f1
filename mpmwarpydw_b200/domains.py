"""Seeded synthetic domains standing in for the reference's HDF5 inputs.

The reference reads particle positions/volumes (+ optional per-particle
material arrays) from HDF5 files written by its generator scripts
(exampleDomains/createInputHDF5.py, benchmarks/*/create*.py).  These
generators build the same kind of inputs in memory, seeded:

  block_collapse  64,000-particle Drucker-Prager block collapse (40^3 lattice)
  caving_block    512,000-particle coupled MPM+XPBD caving block with an undercut
                  and lognormal E / cohesion fields
  tunnel          3,873,600-particle tunnel domain (200 x 100 x 200 lattice at
                  0.5 m minus a 10 m-radius cylinder), geostatic pre-stress
  sweep_scenes    64 block-collapse scenes of 20k..500k particles with per-scene
                  friction angle / cohesion

Each returns a :class:`Domain` (positions in lattice order, x fastest, as the
reference's generators write them) with the argument overrides that define the
scene; :func:`build` turns it into (sim, mpm, xpbd) on a CUDA device.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .utils.getArgs import defaults


def friction_angle_to_alpha(phi_deg):
    """Drucker-Prager alpha from a friction angle, as in
    benchmarks/cavingBenchmark/createRandomRockDomain.py:160-164."""
    s = np.sin(np.radians(phi_deg))
    return 2.0 * s / (np.sqrt(3.0) * (3.0 - s))


@dataclass
class Domain:
    name: str
    x: np.ndarray                     # (N, 3) float32
    vol: np.ndarray                   # (N,) float32
    props: dict = field(default_factory=dict)
    overrides: dict = field(default_factory=dict)
    dx: float | None = None
    minBounds: np.ndarray | None = None
    gridDims: tuple | None = None
    notes: str = ""

    @property
    def n(self):
        return int(self.x.shape[0])

    def args(self, **extra):
        a = defaults()
        for k, v in {**self.overrides, **extra}.items():
            setattr(a, k, v)
        return a


def _lattice(counts, spacing, origin=0.0):
    """Cell-centred lattice, x fastest (origin + spacing*(i + 1/2))."""
    nx, ny, nz = counts
    i = np.arange(nx, dtype=np.float64)
    j = np.arange(ny, dtype=np.float64)
    k = np.arange(nz, dtype=np.float64)
    zz, yy, xx = np.meshgrid(k, j, i, indexing="ij")
    pts = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], 1)
    return origin + spacing * (pts + 0.5)


def block_collapse(n_side=40, spacing=0.25, jitter=0.025, seed=0, box=None, dx=0.5, phi=30.0, cohesion=1e6,
                   E=10e9, nu=0.25, density=2650.0, steps=1000):
    """Plain-MPM Drucker-Prager block collapse under gravity (XPBD off)."""
    rng = np.random.default_rng(seed)
    x = _lattice((n_side,) * 3, spacing)
    x += rng.uniform(-jitter, jitter, size=x.shape)
    vol = np.full(x.shape[0], spacing ** 3, dtype=np.float32)
    box = box if box is not None else n_side * spacing
    # minBounds chosen so the boundary band of the low z face (node index <= 2) ends at z = 0
    minB = np.array([-box / 2, -box / 2, -2 * dx])
    dims = tuple(int(math.ceil(v)) for v in (np.array([2 * box, 2 * box, 2 * box]) / dx))
    ov = dict(dt=1e-4, dtxpbd=1e-4 * steps * 10, density=density, E=E, nu=nu, ys=cohesion,
              alpha=float(friction_angle_to_alpha(phi)), strainCriteria=0.05, hardening=0.0, softening=0.0,
              eff=0.05, rpic_damping=0.0, boundFriction=0.5, boundaryCondition="friction", gravity=-9.81,
              initialise_geostatic=0, volumetric_locking_correction=0, update_cov=0, grid_v_damping_scale=1.1)
    return Domain("block_collapse", x.astype(np.float32), vol, {}, ov, dx, minB, dims,
                  notes=f"{n_side}^3 lattice at {spacing} m, jitter +-{jitter} m, dilation recorded not used")


def caving_block(n_side=80, spacing=0.25, jitter_frac=0.1, seed=1, dx=0.5, undercut=6.0, undercut_h=1.0):
    """Coupled MPM+XPBD caving block: lognormal E / cohesion, base undercut."""
    rng = np.random.default_rng(seed)
    x = _lattice((n_side,) * 3, spacing)
    x += rng.uniform(-jitter_frac * spacing, jitter_frac * spacing, size=x.shape)
    L = n_side * spacing
    c = L / 2
    cut = (np.abs(x[:, 0] - c) < undercut / 2) & (np.abs(x[:, 1] - c) < undercut / 2) & (x[:, 2] < undercut_h)
    x = x[~cut]
    n = x.shape[0]
    vol = np.full(n, spacing ** 3, dtype=np.float32)
    E = (10e9 * np.exp(0.3 * rng.standard_normal(n))).astype(np.float32)
    ys = (0.5e6 * np.exp(0.3 * rng.standard_normal(n))).astype(np.float32)
    props = dict(E=E, ys=ys)
    minB = np.array([-L / 2, -L / 2, -2 * dx])
    dims = tuple(int(math.ceil(v)) for v in (np.array([2 * L, 2 * L, 1.5 * L + 2 * dx]) / dx))
    ov = dict(dt=1e-4, dtxpbd=5e-4, density=2650.0, nu=0.25, alpha=float(friction_angle_to_alpha(32.0)),
              strainCriteria=0.05, eff=0.05, rpic_damping=0.0, boundFriction=0.5, boundaryCondition="friction",
              gravity=-9.81, initialise_geostatic=0, volumetric_locking_correction=0, update_cov=0,
              staticParticleFriction=0.6, dynamicParticleFriction=0.5, particle_cohesion=0.0, xpbd_iterations=4,
              grid_v_damping_scale=1.1)
    return Domain("caving_block", x.astype(np.float32), vol, props, ov, dx, minB, dims,
                  notes="particle_cohesion is a gap length in the reference; '10 kPa' has no mapping (0 used)")


def tunnel(nx=200, ny=100, nz=200, spacing=0.5, radius=10.0, dx=1.0, pad_cells=10, eta=1e-3):
    """Large tunnel domain with geostatic pre-stress (the 4M-particle workload)."""
    x = _lattice((nx, ny, nz), spacing)
    cx, cz = nx * spacing / 2, nz * spacing / 2
    keep = (x[:, 0] - cx) ** 2 + (x[:, 2] - cz) ** 2 >= radius ** 2
    x = x[keep]
    vol = np.full(x.shape[0], spacing ** 3, dtype=np.float32)
    pmin, pmax = x.min(0), x.max(0)
    minB = pmin - pad_cells * dx
    dims = tuple(int(v) for v in np.ceil((pmax + pad_cells * dx - minB) / dx))
    ov = dict(dt=5e-5, dtxpbd=1e-2, density=2600.0, E=20e9, nu=0.25, ys=2e6,
              alpha=float(friction_angle_to_alpha(35.0)), strainCriteria=0.05, eff=0.05, rpic_damping=0.0,
              eta_shear=eta, eta_bulk=eta, K0=0.5, initialise_geostatic=1, boundaryCondition="friction",
              boundFriction=0.5, gravity=-9.81, volumetric_locking_correction=0, update_cov=0,
              grid_v_damping_scale=1.1)
    return Domain("tunnel", x.astype(np.float32), vol, {}, ov, dx, minB, dims,
                  notes=f"{nx}x{ny}x{nz} lattice at {spacing} m minus r<{radius} m cylinder along y")


def sweep_scenes(n_scenes=64, seed=4, nmin=20_000, nmax=500_000, box=10.0):
    """Parameter-sweep scenes: block collapses of uneven size and strength."""
    out = []
    for s in range(n_scenes):
        rng = np.random.default_rng(seed + s)
        n_target = int(rng.integers(nmin, nmax + 1))
        side = int(round(n_target ** (1 / 3)))
        spacing = box / side
        phi = float(rng.uniform(20.0, 45.0))
        coh = float(np.exp(rng.uniform(np.log(0.1e6), np.log(5e6))))
        d = block_collapse(n_side=side, spacing=spacing, jitter=0.1 * spacing, seed=seed + s, box=box, dx=2 * spacing,
                           phi=phi, cohesion=coh)
        d.name = f"sweep_{s:02d}"
        out.append(d)
    return out


def build(domain: Domain, device="cuda:0", **extra):
    """(sim, mpm, xpbd) for a domain on a CUDA device."""
    from .scene import build_states
    args = domain.args(**extra)
    return build_states(args, domain.x, domain.vol, domain.props, device=device, dx=domain.dx,
                        minBounds=domain.minBounds, gridDims=domain.gridDims, adjust_dt=False)


def seed_plastic_trials(sim, mpm, seed=3, emin=1e-6, emax=1e-1):
    """Overwrite a built scene's trial state with the learned-return-map
    benchmark's distributions (in place, on the device): per particle a trial
    log strain of magnitude log-uniform in [emin, emax] along a uniformly
    random direction of principal values, in a uniformly random principal
    frame (F_trial = Q diag(exp(e)) Q^T), a friction angle U(20, 45) deg ->
    alpha, a cohesion log-uniform in [0.1, 5] MPa -> ys and a damage U(0, 1).
    mu, lam and the rest of the scene stay.  Returns the number of particles."""
    import torch
    dev = mpm.particle_F_trial.device
    n = sim.nPoints
    g = torch.Generator(device=dev).manual_seed(int(seed))
    u = lambda *shape: torch.rand(*shape, generator=g, device=dev, dtype=torch.float64)  # noqa: E731
    mag = torch.exp(math.log(emin) + (math.log(emax) - math.log(emin)) * u(n))
    d = torch.randn(n, 3, generator=g, device=dev, dtype=torch.float64)
    e = mag[:, None] * d / d.norm(dim=1, keepdim=True).clamp_min(1e-300)
    q = torch.randn(n, 4, generator=g, device=dev, dtype=torch.float64)
    q = q / q.norm(dim=1, keepdim=True)
    w, x, y, z = q.unbind(1)
    Q = torch.stack([1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                     2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                     2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)], 1).view(n, 3, 3)
    F = Q @ torch.diag_embed(torch.exp(e)) @ Q.transpose(1, 2)
    mpm.particle_F_trial = F.to(torch.float32)
    phi = 20.0 + 25.0 * u(n)
    s = torch.sin(torch.deg2rad(phi))
    # in place: the library holds pointers to these arrays
    mpm.alpha.copy_(2.0 * s / (math.sqrt(3.0) * (3.0 - s)))
    mpm.ys.copy_(torch.exp(math.log(0.1e6) + (math.log(5e6) - math.log(0.1e6)) * u(n)))
    mpm.particle_damage.copy_(u(n))
    return n
