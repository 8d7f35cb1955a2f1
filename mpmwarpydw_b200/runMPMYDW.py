"""Simulation driver with the reference's configuration surface (runMPMYDW.py).

    python -m mpmwarpydw_b200.runMPMYDW --config cfg.json [--flag value ...] [--check_interval K]

Flags, defaults and the JSON merge rule are the reference's (utils/getArgs.py).
The structure is the reference's big-step loop (runMPMYDW.py:633-903):

  for each big step:
    phase 1 (MPM + XPBD): gravity pulse for gravity_pulse_duration, MPM
      substeps with an XPBD step after every substep whose counter is a
      positive multiple of mpmStepsPerXpbdStep; stop after nSteps substeps, or
      once at least 1000 substeps ran and the residual (sum |v|/r over active
      particles / active count) is below residualThreshold, or when the mean
      damage grew by less than damage_stall_threshold per substep for
      damage_stall_duration;
    phase 2 (XPBD only, xpbdOnlyDuration): debris settling, stopping early when
      the sleeping fraction of XPBD particles reaches
      xpbd_sleep_termination_ratio;
    end: XPBD particles below the deactivation datum are deactivated and moved
      out of the domain.

The reference reads the residual and the mean damage back to the host after
every substep; ``--check_interval K`` (K = 1 is the reference) reads them every
K substeps instead, and the MPM substeps in between run as one fused library
call (their XPBD steps still fall on the same counters).  Termination is then
decided at those points.

Domain input (``--domainFile``): an HDF5 file in the reference's schema (read
by the package's own reader, no h5py needed), an .npz with the same keys
(``x`` [3, N] or [N, 3], ``particle_volume`` [N], optional per-particle
``density``, ``E``, ``nu``, ``ys``, ``alpha``, ``hardening``, ``softening``,
``eta_shear``, ``eta_bulk``, ``strainCriteria``, ``damage``), or
``synthetic:<name>`` for a seeded generator of ``domains`` (``block_collapse``,
``caving_block``, ``tunnel``).
Output (``saveFlag``): the reference's files, <prefix>_grid.vti and
<prefix>_particles.vtp per render interval in ``outputFolder``, the end of each
big step a checkpoint with the restart arrays (runMPMYDW.py:606-627).
``--restart <checkpoint.vtp>`` continues from such a checkpoint at the next big
step (runMPMYDW.py:498-576).
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np
import torch

from . import domains as _domains
from .bind import check_status, params_from_states
from .engine import DeviceLoop, PhaseLoop, SubstepGraphCache, XPBDLoop, original_order, sort_particles
from .scene import build_states
from .utils import mpmRoutines
from .utils import simulationRoutines as S
from .utils import fs5PlotUtils
from .utils.getArgs import get_args
from .utils.simStates import vec3

PROPERTY_NAMES = ("density", "E", "nu", "ys", "alpha", "hardening", "softening", "eta_shear", "eta_bulk",
                  "strainCriteria", "damage")
MIN_STEPS = 1000  # runMPMYDW.py:654


def load_domain(path: str, args):
    """(x [N,3], particle_volume [N], props, overrides) for --domainFile."""
    if path.startswith("synthetic:"):
        name = path.split(":", 1)[1]
        d = getattr(_domains, name)()
        return d.x, d.vol, d.props, d.overrides, d
    if path.endswith(".npz"):
        z = np.load(path)
        get = lambda k: np.asarray(z[k])  # noqa: E731
        keys = set(z.files)
    else:
        from .hdf5io import HDF5File
        f = HDF5File(path)
        get = lambda k: np.asarray(f[k])  # noqa: E731
        keys = set(f.keys())
    x = get("x")
    if x.shape[0] == 3 and x.shape[-1] != 3:
        x = x.T
    vol = get("particle_volume").reshape(-1)
    props = {k: get(k).reshape(-1) for k in PROPERTY_NAMES if k in keys}
    return x.astype(np.float32), vol.astype(np.float32), props, {}, None


def save_state(sim, mpm, xpbd, folder, big_step, counter, checkpoint=False):
    """One save as the reference writes it (utils/fs5PlotUtils.py:785-881):
    <prefix>_grid.vti and <prefix>_particles.vtp in ``folder``, particles in
    input order; a checkpoint (the end of a big step) adds the restart
    arrays.  Returns the .vtp path."""
    os.makedirs(folder, exist_ok=True)
    out = sim.outputFolder
    sim.outputFolder = folder
    try:
        return fs5PlotUtils.save_mpm(sim, mpm, big_step, counter, include_restart_data=checkpoint,
                                     xpbd=xpbd if checkpoint else None, order=lambda t: original_order(sim, t))
    finally:
        sim.outputFolder = out


def apply_restart(sim, mpm, xpbd, path):
    """Restore the state of a checkpoint (runMPMYDW.py:498-576) into state
    objects that hold the particles in input order; returns the first big step
    to run (the one after the checkpoint's)."""
    import torch
    r = fs5PlotUtils.load_restart_from_vtp(path)
    if len(r["particle_x"]) != sim.nPoints:
        raise ValueError(f"Restart file has {len(r['particle_x'])} particles, but domain has {sim.nPoints}. "
                         "Cannot restart with different particle count.")
    dev = sim.device
    t = lambda a, dt=torch.float32: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)  # noqa: E731
    sim.t = float(r["sim_time"])
    sim.particle_x, sim.particle_v = t(r["particle_x"]), t(r["particle_v"])
    if r["materialLabel"] is not None:
        sim.materialLabel = t(r["materialLabel"], torch.int32)
    if r["activeLabel"] is not None:
        sim.activeLabel = t(r["activeLabel"], torch.int32)
    mpm.particle_F = t(r["particle_F"])
    mpm.particle_F_trial = t(r["particle_F"])
    mpm.particle_C = t(r["particle_C"])
    for key, attr in (("particle_accumulated_strain", "particle_accumulated_strain"),
                      ("particle_damage", "particle_damage"), ("particle_stress", "particle_stress"),
                      ("ys", "ys"), ("ys_base", "ys_base")):
        if r.get(key) is not None:
            setattr(mpm, attr, t(r[key]))
    for p in fs5PlotUtils.MATERIAL_PROPERTIES:
        if r.get(p) is not None:
            setattr(mpm, p, t(r[p]))
    for key in ("particle_vol", "particle_mass", "particle_density", "particle_radius"):
        if r.get(key) is not None:
            setattr(sim, key, t(r[key]))
    if r.get("particle_x_initial_xpbd") is not None:
        xpbd.particle_x_initial_xpbd = t(r["particle_x_initial_xpbd"])
    if r.get("particle_cumDist_xpbd") is not None:
        xpbd.particle_cumDist_xpbd = t(r["particle_cumDist_xpbd"])
    return int(r["bigStep"]) + 1


class PhaseOneMonitor:
    """Termination of phase 1 (runMPMYDW.py:656-727), host side."""

    def __init__(self, n_steps, residual_threshold, stall_threshold, stall_steps, min_steps=MIN_STEPS):
        self.n_steps, self.residual_threshold = n_steps, residual_threshold
        self.stall_threshold, self.stall_steps, self.min_steps = stall_threshold, stall_steps, min_steps
        self.counter, self.residual, self.stall = 0, 1e10, 0
        self.prev_damage = None
        self.stopped_early = False

    def running(self):
        return self.counter < self.n_steps and (self.counter < self.min_steps or self.residual > self.residual_threshold)

    def update(self, k, residual, mean_damage):
        """Account k substeps ending with (residual, mean damage); returns False
        when the damage stall ends the phase."""
        self.counter += k
        self.residual = residual
        if self.prev_damage is None:
            self.prev_damage = mean_damage
        change = mean_damage - self.prev_damage
        if change < self.stall_threshold * k and self.counter > self.min_steps:
            self.stall += k
        else:
            self.stall = 0
        self.prev_damage = mean_damage
        if self.stall >= self.stall_steps and self.counter > self.min_steps:
            self.stopped_early = True
            return False
        return True


def device_segment(c, k, ratio, n_steps, pulse_steps=0):
    """Substeps the device loop may run from counter c in whole chunks of k:
    every chunk ends within n_steps and, while a gravity pulse of pulse_steps
    substeps is on, by its end, and holds no XPBD substep (a positive multiple
    of ratio), which the host runs with the chunk around it."""
    n = 0
    while True:
        a = c + n
        if a + k > n_steps or (pulse_steps and a < pulse_steps < a + k):
            return n
        first = max(ratio, ((a + ratio - 1) // ratio) * ratio)  # first positive multiple of ratio >= a
        if first < a + k:
            return n
        n += k


def _stats(sim, mpm):
    """(residual, mean damage over active, counts) from one device reduction."""
    s = S.step_stats(sim, mpm).cpu().numpy()
    active = s[1]
    residual = s[0] / active if active > 0 else 0.0
    mean_damage = s[2] / active if active > 0 else 0.0
    return float(residual), float(mean_damage), s


def run(args, check_interval=1, device="cuda:0", verbose=True, max_big_steps=None, device_loop=False,
        resort_interval=0):
    """The big-step loop.  ``resort_interval`` > 0 re-sorts the particles into
    block order on the device (engine.sort_particles) at the first check at or
    after every ``resort_interval`` substeps of phase 1, so the particles of a
    CTA stay within a few cells as the material flows (results do not depend
    on the order; the captured graphs stay valid, as the fields keep their
    storage)."""
    dev = torch.device(device)
    torch.cuda.set_device(dev)
    x, vol, props, overrides, dom = load_domain(args.domainFile, args)
    for k, v in overrides.items():
        setattr(args, k, v)
    kw = {}
    if dom is not None:
        kw = dict(dx=dom.dx, minBounds=dom.minBounds, gridDims=dom.gridDims)
    sim, mpm, xpbd = build_states(args, x, vol, props, device=dev, adjust_dt=True, **kw)
    first_big = 0
    if getattr(args, "restart", None):
        first_big = apply_restart(sim, mpm, xpbd, args.restart)
    sort_particles(sim, mpm, xpbd)
    log = print if verbose else (lambda *a, **k: None)
    log(f"particles {sim.nPoints}, grid {mpm.gridDims}, dx {sim.dx:.4f}, dt {sim.dt:.3e}, "
        f"XPBD every {sim.mpmStepsPerXpbdStep} substeps")
    ratio = max(1, int(sim.mpmStepsPerXpbdStep))
    graphs = SubstepGraphCache()  # the runs of substeps between checks repeat: replay them
    # the stop test on the device between host events (not while saving, which
    # the host checks after every chunk)
    use_loop = device_loop and not sim.saveFlag
    loops = {}
    base_gravity = sim.gravity
    next_save = sim.t + args.render_interval
    start = time.time()
    saved = []
    big_steps = sim.bigSteps if max_big_steps is None else min(sim.bigSteps, max_big_steps)
    for big in range(first_big, big_steps):
        pulse_steps = int(args.gravity_pulse_duration / sim.dt) if args.gravity_pulse_duration > 0 else 0
        pulsing = args.gravity_pulse_factor != 1.0 and pulse_steps > 0
        if pulsing:
            sim.gravity = vec3(*[g * args.gravity_pulse_factor for g in base_gravity])
        _, d0, _ = _stats(sim, mpm)
        mon = PhaseOneMonitor(sim.nSteps, sim.residualThreshold, sim.damage_stall_threshold,
                              int(sim.damage_stall_duration / sim.dt))
        mon.prev_damage = d0
        next_resort = resort_interval if resort_interval > 0 else None
        while mon.running():
            if next_resort is not None and mon.counter >= next_resort:
                sort_particles(sim, mpm, xpbd)
                next_resort = (mon.counter // resort_interval + 1) * resort_interval
            c = mon.counter
            kc = check_interval
            if use_loop and ratio % kc == 0 and c % kc == 1 % kc and c + kc <= sim.nSteps:
                # the rest of phase 1 in one launch: XPBD steps and the pulse's end inside the graph
                key = ("phase", bytes(params_from_states(sim, mpm)), tuple(base_gravity), pulse_steps if pulsing else 0)
                loop = loops.get(key)
                if loop is None:
                    loop = loops[key] = PhaseLoop(
                        sim, mpm, xpbd, kc, sim.nSteps, sim.residualThreshold, sim.damage_stall_threshold,
                        int(sim.damage_stall_duration / sim.dt), mon.min_steps, xpbd_ratio=ratio,
                        pulse_steps=pulse_steps if pulsing else 0,
                        pulse_gravity=[g * args.gravity_pulse_factor for g in base_gravity], gravity=base_gravity)
                seg = ((sim.nSteps - c) // kc) * kc
                if next_resort is not None:
                    seg = min(seg, max(kc, ((next_resort - c + kc - 1) // kc) * kc))
                st = loop.run(c, mon.stall, mon.residual, mon.prev_damage, seg)
                check_status(dev, f"substeps {c}-{st.counter}", log)
                sim.t += (st.counter - c) * sim.dt
                mon.counter, mon.stall, mon.residual, mon.prev_damage = st.counter, st.stall, st.residual, st.prev_damage
                if pulsing and mon.counter >= pulse_steps:
                    sim.gravity = base_gravity
                if st.stopped_early:
                    mon.stopped_early = True
                    log(f"    early termination: damage stalled for {sim.damage_stall_duration}s")
                    break
                s7 = st.stats
                log(f"  big step {big + 1}, substep {mon.counter}, t {sim.t:.4f}s, residual {st.residual:.4e}, "
                    f"mean damage {st.prev_damage:.6f}, MPM {int(s7[3])}+{int(s7[5])}, "
                    f"XPBD {int(s7[4])}+{int(s7[6])}, wall {time.time() - start:.2f}s")
                continue
            if use_loop and ratio % kc != 0:
                seg = device_segment(c, check_interval, ratio, sim.nSteps, pulse_steps if pulsing else 0)
                if seg >= check_interval:
                    key = bytes(params_from_states(sim, mpm))
                    loop = loops.get(key)
                    if loop is None:
                        loop = loops[key] = DeviceLoop(sim, mpm, xpbd, check_interval, sim.nSteps,
                                                       sim.residualThreshold, sim.damage_stall_threshold,
                                                       int(sim.damage_stall_duration / sim.dt), mon.min_steps)
                    st = loop.run(c, mon.stall, mon.residual, mon.prev_damage, seg)
                    check_status(dev, f"substeps {c}-{st.counter}", log)
                    sim.t += (st.counter - c) * sim.dt
                    mon.counter, mon.stall, mon.residual, mon.prev_damage = st.counter, st.stall, st.residual, st.prev_damage
                    if pulsing and mon.counter == pulse_steps:
                        sim.gravity = base_gravity
                    if st.stopped_early:
                        mon.stopped_early = True
                        log(f"    early termination: damage stalled for {sim.damage_stall_duration}s")
                        break
                    if mon.counter // 100 > c // 100:
                        s7 = st.stats
                        log(f"  big step {big + 1}, substep {mon.counter}, t {sim.t:.4f}s, residual {st.residual:.4e}, "
                            f"mean damage {st.prev_damage:.6f}, MPM {int(s7[3])}+{int(s7[5])}, "
                            f"XPBD {int(s7[4])}+{int(s7[6])}, wall {time.time() - start:.2f}s")
                    continue
            # substeps up to the next check: stop at the pulse end and never skip past nSteps
            # (with the phase loop, up to the first counter = 1 mod check_interval)
            k = min(check_interval, sim.nSteps - c)
            if use_loop and ratio % kc == 0 and kc > 1:
                k = min(k, (1 - c) % kc or kc)
            if pulsing and c < pulse_steps:
                k = min(k, pulse_steps - c)
            done = 0
            while done < k:
                cc = c + done
                nxt = ratio if cc == 0 else ((cc + ratio - 1) // ratio) * ratio  # next XPBD counter
                m = min(k - done, nxt - cc + 1)
                if m == 1:
                    S.mpmSimulationStep(sim, mpm, xpbd, dev)
                else:
                    graphs.run(sim, mpm, xpbd, m)
                if cc + m - 1 == nxt:
                    S.xpbdSimulationStep(sim, mpm, xpbd, dev)
                done += m
            sim.t += k * sim.dt
            residual, mean_damage, counts = _stats(sim, mpm)
            check_status(dev, f"substeps {c}-{c + k}", log)
            if pulsing and mon.counter + k == pulse_steps:
                sim.gravity = base_gravity
            if not mon.update(k, residual, mean_damage):
                log(f"    early termination: damage stalled for {sim.damage_stall_duration}s")
                break
            if mon.counter % 100 < k:
                log(f"  big step {big + 1}, substep {mon.counter}, t {sim.t:.4f}s, residual {residual:.4e}, "
                    f"mean damage {mean_damage:.6f}, MPM {int(counts[3])}+{int(counts[5])}, "
                    f"XPBD {int(counts[4])}+{int(counts[6])}, wall {time.time() - start:.2f}s")
            if sim.saveFlag and sim.t >= next_save - 0.5 * sim.dt:
                saved.append(save_state(sim, mpm, xpbd, sim.outputFolder, big, mon.counter))
                next_save += args.render_interval
        if pulsing:
            sim.gravity = base_gravity
        log(f"  phase 1 done after {mon.counter} substeps ({mon.counter * sim.dt:.3f}s simulated)")
        check_status(dev, "phase 1", log)
        # phase 2: XPBD only
        if device_loop and sim.xpbdOnlySteps > 0:
            xl = loops.get("xpbd_only")
            if xl is None:
                xl = loops["xpbd_only"] = XPBDLoop(sim, mpm, xpbd, sim.xpbdOnlySteps, sim.xpbd_sleep_termination_ratio)
            st2 = xl.run_steps(0, sim.xpbdOnlySteps)
            sim.t += st2.counter * sim.dtxpbd
            if st2.stopped_early:
                log(f"    phase 2 stopped early: {int(st2.stats[1])}/{int(st2.stats[0])} XPBD particles asleep")
        for j in range(1, sim.xpbdOnlySteps + 1) if not device_loop else ():
            S.xpbdSimulationStep(sim, mpm, xpbd, dev, xpbd_only=True)
            sim.t += sim.dtxpbd
            if sim.xpbd_sleep_termination_ratio < 1.0:
                tot, slp = int(sim.numTotalXPBD.item()), int(sim.numSleepingXPBD.item())
                if tot > 0 and slp / tot >= sim.xpbd_sleep_termination_ratio:
                    log(f"    phase 2 stopped early: {slp}/{tot} XPBD particles asleep")
                    break
        # end of big step: deactivate XPBD particles below the datum
        minB, maxB = np.asarray(sim.minBounds, np.float64), np.asarray(sim.maxBounds, np.float64)
        z_datum = args.xpbd_deactivation_z_datum if args.xpbd_deactivation_z_datum is not None else float(minB[2])
        check_status(dev, "phase 2", log)
        mpmRoutines.deactivate_and_teleport_xpbd_below_datum(sim.particle_x, sim.particle_v, sim.activeLabel,
                                                              sim.materialLabel, float(z_datum),
                                                              2.0 * float(maxB[2] - minB[2]))
        if sim.saveFlag:
            saved.append(save_state(sim, mpm, xpbd, sim.outputFolder, big, mon.counter, checkpoint=True))
    for loop in loops.values():
        loop.close()
    torch.cuda.synchronize(dev)
    log(f"simulation complete in {time.time() - start:.2f}s")
    return sim, mpm, xpbd, saved


def main(argv=None):
    argv = sys.argv[1:] if argv is None else list(argv)
    extra = argparse.ArgumentParser(add_help=False)
    extra.add_argument("--check_interval", type=int, default=1)
    extra.add_argument("--device_loop", action="store_true",
                       help="run the checks between XPBD steps on the device (one host sync per segment)")
    extra.add_argument("--device", type=str, default="cuda:0")
    extra.add_argument("--resort_interval", type=int, default=0,
                       help="re-sort the particles into block order every N substeps (0: only at set-up)")
    ex, rest = extra.parse_known_args(argv)
    args = get_args(rest)
    run(args, check_interval=max(1, ex.check_interval), device=ex.device, device_loop=ex.device_loop,
        resort_interval=max(0, ex.resort_interval))


if __name__ == "__main__":
    main()
