#!/usr/bin/env python
"""Throughput benchmark of the MPM substep: particle-updates/s on the
3,873,600-particle tunnel domain (200x100x200 lattice at 0.5 m minus a 10 m
tunnel, geostatic pre-stress, Drucker-Prager, dx = 1 m, dt = 5e-5 s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one MPM substep (P2G, grid update, G2P with the next substep's
return map fused in).  ``value`` is device-timed (CUDA events, state resident
in HBM; the 1.3 GB working set is larger than L2, so no flush is needed).
``e2e`` runs the drop-in per-step API (``mpmSimulationStep`` + the per-step
statistics the driver reads back) with the full particle state uploaded from
pinned host memory at the start and downloaded at the end of the timed region.
``--impl reference`` times the CPU oracle (the reference's algorithm restated
in C, OpenMP on all host cores) on a bounded sample of the same workload.
Multi-GPU (torchrun): every rank runs an independent replica (the scene does
not shard); value = all ranks' updates / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "MPM particle-updates/s at 4M, learned vs plain return map at ≤1e-3 stress err"
UNIT = "particle-updates/s"
PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "source": "fallback"}
HBM_NOMINAL_GBS = 7700.0  # B200 HBM3e, HGX nominal: fractions are also reported against it


def load_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        d["source"] = "measured"
        return d
    return dict(PEAKS_FALLBACK)


class ClockSampler:
    """nvidia-smi sampling of SM clock / throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, period_ms=50):
        self.proc = None
        self.gpu = gpu_index
        self.period = period_ms
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-i", str(self.gpu),
                 f"-lms", str(self.period)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, smax, reasons, power = [], None, set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
                power.append(float(f[3]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        busy = [s for s in sm if smax and s > 0.5 * smax] or sm
        return {"sm_mhz": statistics.median(busy), "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


# --------------------------------------------------------------------------
# algorithmic bytes of one particle-substep (elastic path; plastic-only fields
# are extra), as the substep's data flow defines them when P2G, the grid
# update, G2P and the return map each move their own operands:
#   P2G reads x 12, v 12, C 36, stress 24, mass 4, vol 4, labels 8      = 100
#   G2P + return map read x 12, labels 8, F 36, 9 material floats 36,
#   accumulated strain 4, damage 4                                        = 100
#   writes x 12, v 12, C 36, F 36, stress 24, acc 4, damage 4, ys 4       = 132
# per grid node: P2G result 16 W, grid pass 16 R + 12 W, G2P 12 R         =  56
# --------------------------------------------------------------------------
SUBSTEP_BYTES_P = 332
SUBSTEP_BYTES_NODE = 56
GRID_PASS_BYTES_NODE = 28   # the grid update's own share of the 56
# What the fused G2P->stress->P2G kernel must move at minimum for the same
# work: reads x 12, labels 8, F 36, mu lam ys alpha damage 20, eta_shear
# eta_bulk 8, mass vol 8; writes x 12, F 36 (v, C and the stress stay in
# registers); per node it reads v 16 and adds into mv 16.
FUSED_MIN_BYTES_P = (12 + 8 + 36 + 20 + 8 + 8) + (12 + 36)                        # 140
FUSED_MIN_BYTES_NODE = 32
# the getArgs defaults switch on the covariance update (+48 B: cov read and
# written, 6 floats) and the volumetric locking correction (+152 B: pass 1 reads
# x 12, C 36, vol 4, labels 8; pass 2 reads x 12, C 36, labels 8 and writes C 36)
VLC_COV_EXTRA_BYTES_P = 48 + 152

# DRAM bytes of one k_g2p2g launch on the 3,873,600-particle tunnel, measured by
# ncu (dram__bytes_read.sum + dram__bytes_write.sum, one launch, separate run);
# not measured by this script.  Update it with the kernel.
TRAFFIC_NCU = {"g2p2g": 629_440_256}
TRAFFIC_SOURCE = "ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_g2p2g launch in a separate run " \
                 "(profiles/traffic_tunnel_full.md), not measured by this run"


def setup(device, sort=True):
    import torch

    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.engine import sort_particles
    d = domains.tunnel()
    sim, mpm, xpbd = domains.build(d, device=device)
    if sort:
        sort_particles(sim, mpm, xpbd)
    torch.cuda.synchronize(device)
    return d, sim, mpm, xpbd


def run_ours(a):
    import torch
    import torch.distributed as dist

    from mpmwarpydw_b200 import _lib
    from mpmwarpydw_b200.bind import (grid_from_state, params_from_states, particles_from_states, read_status,
                                      status_word, workspace)
    from mpmwarpydw_b200.utils import simulationRoutines as S

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)  # before the process group, so NCCL binds this rank's GPU
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    L = _lib.lib()
    d, sim, mpm, xpbd = setup(dev)
    N = sim.nPoints
    G = int(np.prod(mpm.gridDims))
    P = particles_from_states(sim, mpm, xpbd)
    Gs = grid_from_state(mpm)
    prm = params_from_states(sim, mpm)
    st = status_word(dev).data_ptr()
    stream = torch.cuda.current_stream(dev)
    sh = int(stream.cuda_stream)
    ws = workspace(mpm, N, dev)

    def chk(rc, what):
        _lib.check(rc, what)

    ws_ptr, ws_n = ws.data_ptr(), ws.numel()

    from mpmwarpydw_b200.utils.xpbdRoutines import xpbd_step
    ratio = max(1, int(sim.mpmStepsPerXpbdStep))
    counter = [0]
    launches = [0]

    def run(k):
        # k substeps as the driver steps them (runMPMYDW.py:677-682): an XPBD step
        # follows the MPM substep at every counter % mpmStepsPerXpbdStep == 0
        # (counter > 0).  The MPM substeps between two XPBD steps are one library
        # call: stress + P2G, then per substep grid update (+ accumulator clear)
        # and the fused G2P->stress->P2G kernel, ending with the plain G2P.
        left = int(k)
        while left > 0:
            c = counter[0]
            nxt = ratio if c == 0 else ((c + ratio - 1) // ratio) * ratio
            m = min(left, nxt - c + 1)
            chk(L.mpmw_run_substeps(P, Gs, prm, m, st, ws_ptr, ws_n, sh), "run_substeps")
            launches[0] += 4 + 3 * (m - 1) + 2
            if c + m - 1 == nxt:
                xpbd_step(sim, mpm, xpbd)
                launches[0] += 20
            counter[0] += m
            left -= m

    # The tunnel lattice puts every second particle on a stencil-base boundary;
    # once the particles move they split between neighbouring cells and the
    # scatter has about twice the segments.  Run the settle substeps first so
    # the timed substeps are all in that (slower, long-run) regime.
    run(a.settle)
    torch.cuda.synchronize(dev)
    clocks = ClockSampler(local)
    clocks.start()
    run(a.warmup)
    torch.cuda.synchronize(dev)
    time.sleep(0.3)  # sampler has a few samples before the timed region
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    launches[0] = 0
    t0.record(stream)
    run(a.steps)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks.stop()
    ms = t0.elapsed_time(t1)
    status = read_status(dev)
    n_active_mpm = int(((sim.activeLabel == 1) & (sim.materialLabel <= 1)).sum().item())
    if world > 1:
        t = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # ---------------- per-kernel breakdown (outside the timed region) ----------------
    # the same kernels launched one by one with CUDA events between them: grid
    # update, accumulator clear, fused G2P->stress->P2G (its SVD-path list kernel included)
    kb = min(a.steps, 100)
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(kb)]
    chk(L.mpmw_stress(P, prm, st, sh), "stress")
    mpm._grid_mv.t.zero_()
    chk(L.mpmw_p2g(P, Gs, prm, st, sh), "p2g")
    for k in range(kb):
        e = evs[k]
        e[0].record(stream)
        chk(L.mpmw_grid_update(Gs, prm, sh), "grid")
        e[1].record(stream)
        mpm._grid_mv.t.zero_()
        e[2].record(stream)
        chk(L.mpmw_g2p2g(P, Gs, prm, 1 if k == kb - 1 else 0, st, ws_ptr, ws_n, sh), "g2p2g")
        e[3].record(stream)
    chk(L.mpmw_grid_update(Gs, prm, sh), "grid")
    chk(L.mpmw_g2p(P, Gs, prm, st, sh), "g2p")
    torch.cuda.synchronize(dev)
    per = {"grid": 0.0, "memset": 0.0, "g2p2g": 0.0}
    for e in evs:
        per["grid"] += e[0].elapsed_time(e[1])
        per["memset"] += e[1].elapsed_time(e[2])
        per["g2p2g"] += e[2].elapsed_time(e[3])
    status |= read_status(dev)

    # ---------------- end to end through the drop-in per-step API ----------------
    e2e = run_e2e(a, sim, mpm, xpbd, dev, S, world)

    peaks = load_peaks()
    hbm = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    K = a.steps
    dom = "g2p2g"
    dom_ms = per[dom] / kb
    # one fused launch carries one substep of every particle and the substep's
    # node traffic except the grid pass (a launch of its own)
    alg_dom = SUBSTEP_BYTES_P * N + (SUBSTEP_BYTES_NODE - GRID_PASS_BYTES_NODE) * G
    achieved = alg_dom / (dom_ms * 1e-3) / 1e9
    fused_min = FUSED_MIN_BYTES_P * N + FUSED_MIN_BYTES_NODE * G
    step_bytes = SUBSTEP_BYTES_P * N + SUBSTEP_BYTES_NODE * G
    traffic = TRAFFIC_NCU.get(dom)
    value = N * K * world / (ms * 1e-3)
    variant = run_vlc_cov_variant(a, sim, mpm, xpbd, dev, P, Gs, st, ws_ptr, ws_n, sh, hbm) if world == 1 else None
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": a.warmup,
        "ms_per_step": ms / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded tunnel domain; reference HDF5 inputs not used)",
        "config": {"workload": "tunnel 3,873,600 particles (200x100x200 @0.5 m minus r=10 m tunnel), grid 120x70x120 "
                               "dx=1 m, Drucker-Prager, dt=5e-5 s; K substeps stepped as the driver: MPM substeps "
                               "through mpmw_run_substeps (G2P, return map and next P2G fused), an XPBD step "
                               f"(hash, contacts, sleep, impulses) every {ratio} substeps",
                   "particles": N, "grid_nodes": G, "active_mpm_particles_end": n_active_mpm,
                   "settle_substeps": a.settle, "volumetric_locking_correction": 0, "update_cov": 0,
                   "l2": "working set 1.3 GB > 126 MB L2, no flush", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "traffic_source": TRAFFIC_SOURCE if traffic else None,
                     "peak_source": f"{peaks.get('source')} (MEASURED_PEAKS.json hbm_gbs)" if peaks.get("source") == "measured" else "fallback 6650 GB/s",
                     "algorithmic_bytes_per_launch": alg_dom,
                     "bytes_per_particle": SUBSTEP_BYTES_P, "bytes_per_node": SUBSTEP_BYTES_NODE - GRID_PASS_BYTES_NODE,
                     "fused_min_bytes_per_launch": fused_min,
                     "fused_min_frac": fused_min / (dom_ms * 1e-3) / 1e9 / hbm,
                     "dram_GBps": (traffic / (dom_ms * 1e-3) / 1e9) if traffic else None,
                     "dram_frac": (traffic / (dom_ms * 1e-3) / 1e9 / hbm) if traffic else None,
                     "step_achieved_GBps": step_bytes / (ms / K * 1e-3) / 1e9,
                     "step_frac": step_bytes / (ms / K * 1e-3) / 1e9 / hbm,
                     "nominal_GBps": HBM_NOMINAL_GBS, "frac_nominal": achieved / HBM_NOMINAL_GBS},
        "kernel_ms_per_step": {k: v / kb for k, v in per.items()},
        "e2e": e2e,
        "variant_getargs_defaults": variant,
        "gpu_launches": launches[0],
        "status_word": status,
        "clocks": clocks.summary(),
    }
    if world == 1 and not a.no_surrogate:
        out["surrogate"] = surrogate_comparison(sim, mpm, xpbd, dev)
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(a)
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_vlc_cov_variant(a, sim, mpm, xpbd, dev, P, Gs, st, ws_ptr, ws_n, sh, hbm):
    """The same substeps at the getArgs defaults volumetric_locking_correction = 1
    and update_cov = 1 (each substep then runs stress + P2G, grid update, G2P
    and the two locking-correction passes as separate launches), timed with CUDA
    events after the main measurement; reported with its own bytes per
    particle (332 + 48 + 152 B)."""
    import torch

    from mpmwarpydw_b200 import _lib
    from mpmwarpydw_b200.bind import grid_from_state, params_from_states
    L = _lib.lib()
    k = max(1, int(a.variant_steps))
    old = (mpm.volumetric_locking_correction, mpm.update_cov)
    mpm.volumetric_locking_correction, mpm.update_cov = 1, 1
    try:
        prm = params_from_states(sim, mpm)
        G = grid_from_state(mpm)
        stream = torch.cuda.current_stream(dev)
        _lib.check(L.mpmw_run_substeps(P, G, prm, 3, st, ws_ptr, ws_n, sh), "run_substeps (vlc, cov)")
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(dev)
        e0.record(stream)
        _lib.check(L.mpmw_run_substeps(P, G, prm, k, st, ws_ptr, ws_n, sh), "run_substeps (vlc, cov)")
        e1.record(stream)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
    finally:
        mpm.volumetric_locking_correction, mpm.update_cov = old
    N, Gn = sim.nPoints, int(np.prod(mpm.gridDims))
    bp = SUBSTEP_BYTES_P + VLC_COV_EXTRA_BYTES_P
    step_bytes = bp * N + SUBSTEP_BYTES_NODE * Gn
    gbs = step_bytes / (ms / k * 1e-3) / 1e9
    return {"value": N * k / (ms * 1e-3), "unit": UNIT, "steps": k, "ms_per_step": ms / k,
            "volumetric_locking_correction": 1, "update_cov": 1, "bytes_per_particle": bp,
            "bytes_per_node": SUBSTEP_BYTES_NODE, "achieved_GBps": gbs, "frac": gbs / hbm,
            "note": "whole substep (all its launches) against the algorithmic bytes; the substeps are not fused "
                    "when the locking correction is on"}


def surrogate_comparison(sim, mpm, xpbd, dev, reps=10):
    """Plain vs learned return map in the stress phase.  The network is
    trained on the GPU first (seeded, timed separately).  The tunnel's trial
    state is then overwritten with the learned-return-map configuration's
    distributions (trial log strain |e| log-uniform in [1e-6, 1e-1] along
    random directions and frames, friction angle U(20, 45) deg, cohesion
    log-uniform in [0.1, 5] MPa, damage U(0, 1): domains.seed_plastic_trials),
    so that the stress phase has plastic trials to return; each stress phase
    runs `reps` times from that restored state, timed with CUDA events.  The
    timed surrogate phase audits 1 % of its returns against the exact one (the
    production setting); one more untimed pass audits every return, for the
    accuracy statistics.  The scene state is restored afterwards."""
    import torch

    from mpmwarpydw_b200 import _lib, domains
    from mpmwarpydw_b200.bind import params_from_states, particles_from_states, status_word
    from mpmwarpydw_b200.surrogate import ReturnMapSurrogate, compute_stress, stats_summary
    stream = torch.cuda.current_stream(dev)
    t0 = time.perf_counter()
    net = ReturnMapSurrogate(dev, seed=0)
    x, y = net.samples(4_000_000, 1)
    losses = net.train(x, y, steps=60000, batch=16384)
    torch.cuda.synchronize(dev)
    train_s = time.perf_counter() - t0
    del x, y
    tensors = _state_tensors(sim, mpm, xpbd)
    orig = [t.clone() for t in tensors]
    domains.seed_plastic_trials(sim, mpm, seed=3)
    acc = mpm._s_particle_accumulated_strain
    acc_idx = [i for i, t in enumerate(tensors) if t.data_ptr() == acc.data_ptr()][0]
    lab = sim._s_materialLabel
    snap = [t.clone() for t in tensors]

    def restore(src):
        for t, s0 in zip(tensors, src):
            t.copy_(s0)

    L = _lib.lib()
    P, prm = particles_from_states(sim, mpm, xpbd), params_from_states(sim, mpm)
    st = status_word(dev).data_ptr()
    stress = mpm._s_particle_stress

    def timed(fn):
        ts = []
        for r in range(reps + 2):
            restore(snap)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            torch.cuda.synchronize(dev)
            if r >= 2:
                ts.append(e0.elapsed_time(e1))
        return sorted(ts)[len(ts) // 2]

    ms_plain = timed(lambda: _lib.check(L.mpmw_stress(P, prm, st, stream.cuda_stream), "stress"))
    s_plain, lab_plain = stress.clone(), lab.clone()
    plastic = (acc > snap[acc_idx]) & (lab <= 1)
    stats = torch.zeros(_lib.SURR_NSTATS, dtype=torch.int32, device=dev)

    def surr(audit):
        stats.zero_()
        compute_stress(sim, mpm, xpbd, net, gate_tol=1e-3, audit=audit, audit_seed=7, stats=stats)

    ms_surr_full = timed(lambda: surr(1.0))
    summ_full = stats_summary(stats)
    ms_surr = timed(lambda: surr(0.01))
    flipped = lab != lab_plain
    keep = plastic & ~flipped
    d = (stress - s_plain)[:, keep]
    ref = s_plain[:, keep]
    err = float(torch.linalg.norm(d.double()) / torch.linalg.norm(ref.double()).clamp_min(1e-30)) if ref.numel() else 0.0
    n = sim.nPoints
    summ = stats_summary(stats)
    # the accuracy statistics come from the pass that audits every return; the
    # gate's counts are the same in both passes
    for k in ("audited", "audit_max_rel_err", "audit_mean_rel_err", "audit_within_1e-3", "audited_accepted",
              "accepted_audit_max_rel_err"):
        if k in summ_full:
            summ[k] = summ_full[k]
    restore(orig)
    return {"stress_phase_plain": n / (ms_plain * 1e-3), "stress_phase_surrogate": n / (ms_surr * 1e-3),
            "unit": "particle-updates/s", "speedup": ms_plain / ms_surr, "ms_plain": ms_plain, "ms_surrogate": ms_surr,
            "state": "tunnel particles with seeded plastic trials (|e| log-uniform [1e-6, 1e-1], friction angle "
                     "U(20,45) deg, cohesion log-uniform [0.1,5] MPa, damage U(0,1))",
            "particles": n, "plastic_particles": int(plastic.sum().item()), "label_differences": int(flipped.sum().item()),
            "ms_surrogate_full_audit": ms_surr_full, "audit_fraction_timed": 0.01,
            **summ, "stress_err_vs_plain_over_plastic": err, "gate_tol": 1e-3, "audit_fraction_stats": 1.0,
            "train_seconds": train_s, "train_loss_first_last": [losses[0], losses[-1]],
            "network": "8-64-64-64-4 SiLU; hidden layers tcgen05 BF16 weights with hi+lo BF16 activations, "
                       "FP32 accumulate; last layer FP32"}


def _state_tensors(sim, mpm, xpbd):
    """Every per-particle storage tensor of the three state objects."""
    from mpmwarpydw_b200.state import Mat33Field, ScalarField, Sym33Field, Vec3Field
    out = []
    for obj in (sim, mpm, xpbd):
        for cls in type(obj).__mro__:
            for name, desc in vars(cls).items():
                if isinstance(desc, (ScalarField, Vec3Field, Mat33Field, Sym33Field)):
                    t = desc.storage(obj)
                    if t is not None:
                        out.append(t)
    return out


def run_e2e(a, sim, mpm, xpbd, dev, S, world):
    import torch
    tensors = _state_tensors(sim, mpm, xpbd)
    host = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in tensors]
    for h, t in zip(host, tensors):
        h.copy_(t)
    stats_host = torch.empty(7, dtype=torch.float64, pin_memory=True)
    h2d = sum(t.numel() * t.element_size() for t in tensors)
    K = a.steps
    torch.cuda.synchronize(dev)
    stream = torch.cuda.current_stream(dev)
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    for h, t in zip(host, tensors):
        t.copy_(h, non_blocking=True)
    ratio = max(1, int(sim.mpmStepsPerXpbdStep))
    for counter in range(K):
        S.mpmSimulationStep(sim, mpm, xpbd, dev)
        if counter % ratio == 0 and counter > 0:
            S.xpbdSimulationStep(sim, mpm, xpbd, dev)
        stats_host.copy_(S.step_stats(sim, mpm), non_blocking=True)
        stream.synchronize()  # the driver reads residual / counts every step
    for h, t in zip(host, tensors):
        h.copy_(t, non_blocking=True)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    ms = t0.elapsed_time(t1)
    if world > 1:
        import torch.distributed as dist
        tt = torch.tensor([ms], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms = float(tt.item())
    return {"value": sim.nPoints * K * world / (ms * 1e-3), "unit": UNIT, "steps": K,
            "copies": f"the full particle state ({h2d} B) uploaded from pinned host memory before the first "
                      f"substep and downloaded after the last, amortised over these {K} substeps; the "
                      "statistics read back after every substep",
            "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": (h2d + 7 * 8 * K) / K,
            "api": "mpmwarpydw_b200.utils.simulationRoutines.mpmSimulationStep (+ xpbdSimulationStep every "
                   "mpmStepsPerXpbdStep) + step_stats read back per step",
            "ms_total": ms}


def _oracle_sample(m):
    """FP32 oracle state of the tunnel, built on the CPU: all 3,873,600
    particles when m is 0 (the GPU line's workload), else the first m (input
    order = the bottom slab of the lattice)."""
    from mpmwarpydw_b200 import domains
    from oracle.oracle import Oracle, build_state
    d = domains.tunnel()
    o = Oracle("f32_omp")
    s = build_state(o, d.x, d.vol, d.args(), d.dx, d.minBounds, d.gridDims, limit=(m or None))
    return o, s, d.n


def _sample_text(m, n):
    return f"all {n} tunnel particles" if m == n else f"the first {m} of {n} tunnel particles (bottom slab)"


def _time_oracle(o, s, steps=None, seconds=None):
    from oracle.oracle import mpm_step
    t = time.perf_counter()
    k = 0
    while (steps is not None and k < steps) or (steps is None and (k < 1 or (time.perf_counter() - t < seconds and k < 50))):
        mpm_step(o, s)
        k += 1
    return k, time.perf_counter() - t


def cpu_baseline(a):
    """Oracle (FP32, OpenMP on all host cores) substeps on a bounded sample of
    the tunnel workload."""
    o, s, n = _oracle_sample(a.cpu_sample)
    m = s.particle_x.shape[0]
    k, el = _time_oracle(o, s, seconds=a.cpu_seconds)
    cores = os.cpu_count() or 1
    return {"value": m * k / el, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"{k} substep(s) of {_sample_text(m, n)}, FP32 oracle (reference algorithm restated in C; "
                      f"the reference's Warp CPU path is not installable here or on the GPU box), "
                      f"OpenMP {cores} threads", "seconds": el, "same_config": m == n}


def run_reference(a):
    """Reference arm: the reference is Python + Warp and cannot run on this
    image, so its algorithm restated in C (the oracle, OpenMP on all host
    cores) is timed on a bounded sample of the same workload."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    o, s, n = _oracle_sample(a.cpu_sample)
    m = s.particle_x.shape[0]
    t1 = time.perf_counter()
    _time_oracle(o, s, steps=1)
    per = max(time.perf_counter() - t1, 1e-3)
    k, el = _time_oracle(o, s, steps=max(1, min(a.steps, int(180.0 / per))))
    cores = os.cpu_count() or 1
    v = m * k / el
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT,
        "n_gpus": int(os.environ.get("WORLD_SIZE", 1)), "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": el / k * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded tunnel domain)",
        "config": {"workload": f"tunnel: {_sample_text(m, n)} per substep, oracle substeps timed: {k}",
                   "same_config": m == n},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{_sample_text(m, n)} per substep, FP32 oracle (reference algorithm restated "
                                   f"in C), OpenMP {cores} threads"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def run_sweep(a):
    """The batched parameter sweep (64 Drucker-Prager block collapses of
    20,000-500,000 particles, seeded friction angle and cohesion; domains.
    sweep_scenes) as the sweep runner steps it: the scenes are sharded over the
    ranks by particle count (sweep.partition, no exchange while stepping), each
    rank concatenates its share into one batch (one launch per kernel over its
    scenes), tunes the launch configuration, and runs K substeps of every
    scene in one fused call.  value = all ranks' particle-updates / the
    max-over-ranks device time."""
    import torch
    import torch.distributed as dist

    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.bind import read_status
    from mpmwarpydw_b200.sweep import ConcatBatch, partition
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)
    scenes = domains.sweep_scenes()
    counts = [d.n for d in scenes]
    mine = partition(counts, world)[rank]
    b = ConcatBatch([scenes[i] for i in mine], device=dev)
    N = b.particles
    G = sum(int(np.prod(st[1].gridDims)) for st in b.states)
    b.tune(5, reuse=False)
    stream = torch.cuda.current_stream(dev)
    clocks = ClockSampler(local)
    clocks.start()
    b.step(a.warmup)
    torch.cuda.synchronize(dev)
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize(dev)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0.record(stream)
    b.step(a.steps)
    t1.record(stream)
    torch.cuda.synchronize(dev)
    if world > 1:
        dist.barrier()
    clocks.stop()
    ms = t0.elapsed_time(t1)
    status = b.check("bench sweep", log=lambda *x: None)
    totals = torch.tensor([ms, float(N)], device=dev, dtype=torch.float64)
    if world > 1:
        mx = totals[:1].clone()
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        n_all = totals[1:].clone()
        dist.all_reduce(n_all, op=dist.ReduceOp.SUM)
        ms, n_total = float(mx.item()), int(n_all.item())
    else:
        n_total = N
    K = a.steps
    # end to end: the rank's concatenated particle state uploaded from pinned
    # host memory, K substeps, the per-scene results read back
    fields = [t for t in b.fields.values() if t is not None]
    host = [torch.empty(t.shape, dtype=t.dtype, pin_memory=True) for t in fields]
    for h, t in zip(host, fields):
        h.copy_(t)
    h2d = sum(t.numel() * t.element_size() for t in fields)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for h, t in zip(host, fields):
        t.copy_(h, non_blocking=True)
    b.step(K)
    res = b.results()
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms_e2e = e0.elapsed_time(e1)
    if world > 1:
        tt = torch.tensor([ms_e2e], device=dev, dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_e2e = float(tt.item())
    peaks = load_peaks()
    hbm = float(peaks.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"]))
    step_bytes = SUBSTEP_BYTES_P * N + SUBSTEP_BYTES_NODE * G
    gbs = step_bytes / (ms / K * 1e-3) / 1e9
    out = {
        "metric": METRIC, "value": n_total * K / (ms * 1e-3), "unit": UNIT, "n_gpus": world, "steps": K,
        "warmup": a.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded sweep scenes)",
        "config": {"workload": "batched sweep: 64 Drucker-Prager block collapses (10 m cubes, 20,000-500,000 "
                               "particles, friction angle U(20,45) deg, cohesion log-uniform [0.1,5] MPa, seed 4), "
                               "scenes sharded over ranks by particle count, a rank's scenes in the tuned form (one "
                               "persistent launch, or one launch per kernel per scene group), K substeps of every "
                               "scene per timed call",
                   "particles_total": int(sum(counts)), "particles_rank0": N, "scenes_rank0": len(mine),
                   "grid_nodes_rank0": G, "tuned": {"groups": b.groups, "gather_tile": b.options[0],
                                                    "read_ahead": b.options[1],
                                                    "form": "one persistent launch for the fused substeps"
                                                    if b.groups == 0 else "one launch per kernel per scene group",
                                                    "candidates": {f"groups={g},tile={o[0]},ahead={o[1]}": r
                                                                   for (g, o), r in b.tuning.items()}},
                   "l2": "working set > 126 MB L2, no flush", "parallelism": f"scene shards x{world}"},
        "roofline": {"bound": "hbm", "kernel": "whole batched substep (fused G2P/return map/P2G + grid pass)",
                     "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm, "traffic": None,
                     "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if peaks.get("source") == "measured"
                     else "fallback 6650 GB/s", "bytes_per_particle": SUBSTEP_BYTES_P,
                     "bytes_per_node": SUBSTEP_BYTES_NODE},
        "e2e": {"value": n_total * K / (ms_e2e * 1e-3), "unit": UNIT, "steps": K,
                "copies": "each rank's concatenated particle state uploaded from pinned host memory, K substeps, "
                          "the per-scene results read back",
                "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": 64 * len(res) / K},
        "gpu_launches": 2 + 4 * K,
        "status_word": status,
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        d0 = scenes[0]
        from oracle.oracle import Oracle, build_state
        o = Oracle("f32_omp")
        st = build_state(o, d0.x, d0.vol, d0.args(), d0.dx, d0.minBounds, d0.gridDims, limit=(a.cpu_sample or None))
        k, el = _time_oracle(o, st, seconds=a.cpu_seconds)
        m = st.particle_x.shape[0]
        cores = os.cpu_count() or 1
        out["cpu_baseline"] = {"value": m * k / el, "unit": UNIT, "cores": cores, "kind": "port",
                               "sample": f"{k} substep(s) of sweep scene 0 ({m} particles), FP32 oracle "
                                         f"(reference algorithm restated in C), OpenMP {cores} threads",
                               "seconds": el}
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_resort_study(a):
    """The fused kernel's time as the material flows, with and without
    periodic re-sorting of the particles into block order on the device: the
    caving block (509,696 particles, undercut, lognormal E and cohesion, XPBD
    on: an XPBD step every 5 substeps) stepped 2,000 substeps as the driver
    steps it, re-sorted every `resort_every` substeps or never; the mean
    k_g2p2g launch time (CUDA events, 20 launches on a snapshot of the state)
    at the start and at the end.  One JSON line."""
    import torch

    from mpmwarpydw_b200 import _lib, domains
    from mpmwarpydw_b200.bind import (grid_from_state, params_from_states, particles_from_states, read_status,
                                      status_word, workspace)
    from mpmwarpydw_b200.engine import sort_particles
    from mpmwarpydw_b200.utils import simulationRoutines as S
    dev = torch.device("cuda", 0)
    L = _lib.lib()
    total, every = 2000, 100

    def g2p2g_ms(sim, mpm, xpbd, reps=20):
        tensors = _state_tensors(sim, mpm, xpbd) + [mpm._grid_mv.t, mpm._grid_v.t]
        snap = [t.clone() for t in tensors]
        P, G, prm = particles_from_states(sim, mpm, xpbd), grid_from_state(mpm), params_from_states(sim, mpm)
        st = status_word(dev).data_ptr()
        ws = workspace(mpm, sim.nPoints, dev)
        stream = torch.cuda.current_stream(dev)
        _lib.check(L.mpmw_run_substeps(P, G, prm, 2, st, ws.data_ptr(), ws.numel(), stream.cuda_stream), "warm")
        ts = []
        for _ in range(reps):
            mpm._grid_mv.t.zero_()
            _lib.check(L.mpmw_stress_p2g(P, G, prm, st, ws.data_ptr(), ws.numel(), stream.cuda_stream), "sp")
            _lib.check(L.mpmw_grid_update(G, prm, stream.cuda_stream), "grid")
            mpm._grid_mv.t.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            _lib.check(L.mpmw_g2p2g(P, G, prm, 0, st, ws.data_ptr(), ws.numel(), stream.cuda_stream), "g2p2g")
            e1.record(stream)
            torch.cuda.synchronize(dev)
            ts.append(e0.elapsed_time(e1))
            for t, s0 in zip(tensors, snap):
                t.copy_(s0)
        return sorted(ts)[len(ts) // 2]

    out = {"study": "fused kernel time over 2,000 substeps of the caving block, with and without re-sorting",
           "workload": "caving block, 509,696 particles, XPBD step every 5 substeps", "resort_every": every,
           "unit": "ms per k_g2p2g launch (median of 20)"}
    for resort in (False, True):
        sim, mpm, xpbd = domains.build(domains.caving_block(), device=dev)
        sort_particles(sim, mpm, xpbd)
        ratio = max(1, int(sim.mpmStepsPerXpbdStep))
        t_start = g2p2g_ms(sim, mpm, xpbd)
        t0 = time.perf_counter()
        c = 0
        while c < total:
            nxt = ratio if c == 0 else ((c + ratio - 1) // ratio) * ratio
            m = min(total - c, nxt - c + 1)
            S.run_mpm_substeps(sim, mpm, xpbd, m)
            if c + m - 1 == nxt:
                S.xpbdSimulationStep(sim, mpm, xpbd, dev)
            c += m
            if resort and c % every < m:
                sort_particles(sim, mpm, xpbd)
        torch.cuda.synchronize(dev)
        wall = time.perf_counter() - t0
        t_end = g2p2g_ms(sim, mpm, xpbd)
        xp = int((sim.materialLabel == 2).sum().item())
        out["resort" if resort else "no_resort"] = {"g2p2g_ms_start": t_start, "g2p2g_ms_end": t_end,
                                                    "wall_s_2000_substeps": wall, "xpbd_particles_end": xp,
                                                    "status_word": read_status(dev)}
    print(json.dumps(out))


def run_profile_xpbd(k):
    """K substeps of the caving block (509,696 particles) with an XPBD step
    every 5 substeps, after seeding 35 % of the particles as XPBD particles
    (damage 1, the phase transition's label), for ncu captures of the XPBD
    kernels; prints one status line."""
    import torch

    from mpmwarpydw_b200 import domains
    from mpmwarpydw_b200.bind import read_status
    from mpmwarpydw_b200.engine import sort_particles
    from mpmwarpydw_b200.utils import simulationRoutines as S
    dev = torch.device("cuda", 0)
    sim, mpm, xpbd = domains.build(domains.caving_block(), device=dev)
    sort_particles(sim, mpm, xpbd)
    g = torch.Generator(device=dev).manual_seed(5)
    xp = torch.rand(sim.nPoints, generator=g, device=dev) < 0.35
    sim.materialLabel.copy_(torch.where(xp, 2, sim.materialLabel))
    ratio = max(1, int(sim.mpmStepsPerXpbdStep))
    c = 0
    while c < k:
        nxt = ratio if c == 0 else ((c + ratio - 1) // ratio) * ratio
        m = min(k - c, nxt - c + 1)
        S.run_mpm_substeps(sim, mpm, xpbd, m)
        if c + m - 1 == nxt:
            S.xpbdSimulationStep(sim, mpm, xpbd, dev)
        c += m
    torch.cuda.synchronize(dev)
    print(json.dumps({"profile_xpbd": {"particles": sim.nPoints, "substeps": int(k), "xpbd_ratio": ratio,
                                       "xpbd_particles": int((sim.materialLabel == 2).sum().item()),
                                       "status_word": read_status(dev)}}))


def run_xpbd_study(a):
    """The XPBD step (utils/simulationRoutines.py:295-526) in its two forms --
    one persistent cooperative launch and one launch per pass -- on the caving
    block (509,696 particles, 35 % of them seeded as XPBD particles, 4
    iterations): CUDA-event time of each step, the forms alternating, median
    of 20 steps each after 3 warm-up steps.  One JSON line."""
    import torch

    from mpmwarpydw_b200 import _lib, domains
    from mpmwarpydw_b200.bind import read_status
    from mpmwarpydw_b200.engine import sort_particles
    from mpmwarpydw_b200.utils import simulationRoutines as S
    dev = torch.device("cuda", 0)
    L = _lib.lib()
    sim, mpm, xpbd = domains.build(domains.caving_block(), device=dev)
    sort_particles(sim, mpm, xpbd)
    g = torch.Generator(device=dev).manual_seed(5)
    xp = torch.rand(sim.nPoints, generator=g, device=dev) < 0.35
    sim.materialLabel.copy_(torch.where(xp, 2, sim.materialLabel))
    S.run_mpm_substeps(sim, mpm, xpbd, 5)
    times = {1: [], 0: []}
    stream = torch.cuda.current_stream(dev)
    try:
        for rep in range(23):
            for form in (1, 0):
                _lib.check(L.mpmw_xpbd_set_options(form), "xpbd options")
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                S.xpbdSimulationStep(sim, mpm, xpbd, dev)
                e1.record(stream)
                torch.cuda.synchronize(dev)
                if rep >= 3:
                    times[form].append(e0.elapsed_time(e1))
    finally:
        _lib.check(L.mpmw_xpbd_set_options(1), "xpbd options")
    med = {f: sorted(t)[len(t) // 2] for f, t in times.items()}
    print(json.dumps({"study": "XPBD step: one persistent launch vs one launch per pass",
                      "workload": "caving block, 509,696 particles, 35 % XPBD particles, 4 iterations",
                      "unit": "ms per XPBD step (median of 20)", "persistent": med[1], "per_pass": med[0],
                      "persistent_launches": int(L.mpmw_xpbd_persistent_launches()),
                      "xpbd_particles": int((sim.materialLabel == 2).sum().item()),
                      "status_word": read_status(dev)}))


def run_profile_mlp(n):
    """Tensor-core inference of the surrogate network on n samples (after a
    short training), for ncu captures of k_mlp_infer_tc; prints one line."""
    import torch

    from mpmwarpydw_b200.bind import read_status
    from mpmwarpydw_b200.surrogate import ReturnMapSurrogate
    dev = torch.device("cuda", 0)
    net = ReturnMapSurrogate(dev, seed=0)
    x, y = net.samples(int(n), 1)
    net.train(x, y, steps=200, batch=16384)
    for _ in range(3):
        out = net.infer(x)
    torch.cuda.synchronize(dev)
    print(json.dumps({"profile_mlp": {"samples": int(n), "mse": float(((out - y) ** 2).mean().item()),
                                      "status_word": read_status(dev)}}))


def run_profile_small(k):
    """K substeps of a 788,160-particle tunnel (120x60x120 lattice cells, same
    per-particle work as the bench workload) through mpmw_run_substeps, for
    ncu captures that must stay small; prints one status line."""
    import torch

    from mpmwarpydw_b200 import _lib, domains
    from mpmwarpydw_b200.bind import grid_from_state, params_from_states, particles_from_states, status_word, workspace
    from mpmwarpydw_b200.engine import sort_particles
    dev = torch.device("cuda", 0)
    d = domains.tunnel(nx=120, ny=60, nz=120)
    sim, mpm, xpbd = domains.build(d, device=dev)
    sort_particles(sim, mpm, xpbd)
    L = _lib.lib()
    P, G, prm = particles_from_states(sim, mpm, xpbd), grid_from_state(mpm), params_from_states(sim, mpm)
    ws = workspace(mpm, sim.nPoints, dev)
    st = status_word(dev)
    _lib.check(L.mpmw_run_substeps(P, G, prm, int(k), st.data_ptr(), ws.data_ptr(), ws.numel(),
                                   torch.cuda.current_stream(dev).cuda_stream), "run_substeps")
    torch.cuda.synchronize(dev)
    print(json.dumps({"profile_small": {"particles": sim.nPoints, "grid": list(mpm.gridDims), "substeps": int(k),
                                        "status_word": int(st.item())}}))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--profile-small", type=int, default=0, metavar="K",
                    help="run K substeps of the 788,160-particle tunnel and exit (small case for ncu)")
    ap.add_argument("--profile-xpbd", type=int, default=0, metavar="K",
                    help="K substeps of the caving block with 35%% XPBD particles (small case for ncu)")
    ap.add_argument("--profile-mlp", type=int, default=0, metavar="N",
                    help="tensor-core inference of the surrogate on N samples (small case for ncu)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--settle", type=int, default=200,
                    help="untimed substeps before the warm-up (the tunnel's particles leave their lattice cells)")
    ap.add_argument("--variant-steps", type=int, default=50,
                    help="substeps of the getArgs-default (VLC + covariance) variant")
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--study", choices=["resort", "xpbd"], default=None,
                    help="resort: the fused kernel's time over 2,000 caving-block substeps with and without "
                         "re-sorting; xpbd: the XPBD step as one persistent launch and as one launch per pass "
                         "(each prints its own JSON line, not a bench line)")
    ap.add_argument("--workload", choices=["tunnel", "sweep"], default="tunnel",
                    help="tunnel: the 3,873,600-particle tunnel (replicas over ranks); sweep: the batched "
                         "64-scene parameter sweep (scenes sharded over ranks)")
    ap.add_argument("--cpu-sample", type=int, default=0,
                    help="particles of the tunnel the CPU baseline steps (0: all, the GPU line's workload)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-surrogate", action="store_true", help="skip the plain-vs-learned return map comparison")
    a = ap.parse_args()
    if a.warmup < 3:
        a.warmup = 3
    if a.profile_small:
        run_profile_small(a.profile_small)
    elif a.profile_xpbd:
        run_profile_xpbd(a.profile_xpbd)
    elif a.profile_mlp:
        run_profile_mlp(a.profile_mlp)
    elif a.study == "resort":
        run_resort_study(a)
    elif a.study == "xpbd":
        run_xpbd_study(a)
    elif a.impl == "reference":
        run_reference(a)
    elif a.workload == "sweep":
        run_sweep(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
