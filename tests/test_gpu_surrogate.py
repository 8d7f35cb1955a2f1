"""The learned return-map surrogate's kernels against the CPU restatement of
the network (oracle/mlp_oracle.py, FP64): forward, loss and gradient, the
tensor-core inference, the training samples, and what training gains."""
import numpy as np
import pytest

from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / (np.max(np.abs(b)) + 1e-30))


def _net(seed=0):
    from mpmwarpydw_b200.surrogate import ReturnMapSurrogate
    return ReturnMapSurrogate("cuda:0", seed=seed)


def test_forward_matches_cpu():
    import torch
    net = _net(1)
    x, _ = net.samples(1000, 11)
    y = net.forward_fp32(x)
    torch.cuda.synchronize()
    ref, _ = M.forward(net.params.cpu().numpy(), x.cpu().numpy())
    assert _rel(y.cpu().numpy(), ref) <= 1e-5


def test_gradient_matches_cpu():
    """FP32 kernels vs the FP64 restatement: loss to 1e-5, every parameter
    block's gradient to 1e-4 of its magnitude."""
    import torch
    net = _net(2)
    x, y = net.samples(700, 12)           # not a multiple of the 64-sample tile
    loss, grad = net.loss_and_grad(x, y)
    torch.cuda.synchronize()
    l_ref, g_ref = M.loss_and_grad(net.params.cpu().numpy(), x.cpu().numpy(), y.cpu().numpy())
    assert abs(float(loss.item()) - l_ref) <= 1e-5 * l_ref
    g = grad.cpu().numpy()
    for name, (off, shape) in M.OFFSETS.items():
        n = int(np.prod(shape))
        assert _rel(g[off:off + n], g_ref[off:off + n]) <= 1e-4, name


def test_tensor_core_gradient_matches_cpu():
    """The tensor-core training kernel (mpmw_mlp_grad_tc) against the FP64
    restatement and the FP32 CUDA-core kernel on 700 samples (5 full 128-row
    CTAs and a partial one): the loss to 1e-5 (the forward pass carries split
    BF16 activations), every parameter block's gradient to 1e-2 norm-wise (the
    weight gradients take the layer inputs in BF16)."""
    import torch
    net = _net(2)
    x, y = net.samples(700, 12)
    l_tc, g_tc = net.loss_and_grad(x, y, tensor_cores=True)
    l_tc, g_tc = float(l_tc.item()), g_tc.clone().cpu().numpy()
    l_32, g_32 = net.loss_and_grad(x, y, tensor_cores=False)
    l_32, g_32 = float(l_32.item()), g_32.clone().cpu().numpy()
    torch.cuda.synchronize()
    from mpmwarpydw_b200.bind import read_status
    assert read_status(x.device) == 0
    l_ref, g_ref = M.loss_and_grad(net.params.cpu().numpy(), x.cpu().numpy(), y.cpu().numpy())
    assert abs(l_tc - l_ref) <= 1e-5 * l_ref and abs(l_tc - l_32) <= 1e-5 * l_ref
    for name, (off, shape) in M.OFFSETS.items():
        n = int(np.prod(shape))
        a, b, c = g_tc[off:off + n], g_ref[off:off + n], g_32[off:off + n]
        err = float(np.linalg.norm(a - b) / (np.linalg.norm(b) + 1e-30))
        assert err <= 1e-2, (name, err)
        assert float(np.linalg.norm(a - c) / (np.linalg.norm(c) + 1e-30)) <= 1e-2, name


def test_tensor_core_training_tracks_fp32_training():
    """Training on the tensor cores reaches the loss the FP32 kernels reach
    from the same start (3,000 Adam steps): within 1.5x, both below 2e-2."""
    import torch
    x, y = _net(7).samples(400_000, 18)
    out = []
    for tc in (True, False):
        net = _net(7)
        losses = net.train(x, y, steps=3000, batch=8192, tensor_cores=tc)
        torch.cuda.synchronize()
        out.append(float(np.mean(losses[-3:])))
    print(f"training loss after 3,000 steps: tensor cores {out[0]:.3e}, FP32 kernels {out[1]:.3e}")
    assert max(out) < 2e-2
    assert out[0] <= 1.5 * out[1]


def test_tensor_core_inference_matches_split_emulation():
    """tcgen05 MMA path (BF16 weights, every hidden-layer input fed as hi + lo
    BF16 terms, FP32 accumulate, FP32 last layer) against the same network
    with that rounding emulated on the CPU, and against the FP32 forward."""
    import torch
    net = _net(3)
    x, _ = net.samples(1000, 13)          # 7 full 128-row tiles and a partial one
    y_tc = net.infer(x)
    y32 = net.forward_fp32(x)
    torch.cuda.synchronize()
    from mpmwarpydw_b200.bind import read_status
    assert read_status(x.device) == 0
    emu, _ = M.forward(net.params.cpu().numpy(), x.cpu().numpy(), split_activations=True)
    a = y_tc.cpu().numpy()
    assert np.all(np.isfinite(a))
    assert _rel(a, emu) <= 1e-4
    assert _rel(a, y32.cpu().numpy()) <= 1e-4


def test_samples_satisfy_radial_return_identities():
    """Targets of a radial return: y[2] is the dilation beta (feature 5), y[3]
    is sqrt(2/3), rho + (1 - rho) = 1, and ln rho is the ratio the features
    define: (1 - D)(10^-f3 - alpha (1/3 + nu/(1 - 2 nu)) tr(e/|e|)) / |dev e/|e||."""
    import torch
    net = _net(4)
    x, y = net.samples(20000, 14)
    torch.cuda.synchronize()
    x, y = x.cpu().numpy().astype(np.float64), y.cpu().numpy().astype(np.float64)
    assert np.all(np.isfinite(y))
    assert np.max(np.abs(y[:, 2] - x[:, 5])) <= 1e-7
    assert np.max(np.abs(y[:, 3] - np.sqrt(2.0 / 3.0))) <= 1e-7
    rho = np.exp(y[:, 0])
    assert np.all((rho > 0) & (rho < 1))
    far = y[:, 1] > -12.0 + 1e-6          # targets not clamped at the floor
    assert np.max(np.abs(rho + np.exp(y[:, 1]) - 1.0)[far]) <= 1e-5
    d = x[:, :3]
    dd = d - d.mean(1, keepdims=True)
    nu = x[:, 7]
    c = 1.0 / 3.0 + nu / (1.0 - 2.0 * nu)
    rho_f = np.exp(x[:, 6]) * (10.0 ** (-x[:, 3]) - x[:, 4] * c * d.sum(1)) / np.linalg.norm(dd, axis=1)
    assert np.median(np.abs(np.log(rho_f) - y[:, 0])) <= 1e-5
    assert np.quantile(np.abs(np.log(rho_f) - y[:, 0]), 0.99) <= 1e-3


def _stress_phase_compare(net, n_side=60, seed=31):
    """The plain stress phase (mpmw_stress) and the surrogate's on the same
    seeded plastic trial state (config 3's distributions): (plain stress,
    surrogate stress, plastic mask, stats summary, ms plain, ms surrogate,
    particles whose material label differs between the two)."""
    import torch

    from mpmwarpydw_b200 import _lib, domains
    from mpmwarpydw_b200.bind import params_from_states, particles_from_states, status_word, stream_handle
    from mpmwarpydw_b200.surrogate import compute_stress, stats_summary
    d = domains.block_collapse(n_side=n_side, spacing=0.25, seed=seed)
    sim, mpm, xpbd = domains.build(d, device="cuda:0")
    domains.seed_plastic_trials(sim, mpm, seed=seed, emax=1e-2)
    fields = [mpm._s_particle_F, mpm._s_particle_stress, mpm._s_particle_accumulated_strain,
              mpm._s_particle_damage, mpm._s_ys, mpm._s_mu, mpm._s_lam, mpm._s_alpha,
              sim._s_materialLabel, sim._s_particle_v]
    snap = [t.clone() for t in fields]
    acc0 = mpm._s_particle_accumulated_strain.clone()

    def restore():
        for t, s0 in zip(fields, snap):
            t.copy_(s0)

    L = _lib.lib()
    P, prm = particles_from_states(sim, mpm, xpbd), params_from_states(sim, mpm)
    st = status_word("cuda:0")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    ev[0].record()
    _lib.check(L.mpmw_stress(P, prm, st.data_ptr(), stream_handle()), "stress")
    ev[1].record()
    torch.cuda.synchronize()
    plain = mpm._s_particle_stress.clone()
    lab_plain = sim._s_materialLabel.clone()
    plastic = (mpm._s_particle_accumulated_strain > acc0) & (sim._s_materialLabel <= 1)
    restore()
    stats = torch.zeros(_lib.SURR_NSTATS, dtype=torch.int32, device="cuda:0")
    ev[2].record()
    compute_stress(sim, mpm, xpbd, net, gate_tol=1e-3, audit=1.0, audit_seed=5, stats=stats)
    ev[3].record()
    torch.cuda.synchronize()
    surr = mpm._s_particle_stress.clone()
    flipped = sim._s_materialLabel != lab_plain
    return (plain, surr, plastic & ~flipped, stats_summary(stats), ev[0].elapsed_time(ev[1]),
            ev[2].elapsed_time(ev[3]), int(flipped.sum()))


def test_surrogate_against_plain_return_map():
    """What the trained network gains over the method without it.  On 216,000
    seeded plastic trial states (config 3's distributions, |e| up to 1e-2, the
    tensor form's range), the stress phase runs with the plain return map and
    with the surrogate (gate 1e-3, every return audited):
      - untrained, the gate rejects every surrogate return (all fall back);
      - trained, the gate accepts returns, every accepted and audited return
        is within 1e-3 (relative stress error against the exact return), and
        the stress over the plastic particles is within 1e-3 norm-wise of the
        plain path's (particles whose phase-transition label differs, a damage
        threshold reached with the predicted increment, are counted apart:
        at most 0.1 % of the candidates);
    the times of both phases are printed (the plain map is a closed form of a
    few dozen FLOPs; the network costs 17,920 per candidate)."""
    import torch
    net = _net(5)
    st0 = _stress_phase_compare(net)[3]
    x, y = net.samples(4_000_000, 15)
    losses = net.train(x, y, steps=40000, batch=16384)
    del x, y
    plain, surr, plastic, st1, ms_p, ms_s, flipped = _stress_phase_compare(net)
    d = (surr - plain)[:, plastic].double()
    err = float(torch.linalg.norm(d) / torch.linalg.norm(plain[:, plastic].double()))
    print(f"untrained: {st0}\ntrained (loss {losses[0]:.2e} -> {losses[-1]:.2e}): {st1}\n"
          f"plastic particles {int(plastic.sum())}, label differences {flipped}, stress error vs plain {err:.2e}, "
          f"stress phase plain {ms_p:.3f} ms, surrogate {ms_s:.3f} ms")
    assert st0["candidates"] > 10000 and st0["accepted"] == 0
    assert st1["candidates"] == st0["candidates"]
    assert st1["accepted"] > 0
    assert st1["audited_accepted"] == st1["accepted"]
    assert st1["accepted_audit_max_rel_err"] <= 1e-3
    assert flipped <= max(1, st1["candidates"] // 1000)
    assert err <= 1e-3


def test_surrogate_stress_phase_vs_fp64_oracle():
    """The stress phase with the trained surrogate for plastic returns (gate
    1e-3, every accepted return audited) against the FP64 oracle's plain stress
    phase on the parity scene: stress error at most 1e-3 norm-wise over the
    plastic particles, labels equal except at most 1 % of the surrogate
    candidates (damage thresholds reached with the predicted increment).
    Elastic and out-of-range particles take the exact path."""
    import torch

    from mpmwarpydw_b200.surrogate import ReturnMapSurrogate, compute_stress, stats_summary
    from tests.harness import gpu_fields, oracle, small_scene, to_oracle
    net = ReturnMapSurrogate("cuda:0", seed=6)
    x, y = net.samples(4_000_000, 17)
    net.train(x, y, steps=40000, batch=16384)
    sim, mpm, xpbd = small_scene(seed=21, n_side=30)
    s64 = to_oracle(sim, mpm, xpbd, np.float64)
    stats = compute_stress(sim, mpm, xpbd, net, gate_tol=1e-3, audit=1.0, audit_seed=3)
    torch.cuda.synchronize()
    o = oracle("f64")
    o.compute_stress_from_F_trial(
        s64.activeLabel, s64.materialLabel, s64.particle_x, s64.particle_v, s64.particle_x_initial_xpbd,
        s64.particle_v_initial_xpbd, s64.particle_F, s64.particle_F_trial, s64.mu, s64.lam, s64.ys, s64.hardening,
        s64.softening, s64.particle_density, s64.strainCriteria, s64.eff, s64.eta_shear, s64.eta_bulk, s64.particle_C,
        s64.particle_stress, s64.particle_accumulated_strain, s64.particle_damage, s64.constitutive_model, s64.alpha)
    g = gpu_fields(sim, mpm, xpbd)
    st = stats_summary(stats)
    plastic = s64.particle_accumulated_strain > to_oracle(*small_scene(seed=21, n_side=30),
                                                          np.float64).particle_accumulated_strain
    mpm_now = (s64.materialLabel <= 1) & plastic
    d = (g["particle_stress"].reshape(-1, 9) - s64.particle_stress.reshape(-1, 9))[mpm_now]
    ref = s64.particle_stress.reshape(-1, 9)[mpm_now]
    err = float(np.linalg.norm(d) / np.linalg.norm(ref))
    mism = int((g["materialLabel"] != s64.materialLabel).sum())
    print(f"surrogate stress phase: {st}, plastic particles {int(mpm_now.sum())}, "
          f"norm-wise stress error vs FP64 {err:.2e}, label mismatches {mism}")
    assert st["candidates"] > 1000
    assert st["accepted"] > 0
    assert st["accepted_audit_max_rel_err"] <= 1e-3
    assert err <= 1e-3
    assert mism <= max(1, st["candidates"] // 100)
