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


def test_tensor_core_inference_matches_bf16_emulation():
    """tcgen05 MMA path (BF16 operands, FP32 accumulate) against the same
    network with every layer input rounded to BF16 on the CPU; and within the
    BF16 envelope of the FP32 forward."""
    import torch
    net = _net(3)
    x, _ = net.samples(1000, 13)          # 7 full 128-row tiles and a partial one
    y_tc = net.infer(x)
    y32 = net.forward_fp32(x)
    torch.cuda.synchronize()
    from mpmwarpydw_b200.bind import read_status
    assert read_status(x.device) == 0
    emu, _ = M.forward(net.params.cpu().numpy(), x.cpu().numpy(), bf16_activations=True)
    a = y_tc.cpu().numpy()
    assert np.all(np.isfinite(a))
    assert _rel(a, emu) <= 1e-2
    assert float(np.mean(np.abs(a - emu))) <= 1e-3 * float(np.mean(np.abs(emu)))
    assert _rel(a, y32.cpu().numpy()) <= 5e-2


def test_samples_satisfy_radial_return_identities():
    """Targets of a radial return: the deviatoric part of e_ret - e is
    anti-parallel to dev e, and its trace is 3 beta dgamma with
    dgamma = d_acc / sqrt(2/3)."""
    import torch
    net = _net(4)
    x, y = net.samples(20000, 14)
    torch.cuda.synchronize()
    x, y = x.cpu().numpy().astype(np.float64), y.cpu().numpy().astype(np.float64)
    d = x[:, :3]
    dd = d - d.mean(1, keepdims=True)
    de = y[:, :3]
    dde = de - de.mean(1, keepdims=True)
    plastic = y[:, 3] > 0
    assert plastic.mean() > 0.99
    cos = np.sum(dd * dde, 1) / (np.linalg.norm(dd, axis=1) * np.linalg.norm(dde, axis=1) + 1e-30)
    assert np.all(cos[plastic] < -0.999)
    beta = x[:, 5]
    tr = de.sum(1)
    expect = 3.0 * beta * y[:, 3] / np.sqrt(2.0 / 3.0)
    assert np.max(np.abs(tr - expect)[plastic]) <= 1e-5 * (np.max(np.abs(expect)) + 1e-6)


def test_training_gain():
    """What training gains: validation error of the trained network against
    the same network untrained, on fresh samples (printed)."""
    import torch
    net = _net(5)
    x, y = net.samples(1_000_000, 15)
    xv, yv = net.samples(50_000, 16)
    l0 = float(((net.infer(xv) - yv) ** 2).mean().item())
    losses = net.train(x, y, steps=1500, batch=8192)
    torch.cuda.synchronize()
    l1 = float(((net.infer(xv) - yv) ** 2).mean().item())
    print(f"surrogate validation MSE: untrained {l0:.3e}, trained {l1:.3e} (train loss {losses[0]:.2e} -> {losses[-1]:.2e})")
    assert l1 <= 1e-2 * l0


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
    x, y = net.samples(2_000_000, 17)
    net.train(x, y, steps=6000, batch=16384)
    sim, mpm, xpbd = small_scene(seed=21)
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
    plastic = s64.particle_accumulated_strain > to_oracle(*small_scene(seed=21), np.float64).particle_accumulated_strain
    mpm_now = (s64.materialLabel <= 1) & plastic
    d = (g["particle_stress"].reshape(-1, 9) - s64.particle_stress.reshape(-1, 9))[mpm_now]
    ref = s64.particle_stress.reshape(-1, 9)[mpm_now]
    err = float(np.linalg.norm(d) / np.linalg.norm(ref))
    mism = int((g["materialLabel"] != s64.materialLabel).sum())
    print(f"surrogate stress phase: {st}, plastic particles {int(mpm_now.sum())}, "
          f"norm-wise stress error vs FP64 {err:.2e}, label mismatches {mism}")
    assert st["candidates"] > 50
    assert err <= 1e-3
    assert mism <= max(1, st["candidates"] // 100)
