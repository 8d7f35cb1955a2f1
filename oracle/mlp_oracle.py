"""FP64 numpy restatement of the return-map surrogate network (TEST
INFRASTRUCTURE ONLY: loaded by tests/ as the CPU reference of the library's
MLP kernels; the product never imports it).

Same definitions as include/mpmw_mlp.h: 8 -> 64 -> 64 -> 64 -> 4, SiLU after the
hidden layers, parameters packed W1 b1 W2 b2 W3 b3 W4 b4 (W[out][in]); the
hidden layers' weights W1..W3 are rounded to BF16 (round to nearest even)
before use, W4 and the biases are not.  ``split_activations=True`` rounds the
inputs of the three hidden layers to the sum of two BF16 terms (hi = bf16(a),
lo = bf16(a - hi)), which is what the tensor-core inference kernel feeds its
MMAs.  :func:`targets` restates the sample labels (the radial return's ratios).
"""
from __future__ import annotations

import numpy as np

OFFSETS = dict(W1=(0, (64, 8)), b1=(512, (64,)), W2=(576, (64, 64)), b2=(4672, (64,)), W3=(4736, (64, 64)),
               b3=(8832, (64,)), W4=(8896, (4, 64)), b4=(9152, (4,)))


def bf16_round(a):
    """Round float32 values to the nearest bfloat16 (ties to even), returned as float64."""
    b = np.ascontiguousarray(np.asarray(a, np.float32)).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, np.float64)
    out = {}
    for k, (off, shape) in OFFSETS.items():
        n = int(np.prod(shape))
        out[k] = p[off:off + n].reshape(shape)
    return out


def _silu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return z * s, s * (1.0 + z * (1.0 - s))


def split_round(a):
    """a as the sum of its two BF16 terms hi = bf16(a), lo = bf16(a - hi)."""
    a32 = np.asarray(a, np.float32)
    hi = bf16_round(a32)
    lo = bf16_round((a32.astype(np.float64) - hi).astype(np.float32))
    return hi + lo


def forward(p, x, split_activations=False):
    """Outputs and the cache for backward."""
    P = unpack(p)
    W = {k: bf16_round(P[k].astype(np.float32)) for k in ("W1", "W2", "W3")}
    W["W4"] = P["W4"].astype(np.float32).astype(np.float64)
    r = split_round if split_activations else (lambda a: np.asarray(a, np.float64))
    a0 = r(np.asarray(x, np.float32))
    z1 = a0 @ W["W1"].T + P["b1"]; a1, d1 = _silu(z1)
    z2 = r(a1) @ W["W2"].T + P["b2"]; a2, d2 = _silu(z2)
    z3 = r(a2) @ W["W3"].T + P["b3"]; a3, d3 = _silu(z3)
    out = a3 @ W["W4"].T + P["b4"]
    return out, (a0, a1, a2, a3, d1, d2, d3, W)


def loss_and_grad(p, x, y):
    """mean((out - y)^2) over all entries and its gradient (straight-through
    through the BF16 rounding of the hidden layers' weights), packed like p."""
    out, (a0, a1, a2, a3, d1, d2, d3, W) = forward(p, x)
    r = out - np.asarray(y, np.float64)
    n = r.size
    loss = float(np.sum(r * r) / n)
    g4 = 2.0 * r / n
    grads = {"W4": g4.T @ a3, "b4": g4.sum(0)}
    gz3 = (g4 @ W["W4"]) * d3
    grads.update(W3=gz3.T @ a2, b3=gz3.sum(0))
    gz2 = (gz3 @ W["W3"]) * d2
    grads.update(W2=gz2.T @ a1, b2=gz2.sum(0))
    gz1 = (gz2 @ W["W2"]) * d1
    grads.update(W1=gz1.T @ a0, b1=gz1.sum(0))
    g = np.zeros(9156)
    for k, (off, shape) in OFFSETS.items():
        g[off:off + int(np.prod(shape))] = grads[k].ravel()
    return loss, g


def dp_return_principal(e, mu, lam, ys, alpha, beta, D):
    """The reference's principal-space radial return (utils/mpmRoutines.py:339-453)
    for one trial state: (e_ret, d_acc) or None if the trial is elastic."""
    e = np.asarray(e, np.float64)
    tr = e.sum()
    ed = e - tr / 3.0
    tau = 2.0 * mu * e + lam * tr
    p = tau.sum() / 3.0
    seq = np.sqrt(np.sum((tau - p) ** 2))
    ye = (1.0 - D) * (ys - alpha * p)
    if not (seq > ye):
        return None
    edn = np.sqrt(np.sum(ed * ed)) + 1e-6
    dg = edn - ye / (2.0 * mu)
    return e - (dg / edn) * ed + beta * dg, np.sqrt(2.0 / 3.0) * dg


def targets(e, mu, lam, ys, alpha, beta, D):
    """The sample labels of one plastic trial (include/mpmw_mlp.h): (ln rho,
    ln(1 - rho), beta, sqrt(2/3)) with rho = yield / (2 mu |dev e|), and the
    return they encode, e_ret = e + (rho n / (n + 1e-6) - 1) dev e + beta dgamma,
    dgamma = n (1 - rho) + 1e-6, which equals dp_return_principal's."""
    e = np.asarray(e, np.float64)
    tr = e.sum()
    ed = e - tr / 3.0
    n = np.sqrt(np.sum(ed * ed))
    p = (2.0 * mu / 3.0 + lam) * tr
    rho = (1.0 - D) * (ys - alpha * p) / (2.0 * mu * n)
    y = np.array([np.log(rho), max(np.log1p(-rho), -12.0), beta, np.sqrt(2.0 / 3.0)])
    dg = n * (1.0 - rho) + 1e-6
    e_ret = e + (rho * n / (n + 1e-6) - 1.0) * ed + beta * dg
    return y, e_ret, np.sqrt(2.0 / 3.0) * dg
