"""Learned surrogate of the Drucker-Prager return map (no counterpart in the
reference, whose return map is closed form: utils/mpmRoutines.py:314-453).

An MLP 8 -> 64 -> 64 -> 64 -> 4 (SiLU) maps the features of a plastic trial
state to its return (feature and target definitions in include/mpmw_mlp.h).
It is trained on the GPU by the library's own kernels: labelled samples from
the plain return map (``mpmw_dp_samples``), forward and backward on the
tensor cores (``mpmw_mlp_grad_tc``; ``mpmw_mlp_grad`` is the FP32 CUDA-core
version) with the hidden weights rounded to BF16, Adam (``mpmw_mlp_adam``).
Inference runs on the tensor cores (``mpmw_mlp_infer_tc``: tcgen05.mma with
BF16 weights, each hidden-layer input split into hi + lo BF16 terms, FP32
accumulation in tensor memory; the last layer in FP32).
"""
from __future__ import annotations

import math

import torch

from . import _lib
from .bind import params_from_states, particles_from_states, status_word, stream_handle

OFFSETS = dict(W1=(0, (64, 8)), b1=(512, (64,)), W2=(576, (64, 64)), b2=(4672, (64,)), W3=(4736, (64, 64)),
               b3=(8832, (64,)), W4=(8896, (4, 64)), b4=(9152, (4,)))


def init_params(seed: int = 0, device="cuda") -> torch.Tensor:
    """Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights and biases, as torch.nn.Linear."""
    g = torch.Generator().manual_seed(seed)
    p = torch.empty(_lib.MLP_NPARAM, dtype=torch.float32)
    for name, (off, shape) in OFFSETS.items():
        fan_in = shape[1] if len(shape) == 2 else (8 if name == "b1" else 64)
        bound = 1.0 / math.sqrt(fan_in)
        n = int(torch.tensor(shape).prod())
        p[off:off + n] = (torch.rand(n, generator=g) * 2 - 1) * bound
    return p.to(device)


class ReturnMapSurrogate:
    """Parameters, optimizer state and packed tensor-core weights on one device."""

    def __init__(self, device="cuda:0", seed: int = 0):
        self.device = torch.device(device)
        self.params = init_params(seed, self.device)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.grad = torch.zeros_like(self.params)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.packed = torch.zeros(_lib.MLP_PACKED_BYTES // 2, dtype=torch.int16, device=self.device)
        self.step = 0
        self._packed_step = -1

    @staticmethod
    def samples(n: int, seed: int, device="cuda:0"):
        """n labelled plastic trial states (features [n, 8], targets [n, 4])."""
        x = torch.empty(n, _lib.MLP_IN, dtype=torch.float32, device=device)
        y = torch.empty(n, _lib.MLP_OUT, dtype=torch.float32, device=device)
        _lib.check(_lib.lib().mpmw_dp_samples(n, seed, x.data_ptr(), y.data_ptr(), stream_handle()), "dp_samples")
        return x, y

    def loss_and_grad(self, x, y, tensor_cores: bool = False):
        """Loss and gradient of (x, y): FP32 CUDA-core kernel, or the
        tensor-core kernel (mpmw_mlp_grad_tc)."""
        L = _lib.lib()
        if tensor_cores:
            st = status_word(x.device)
            _lib.check(L.mpmw_mlp_grad_tc(self.params.data_ptr(), x.data_ptr(), y.data_ptr(), x.shape[0],
                                          self.grad.data_ptr(), self.loss.data_ptr(), st.data_ptr(),
                                          stream_handle()), "mlp_grad_tc")
        else:
            _lib.check(L.mpmw_mlp_grad(self.params.data_ptr(), x.data_ptr(), y.data_ptr(), x.shape[0],
                                       self.grad.data_ptr(), self.loss.data_ptr(), stream_handle()), "mlp_grad")
        return self.loss, self.grad

    def train(self, x, y, steps: int, batch: int = 8192, lr: float = 2e-3, lr_end: float = 2e-5,
              tensor_cores: bool = True):
        """Adam over contiguous mini-batches of (x, y); cosine learning-rate
        decay.  The loss and gradient of each batch come from the tensor-core
        kernel by default (``tensor_cores=False``: the FP32 CUDA-core one)."""
        n = x.shape[0]
        L = _lib.lib()
        losses = []
        for k in range(steps):
            i0 = (k * batch) % max(1, n - batch + 1)
            xb, yb = x[i0:i0 + batch], y[i0:i0 + batch]
            self.loss_and_grad(xb, yb, tensor_cores)
            self.step += 1
            lrk = lr_end + 0.5 * (lr - lr_end) * (1 + math.cos(math.pi * k / max(1, steps)))
            _lib.check(L.mpmw_mlp_adam(self.params.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(),
                                       self.v.data_ptr(), self.step, lrk, stream_handle()), "mlp_adam")
            if k % 200 == 0 or k == steps - 1:
                losses.append(float(self.loss.item()))
        return losses

    def forward_fp32(self, x):
        y = torch.empty(x.shape[0], _lib.MLP_OUT, dtype=torch.float32, device=x.device)
        _lib.check(_lib.lib().mpmw_mlp_forward(self.params.data_ptr(), x.data_ptr(), x.shape[0], y.data_ptr(),
                                               stream_handle()), "mlp_forward")
        return y

    def pack(self):
        if self._packed_step != self.step:
            _lib.check(_lib.lib().mpmw_mlp_pack(self.params.data_ptr(), self.packed.data_ptr(), stream_handle()),
                       "mlp_pack")
            self._packed_step = self.step
        return self.packed

    def infer(self, x, out=None):
        """Tensor-core inference (tcgen05, BF16 weights, split BF16 activations, FP32 accumulation)."""
        packed = self.pack()
        y = out if out is not None else torch.empty(x.shape[0], _lib.MLP_OUT, dtype=torch.float32, device=x.device)
        st = status_word(x.device)
        _lib.check(_lib.lib().mpmw_mlp_infer_tc(packed.data_ptr(), self.params.data_ptr(), x.data_ptr(), x.shape[0],
                                                y.data_ptr(), st.data_ptr(), stream_handle()), "mlp_infer_tc")
        return y

    def state_dict(self):
        return {"params": self.params.detach().cpu(), "step": self.step}

    def load_state_dict(self, d):
        self.params.copy_(d["params"].to(self.device))
        self.step = int(d.get("step", 0))
        self._packed_step = -1


def compute_stress(sim, mpm, xpbd, net: ReturnMapSurrogate, gate_tol: float = 1e-3, audit: float = 0.01,
                   audit_seed: int = 0, stats=None):
    """The stress phase (compute_stress_from_F_trial) with the surrogate for
    plastic returns: gate, audit and exact fallback as mpmw_stress_surrogate.
    Returns the (8,) int32 device stats (see :func:`stats_summary`),
    accumulated into ``stats``."""
    dev = sim.device
    if stats is None:
        stats = torch.zeros(_lib.SURR_NSTATS, dtype=torch.int32, device=dev)
    n = sim.nPoints
    need = int(_lib.lib().mpmw_surrogate_workspace_bytes(n))
    ws = getattr(mpm, "_mpmw_surr_ws", None)
    if ws is None or ws.numel() < need:
        ws = torch.empty(max(need, 256), dtype=torch.uint8, device=dev)
        mpm._mpmw_surr_ws = ws
    P = particles_from_states(sim, mpm, xpbd)
    prm = params_from_states(sim, mpm)
    packed = net.pack()
    st = status_word(dev)
    _lib.check(_lib.lib().mpmw_stress_surrogate(P, prm, packed.data_ptr(), net.params.data_ptr(), float(gate_tol),
                                                int(round(audit * 1000)), int(audit_seed), stats.data_ptr(),
                                                st.data_ptr(), ws.data_ptr(), ws.numel(), stream_handle()),
               "stress_surrogate")
    return stats


def stats_summary(stats) -> dict:
    """[candidates, fallbacks, audited, largest audited relative stress error,
    sum of audited relative errors, audited within 1e-3, audited and accepted,
    largest audited relative stress error among the accepted] as a dict."""
    import struct
    s = [v & 0xFFFFFFFF for v in stats.detach().cpu().to(torch.int64).tolist()]
    f = lambda u: struct.unpack("<f", struct.pack("<I", u))[0]  # noqa: E731
    aud = s[2]
    return {"candidates": s[0], "fallbacks": s[1], "accepted": s[0] - s[1], "audited": aud,
            "audit_max_rel_err": f(s[3]), "audit_mean_rel_err": f(s[4]) / aud if aud else 0.0,
            "audit_within_1e-3": s[5], "audited_accepted": s[6], "accepted_audit_max_rel_err": f(s[7])}
