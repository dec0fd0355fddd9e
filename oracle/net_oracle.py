"""CPU oracle of the correction network -- TEST INFRASTRUCTURE ONLY.

Nothing in the product imports this module; only tests/ use it, as the
checker of the CUDA network kernels (libdeepgreen.so, deepgreen_net.h).  The
reference solver has no learned component, so this oracle restates the
network the C ABI documents, not a reference file:

  4 "valid" 3x3x3 convolutions, channels 16 -> 32 -> 32 -> 32 -> 16 (real
  channels padded with zeros), GELU(x) = x/2 (1 + tanh(sqrt(2/pi)(x + 0.044715 x^3)))
  (the tanh form of Hendrycks & Gimpel) after the
  first three, a linear last layer; loss = mean over positions and the first
  `nout` output channels of (out - target)^2.

It computes in float64 (torch CPU) and rounds to BF16 exactly where the GPU
stores BF16: weights, activations, saved pre-activations, and the gradients
w.r.t. pre-activations.  Accumulation is exact-ish (float64) where the GPU
accumulates in FP32 on the tensor cores, so the two differ only by FP32
accumulation error and the rare BF16 rounding flip it causes.
"""
from __future__ import annotations

import math

import numpy as np
import torch
import torch.nn.functional as F

IO, HIDDEN = 16, 32
CIN = (IO, HIDDEN, HIDDEN, HIDDEN)
COUT = (HIDDEN, HIDDEN, HIDDEN, IO)


def bf16(t: torch.Tensor) -> torch.Tensor:
    """Round to the nearest BF16 value (ties to even), keep the dtype."""
    return t.to(torch.bfloat16).to(t.dtype)


def gelu(x):
    t = torch.tanh(math.sqrt(2.0 / math.pi) * (x + 0.044715 * x ** 3))
    return 0.5 * x * (1.0 + t)


def gelu_grad(x):
    c0 = math.sqrt(2.0 / math.pi)
    t = torch.tanh(c0 * (x + 0.044715 * x ** 3))
    return 0.5 * (1.0 + t) + 0.5 * x * (1.0 - t * t) * c0 * (1.0 + 3.0 * 0.044715 * x * x)


def pad_params(params, inputs, outputs):
    """[(w[co][ci][3][3][3], b[co])] over real channels -> full padded float64 tensors."""
    out = []
    for l, (w, b) in enumerate(params):
        wp = torch.zeros((COUT[l], CIN[l], 3, 3, 3), dtype=torch.float64)
        bp = torch.zeros(COUT[l], dtype=torch.float64)
        w = torch.as_tensor(np.asarray(w), dtype=torch.float64)
        b = torch.as_tensor(np.asarray(b), dtype=torch.float64)
        wp[: w.shape[0], : w.shape[1]] = w
        bp[: b.shape[0]] = b
        out.append((wp, bp))
    return out


def flux_divergence(F):
    """dU_c(t) = sum_d F[5d+c](t+1) - F[5d+c](t+1-e_d) over the target cells
    t, for F of shape (n, 16, s+1, s+1, s+1); returns (n, 5, s, s, s)."""
    hi = F[:, :, 1:, 1:, 1:]
    lo = [F[:, :, :-1, 1:, 1:], F[:, :, 1:, :-1, 1:], F[:, :, 1:, 1:, :-1]]
    return sum(hi[:, 5 * d:5 * d + 5] - lo[d][:, 5 * d:5 * d + 5] for d in range(3))


def forward_backward(params, feat, target, inputs, outputs, round_bf16=True, flux=False):
    """params: real-channel (w, b) per layer (FP32 master values); feat:
    (n, x, y, z, 16) array of BF16-representable values; target: (n, x-8,
    y-8, z-8, 16).  Returns dict with loss, out, act[l], pre[l], dz[l]
    (channels last, padded channel counts) and grads [(gw, gb)] over real
    channels.  round_bf16=False drops every BF16 rounding (plain float64
    arithmetic), which is what the oracle's own CPU test checks against
    autograd."""
    rnd = bf16 if round_bf16 else (lambda v: v)
    P = pad_params(params, inputs, outputs)
    W = [rnd(w) for w, _ in P]
    B = [b for _, b in P]
    x = torch.as_tensor(np.asarray(feat, dtype=np.float64)).permute(0, 4, 1, 2, 3).contiguous()
    t = torch.as_tensor(np.asarray(target, dtype=np.float64)).permute(0, 4, 1, 2, 3).contiguous()
    # flux form: target extent is one less than the output's
    acts, pres = [x], []
    a = x
    for l in range(3):
        z = F.conv3d(a, W[l]) + B[l].view(1, -1, 1, 1, 1)
        pres.append(rnd(z))
        a = rnd(gelu(z))
        acts.append(a)
    out = F.conv3d(a, W[3]) + B[3].view(1, -1, 1, 1, 1)
    if flux:
        # the divergence is linear: its adjoint comes from autograd, exactly
        o = out.detach().requires_grad_(True)
        d = flux_divergence(o) - t[:, :5]
        lsum = (d * d).sum()
        loss = float(lsum) / d.numel()
        (gr,) = torch.autograd.grad(lsum, o)
        g = (gr / d.numel()).detach()
        # the GPU stores the per-cell residual gradient in FP32 first
        if round_bf16:
            res = (2.0 * d.detach() / d.numel()).to(torch.float32).to(torch.float64)
            ores = torch.zeros_like(o)
            ores.requires_grad_(True)
            g = torch.autograd.grad((flux_divergence(ores) * res).sum(), ores)[0]
    else:
        d = out[:, :outputs] - t[:, :outputs]
        loss = float((d * d).mean())
        g = torch.zeros_like(out)
        g[:, :outputs] = 2.0 * d / d.numel()
    g[:, 15:] = 0.0
    dz = rnd(g.to(torch.float32).to(torch.float64)) if round_bf16 else g
    dzs = [None] * 4
    dzs[3] = dz
    grads = [None] * 4
    for l in range(3, -1, -1):
        gw = torch.nn.grad.conv3d_weight(acts[l], W[l].shape, dz)
        gb = dz.sum(dim=(0, 2, 3, 4))
        co = outputs if l == 3 else HIDDEN
        ci = inputs if l == 0 else HIDDEN
        grads[l] = (gw[:co, :ci].numpy(), gb[:co].numpy())
        if l == 0:
            break
        da = torch.nn.grad.conv3d_input(acts[l].shape, W[l], dz)
        dz = rnd(da * gelu_grad(pres[l - 1]))
        dzs[l - 1] = dz

    def cl(v):
        return v.permute(0, 2, 3, 4, 1).contiguous().numpy()

    return {
        "loss": loss,
        "out": cl(out),
        "act": [cl(v) for v in acts[1:]],
        "pre": [cl(v) for v in pres],
        "dz": [cl(v) for v in dzs],
        "grads": grads,
    }
