"""CPU checks of the network oracle (oracle/net_oracle.py) itself.

With BF16 rounding switched off, its hand-written backward pass must equal
torch autograd on the same float64 network; with rounding on, it must stay
close to the unrounded result (the rounding only perturbs at BF16 level)."""
import numpy as np
import torch

import net_oracle


def _problem(seed=0, shape=(2, 11, 10, 12), inputs=14, outputs=5):
    rng = np.random.default_rng(seed)
    params = []
    for l in range(4):
        co = outputs if l == 3 else 32
        ci = inputs if l == 0 else 32
        params.append(((rng.standard_normal((co, ci, 3, 3, 3)) * np.sqrt(2.0 / (27 * ci))).astype(np.float32),
                       (0.1 * rng.standard_normal(co)).astype(np.float32)))
    n, x, y, z = shape
    feat = np.zeros((n, x, y, z, 16), np.float32)
    feat[..., :inputs] = rng.standard_normal((n, x, y, z, inputs))
    tgt = np.zeros((n, x - 8, y - 8, z - 8, 16), np.float32)
    tgt[..., :outputs] = rng.standard_normal((n, x - 8, y - 8, z - 8, outputs))
    return params, feat, tgt, inputs, outputs


def test_unrounded_backward_equals_autograd():
    params, feat, tgt, inputs, outputs = _problem()
    ref = net_oracle.forward_backward(params, feat, tgt, inputs, outputs, round_bf16=False)
    ws = [torch.tensor(w, dtype=torch.float64, requires_grad=True) for w, _ in params]
    bs = [torch.tensor(b, dtype=torch.float64, requires_grad=True) for _, b in params]
    a = torch.tensor(feat[..., :inputs], dtype=torch.float64).permute(0, 4, 1, 2, 3)
    for l in range(3):
        a = net_oracle.gelu(torch.nn.functional.conv3d(a, ws[l], bs[l]))
    out = torch.nn.functional.conv3d(a, ws[3], bs[3])
    t = torch.tensor(tgt[..., :outputs], dtype=torch.float64).permute(0, 4, 1, 2, 3)
    loss = ((out - t) ** 2).mean()
    loss.backward()
    assert abs(float(loss) - ref["loss"]) < 1e-12 * float(loss)
    for l in range(4):
        np.testing.assert_allclose(ref["grads"][l][0], ws[l].grad.numpy(), rtol=1e-9, atol=1e-14)
        np.testing.assert_allclose(ref["grads"][l][1], bs[l].grad.numpy(), rtol=1e-9, atol=1e-14)


def test_bf16_rounding_is_a_small_perturbation():
    params, feat, tgt, inputs, outputs = _problem(seed=1)
    feat = torch.tensor(feat).to(torch.bfloat16).to(torch.float32).numpy()
    a = net_oracle.forward_backward(params, feat, tgt, inputs, outputs, round_bf16=True)
    b = net_oracle.forward_backward(params, feat, tgt, inputs, outputs, round_bf16=False)
    for l in range(4):
        gw, rw = a["grads"][l][0], b["grads"][l][0]
        assert np.linalg.norm(gw - rw) / np.linalg.norm(rw) < 3e-2


def test_flux_divergence_is_conservative_and_vanishes_for_uniform_fluxes():
    rng = np.random.default_rng(3)
    F = torch.tensor(rng.standard_normal((2, 16, 7, 7, 7)))
    div = net_oracle.flux_divergence(F)
    # direct restatement for one cell
    t = (1, 2, 3)
    for c in range(5):
        exp = sum(float(F[0, 5 * d + c, t[0] + 1, t[1] + 1, t[2] + 1])
                  - float(F[0, 5 * d + c, t[0] + 1 - (d == 0), t[1] + 1 - (d == 1), t[2] + 1 - (d == 2)])
                  for d in range(3))
        assert abs(float(div[0, c, t[0], t[1], t[2]]) - exp) < 1e-12
    # uniform fluxes: no correction
    U = torch.ones((1, 16, 5, 5, 5), dtype=torch.float64) * 3.7
    assert float(net_oracle.flux_divergence(U).abs().max()) == 0.0
    # periodic sum of a divergence telescopes to zero
    P = torch.tensor(rng.standard_normal((1, 16, 6, 6, 6)))
    Pw = torch.cat([P[:, :, -1:], P], 2)
    Pw = torch.cat([Pw[:, :, :, -1:], Pw], 3)
    Pw = torch.cat([Pw[:, :, :, :, -1:], Pw], 4)
    assert float(net_oracle.flux_divergence(Pw).sum(dim=(2, 3, 4)).abs().max()) < 1e-10


def test_flux_backward_equals_autograd_unrounded():
    params, feat, tgt, inputs, _ = _problem(seed=4, shape=(1, 12, 12, 12), outputs=15)
    tgt = tgt[:, :3, :3, :3]          # flux form: target one cell smaller than the output
    tgt = np.ascontiguousarray(tgt)
    ref = net_oracle.forward_backward(params, feat, tgt, inputs, 15, round_bf16=False, flux=True)
    ws = [torch.tensor(w, dtype=torch.float64, requires_grad=True) for w, _ in params]
    bs = [torch.tensor(b, dtype=torch.float64, requires_grad=True) for _, b in params]
    a = torch.tensor(feat[..., :inputs], dtype=torch.float64).permute(0, 4, 1, 2, 3)
    for l in range(3):
        a = net_oracle.gelu(torch.nn.functional.conv3d(a, ws[l], bs[l]))
    out = torch.nn.functional.conv3d(a, ws[3], bs[3])
    out16 = torch.cat([out, torch.zeros_like(out[:, :1])], 1)
    t = torch.tensor(tgt[..., :5], dtype=torch.float64).permute(0, 4, 1, 2, 3)
    loss = ((net_oracle.flux_divergence(out16) - t) ** 2).mean()
    loss.backward()
    assert abs(float(loss) - ref["loss"]) < 1e-12 * float(loss)
    for l in range(4):
        np.testing.assert_allclose(ref["grads"][l][0], ws[l].grad.numpy(), rtol=1e-9, atol=1e-14)
