"""The correction network's tensor-core kernels against the CPU oracle.

One forward + backward pass through dg_net_forward_backward (tcgen05 BF16
convolutions, FP32 accumulation) is compared, tensor by tensor, with
oracle/net_oracle.py (float64, BF16 rounding at the same points).  They can
differ only by FP32 accumulation error and the occasional BF16 rounding flip
it causes, so every tensor must agree to 5e-3 relative L2 and the loss to
1e-4 relative.  Shapes cover ragged extents, rows longer than one 128-position
tile and more than one batch entry.
"""
import numpy as np
import pytest

from deepgreen import net as dnet

pytestmark = pytest.mark.gpu

TOL = 5e-3


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def bf16_round(x):
    import torch
    return torch.as_tensor(x, dtype=torch.float32).to(torch.bfloat16).to(torch.float32).numpy()


def make_inputs(shape, inputs, outputs, seed):
    rng = np.random.default_rng(seed)
    n, x, y, z = shape
    feat = np.zeros((n, x, y, z, dnet.IO_CHANNELS), np.float32)
    feat[..., :inputs] = bf16_round(rng.standard_normal((n, x, y, z, inputs)))
    tgt = np.zeros((n, x - 8, y - 8, z - 8, dnet.IO_CHANNELS), np.float32)
    tgt[..., :outputs] = rng.standard_normal((n, x - 8, y - 8, z - 8, outputs)).astype(np.float32)
    return feat, tgt


@pytest.mark.parametrize("shape", [(2, 14, 14, 14), (1, 13, 11, 21), (1, 10, 12, 150), (2, 40, 11, 35)])
def test_forward_backward_matches_cpu_oracle(shape):
    import torch
    import net_oracle

    inputs, outputs = 14, 5
    net = dnet.Net(inputs, outputs, seed=11, out_scale=1.0)
    params = net.params()
    feat, tgt = make_inputs(shape, inputs, outputs, seed=5)
    dev = torch.device("cuda", 0)
    f = torch.from_numpy(feat).to(dev).to(torch.bfloat16).contiguous()
    t = torch.from_numpy(tgt).to(dev).contiguous()
    loss = net.forward_backward(f, t)
    ref = net_oracle.forward_backward(params, feat, tgt, inputs, outputs)

    n, x, y, z = shape
    for l in range(3):
        k = 2 * (l + 1)
        sh = (n, x - k, y - k, z - k, 32)
        assert rel_l2(net.get_tensor(l, 1, sh), ref["pre"][l]) < TOL, ("pre", l)
        assert rel_l2(net.get_tensor(l, 0, sh), ref["act"][l]) < TOL, ("act", l)
    out = net.get_tensor(3, 2, (n, x - 8, y - 8, z - 8, 16))
    assert rel_l2(out, ref["out"]) < TOL
    assert abs(loss - ref["loss"]) <= 1e-4 * abs(ref["loss"])
    for l in range(4):
        k = 2 * (l + 1)
        sh = (n, x - k, y - k, z - k, 32 if l < 3 else 16)
        assert rel_l2(net.get_tensor(l, 3, sh), ref["dz"][l]) < TOL, ("dz", l)
        gw, gb = net.get_grad(l)
        rw, rb = ref["grads"][l]
        assert rel_l2(gw, rw) < TOL, ("gw", l, rel_l2(gw, rw))
        assert rel_l2(gb, rb) < TOL, ("gb", l, rel_l2(gb, rb))


def test_inference_forward_equals_training_forward():
    import torch

    net = dnet.Net(14, 5, seed=3, out_scale=1.0)
    feat, tgt = make_inputs((2, 16, 12, 40), 14, 5, seed=9)
    dev = torch.device("cuda", 0)
    f = torch.from_numpy(feat).to(dev).to(torch.bfloat16).contiguous()
    out = net.forward(f)
    net.synchronize()
    net.forward_backward(f, torch.from_numpy(tgt).to(dev))
    ref = net.get_tensor(3, 2, tuple(out.shape))
    assert np.array_equal(out.cpu().numpy(), ref)


def test_adam_step_matches_reference_update():
    import torch

    net = dnet.Net(14, 5, seed=4, out_scale=1.0)
    feat, tgt = make_inputs((1, 12, 12, 12), 14, 5, seed=2)
    dev = torch.device("cuda", 0)
    f = torch.from_numpy(feat).to(dev).to(torch.bfloat16).contiguous()
    t = torch.from_numpy(tgt).to(dev)
    before = net.params()
    net.forward_backward(f, t)
    grads = [net.get_grad(l) for l in range(4)]
    lr, b1, b2, eps = 1e-3, 0.9, 0.999, 1e-8
    net.adam_step(lr, b1, b2, eps)
    after = net.params()
    for l in range(4):
        for p0, g, p1 in zip(before[l], grads[l], after[l]):
            m = (1 - b1) * g.astype(np.float64)
            v = (1 - b2) * g.astype(np.float64) ** 2
            exp = p0 - lr * (m / (1 - b1)) / (np.sqrt(v / (1 - b2)) + eps)
            np.testing.assert_allclose(p1, exp, rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("n,ext", [(2, 14), (1, 19)])
def test_flux_form_loss_and_gradients_match_cpu_oracle(n, ext):
    import torch
    import net_oracle

    inputs, outputs = 14, 15
    net = dnet.Net(inputs, outputs, seed=13, out_scale=1.0)
    params = net.params()
    rng = np.random.default_rng(8)
    feat = np.zeros((n, ext, ext, ext, 16), np.float32)
    feat[..., :inputs] = bf16_round(rng.standard_normal((n, ext, ext, ext, inputs)))
    s = ext - 9
    tgt = np.zeros((n, s, s, s, 16), np.float32)
    tgt[..., :5] = rng.standard_normal((n, s, s, s, 5)).astype(np.float32)
    dev = torch.device("cuda", 0)
    f = torch.from_numpy(feat).to(dev).to(torch.bfloat16).contiguous()
    loss = net.forward_backward_flux(f, torch.from_numpy(tgt).to(dev).contiguous())
    ref = net_oracle.forward_backward(params, feat, tgt, inputs, outputs, flux=True)
    assert abs(loss - ref["loss"]) <= 1e-4 * abs(ref["loss"])
    o = ext - 8
    assert rel_l2(net.get_tensor(3, 3, (n, o, o, o, 16)), ref["dz"][3]) < TOL
    for l in range(4):
        gw, gb = net.get_grad(l)
        rw, rb = ref["grads"][l]
        assert rel_l2(gw, rw) < TOL, ("gw", l, rel_l2(gw, rw))
        if l < 3:
            assert rel_l2(gb, rb) < TOL, ("gb", l, rel_l2(gb, rb))
        else:
            # the output bias gradient is the sum of the flux gradients, which
            # telescopes to boundary terms: compare against the summands' size
            scale = np.abs(ref["dz"][3]).reshape(-1, 16).sum(0)[:15]
            assert np.all(np.abs(gb - rb) <= TOL * scale), ("gb", l, np.abs(gb - rb) / scale)
