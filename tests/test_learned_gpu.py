"""The learned coarse step's building blocks on the GPU: exact coarsening,
the fixed-dt step, network inputs / targets against NumPy, and the
corrector's contract (zero correction = plain step bit for bit, positivity
mask, conservation to 1e-10 of each field's L1 norm, whole-step fallback)."""
import numpy as np
import pytest

from conftest import random_primitives
from deepgreen import learned
from deepgreen import net as dnet

pytestmark = pytest.mark.gpu


def _interior(a):
    return np.asarray(a)[2:-2, 2:-2, 2:-2]


def _grid(n, seed):
    g = learned.grid(n)
    g.set_primitives(random_primitives((n,) * 3, seed))
    return g


def test_coarsen_is_the_sum_of_eight_fine_cells():
    fine = _grid(16, 1)
    coarse = learned.grid(8)
    learned.coarsen(fine, coarse)
    f = [_interior(a) for a in fine.get_conserved()]
    c = [_interior(a) for a in coarse.get_conserved()]
    for ff, cc in zip(f, c):
        s = np.zeros((8, 8, 8), np.float32)
        for a in range(2):
            for b in range(2):     # the kernel's order: pairs along z, then (a, b)
                s = s + (ff[a::2, b::2, 0::2] + ff[a::2, b::2, 1::2])
        assert np.array_equal(cc, s)


def test_fixed_dt_step_equals_the_cfl_step():
    a, b = _grid(12, 2), _grid(12, 2)
    dt = float(a.compute_step(1)[0])
    assert b.next_dt() == dt
    b.compute_step_dt(dt)
    for x, y in zip(a.get_conserved(), b.get_conserved()):
        assert np.array_equal(x, y)
    assert float(b.get_dts(1)[0]) == dt


def _packs(n, seed):
    import torch
    g = _grid(n, seed)
    pool = learned.PackPool(n, 3)
    pool.store(g, 0)
    g.compute_step(1)
    pool.store(g, 1)
    g.compute_step(1)
    pool.store(g, 2)
    torch.cuda.synchronize()
    host = pool.data.cpu().numpy().reshape(3, 5, n + 4, n + 4, n + 4)
    return pool, host


def test_features_and_targets_match_numpy():
    import torch
    n = 12
    pool, host = _packs(n, 3)
    norm = learned.Norm.identity()
    rng = np.random.default_rng(0)
    for c in range(14):
        norm.in_mean[c] = float(rng.uniform(-1, 1))
        norm.in_inv_std[c] = float(rng.uniform(0.5, 2))
    for c in range(5):
        norm.out_std[c] = float(rng.uniform(0.5, 2))
    ext, origin = 9, (-4, 7, 10)
    feat = torch.zeros((ext, ext, ext, 16), dtype=torch.bfloat16, device="cuda")
    learned.features(norm, pool.ptr(0), pool.ptr(1), n, origin, ext, feat.data_ptr())
    tgt = torch.zeros((ext, ext, ext, 16), dtype=torch.float32, device="cuda")
    learned.targets(norm, pool.ptr(1), pool.ptr(2), n, origin, ext, tgt.data_ptr())
    torch.cuda.synchronize()

    vol = (1.0 / n) ** 3
    idx = [(np.arange(ext) + o) % n + 2 for o in origin]
    sel = np.ix_(*idx)
    u0 = np.stack([host[0, f][sel] for f in range(5)], -1).astype(np.float64) / vol
    u1 = np.stack([host[1, f][sel] for f in range(5)], -1).astype(np.float64) / vol
    tr = np.stack([host[2, f][sel] for f in range(5)], -1).astype(np.float64) / vol
    raw = np.zeros((ext, ext, ext, 16))
    raw[..., :5] = u1
    raw[..., 5:10] = u1 - u0
    raw[..., 10:13] = u1[..., 1:4] / u1[..., :1]
    raw[..., 13] = 0.4 * (u1[..., 4] - 0.5 * (u1[..., 1:4] ** 2).sum(-1) / u1[..., 0])
    mean = np.array(norm.in_mean)
    inv = np.array(norm.in_inv_std)
    inv[14:] = 0.0
    exp = (raw - mean) * inv
    got = feat.float().cpu().numpy()
    np.testing.assert_allclose(got, exp, rtol=1e-2, atol=2e-2 * np.abs(exp).max())
    et = np.zeros((ext, ext, ext, 16))
    et[..., :5] = (tr - u1) / np.array(norm.out_std)[:5]
    np.testing.assert_allclose(tgt.cpu().numpy(), et, rtol=1e-4, atol=1e-4 * np.abs(et).max())


def _net(out_scale, seed=5):
    return dnet.Net(learned.INPUTS, learned.OUTPUTS, seed=seed, out_scale=out_scale)


def _norm(out_std=1e-3):
    norm = learned.Norm.identity()
    for c in range(14, 16):
        norm.in_inv_std[c] = 0.0
    for c in range(5):
        norm.out_std[c] = out_std
    return norm


def test_zero_correction_is_the_plain_step_bit_for_bit():
    n = 16
    plain, corr = _grid(n, 4), _grid(n, 4)
    net = _net(0.0)
    cor = learned.Corrector(corr, net, _norm())
    dts = plain.compute_step(3)
    cor.step(3)
    for x, y in zip(plain.get_conserved(), corr.get_conserved()):
        assert np.array_equal(x, y)
    assert np.array_equal(corr.get_dts(3), dts)
    st = cor.stats()
    assert st["steps"] == 3 and st["fallback_steps"] == 0 and st["masked_cells"] == 0


def _flux_of_density_net(lam):
    """A network whose x-flux of mass is exactly lam * rho1 (input channel 0):
    hidden channel 0 carries rho1 + 10 through the GELUs' linear range."""
    net = _net(0.0)
    w0 = np.zeros((32, 14, 3, 3, 3), np.float32)
    w0[0, 0, 1, 1, 1] = 1.0
    b0 = np.zeros(32, np.float32)
    b0[0] = 10.0
    net.set_layer(0, w0, b0)
    for l in (1, 2):
        w = np.zeros((32, 32, 3, 3, 3), np.float32)
        w[0, 0, 1, 1, 1] = 1.0
        net.set_layer(l, w, np.zeros(32, np.float32))
    w3 = np.zeros((15, 32, 3, 3, 3), np.float32)
    w3[0, 0, 1, 1, 1] = lam
    b3 = np.zeros(15, np.float32)
    b3[0] = -10.0 * lam
    net.set_layer(3, w3, b3)
    return net


def test_cells_that_would_lose_positivity_keep_the_plain_value():
    # uniform gas with one low-density cell: the plain step's dissipation turns it
    # into a bump (rho1 ~ 1.18 against 0.82 around it); the correction
    # d(rho) = -4 (rho1(i) - rho1(i - e_x)) drives that cell negative (masked)
    # and raises its +x neighbour
    n = 16
    shape = (n + 4,) * 3
    prim = [np.ones(shape), np.zeros(shape), np.zeros(shape), np.zeros(shape), np.ones(shape)]
    prim[0][10, 10, 10] = 0.1
    plain, corr = learned.grid(n), learned.grid(n)
    plain.set_primitives(prim)
    corr.set_primitives(prim)
    # 16^3 is too small for the 1e-10 conservation bound (FP32 rounding alone
    # moves the totals by ~5e-10 here): this test is about the mask
    cor = learned.Corrector(corr, _flux_of_density_net(-4.0), _norm(1.0), tolerance=1e-6)
    plain.compute_step(1)
    cor.step(1)
    st = cor.stats()
    assert st["fallback_steps"] == 0 and st["masked_cells"] >= 1, st
    p = plain.get_conserved()
    c = corr.get_conserved()
    hole = (10, 10, 10)
    for f in range(5):
        assert p[f][hole] == c[f][hole]                      # masked: the plain value
    assert c[0][11, 10, 10] > p[0][11, 10, 10]               # the neighbour took the mass
    assert np.all(_interior(c[0]) > 0)


def test_correction_conserves_totals():
    # FP32 rounding of U + dU alone moves a field's total by ~3e-8 / sqrt(cells)
    # of its L1 norm; at 160^3 that is ~2e-11, inside the 1e-10 bound.
    n = 160
    plain, corr = _grid(n, 7), _grid(n, 7)
    net = _net(1.0)
    cor = learned.Corrector(corr, net, _norm(1e-3))
    plain.compute_step(1)
    cor.step(1)
    st = cor.stats()
    assert st["fallback_steps"] == 0 and st["steps"] == 1 and st["masked_cells"] == 0, st
    p = [_interior(a).astype(np.float64) for a in plain.get_conserved()]
    c = [_interior(a).astype(np.float64) for a in corr.get_conserved()]
    assert any(not np.array_equal(x, y) for x, y in zip(p, c))        # a real correction
    for x, y in zip(p, c):
        assert abs(y.sum() - x.sum()) <= 1e-10 * np.abs(x).sum()
    assert 0 < st["max_drift"] <= 1e-10
    cor.close()


def test_step_falls_back_when_the_totals_move():
    # tolerance 0: any rounding drift of the totals rejects the correction
    n = 16
    plain, strict = _grid(n, 7), _grid(n, 7)
    cor = learned.Corrector(strict, _net(1.0), _norm(1e-3), tolerance=0.0)
    plain.compute_step(1)
    cor.step(1)
    for x, y in zip(plain.get_conserved(), strict.get_conserved()):
        assert np.array_equal(x, y)
    st = cor.stats()
    assert st["fallback_steps"] == 1 and st["steps"] == 1
    cor.close()


def test_initial_states_on_the_gpu_match_numpy():
    from deepgreen import setups
    a, _, _ = setups.kelvin_helmholtz(20, seed=3, shear=0.6, ratio=1.5)
    b, _, _ = setups.kelvin_helmholtz(20, seed=3, shear=0.6, ratio=1.5, device="cuda")
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    a, _, _ = setups.fourier_modes(20, 4)
    b, _, _ = setups.fourier_modes(20, 4, device="cuda")
    assert all(np.allclose(x, y, rtol=0, atol=4 * np.finfo(np.float64).eps) for x, y in zip(a, b))
