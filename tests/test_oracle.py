"""CPU tests of the oracle: two independent restatements of the reference
agree bit for bit, the golden fixtures reproduce, and physics invariants hold."""
import numpy as np
import pytest

import numpy_twin
import pyoracle
from conftest import INTERIOR, random_primitives
from deepgreen import setups

P, O, W = 0, 1, 2
BC_SETS = [(P,) * 6, (O,) * 6, (W,) * 6, (W, W, P, P, O, O), (P, P, W, W, O, O), (O, W, W, O, P, P)]


@pytest.mark.parametrize("bcs", BC_SETS)
@pytest.mark.parametrize("limiter", [0, 1])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_matches_numpy_twin_bitwise(bcs, limiter, dtype):
    shape = (6, 5, 7)
    prim = random_primitives(shape, 7)
    o = pyoracle.Oracle(shape, 0.1, bcs, gamma=1.4, cfl=0.4, limiter=limiter, dtype=dtype)
    o.set_primitives([a.astype(dtype) for a in prim])
    t = numpy_twin.TwinState(shape, 0.1, bcs, 1.4, 0.4, dtype=dtype, limiter=limiter)
    for f in range(5):
        t.prim[f][...] = prim[f].astype(dtype)
    t.calc_conserved()
    t._prim_ghosts(t.prim)
    for _ in range(3):
        assert o.step(1)[0] == t.compute_step()
    for f in range(5):
        np.testing.assert_array_equal(o.conserved()[f][INTERIOR], t.cons[f][INTERIOR])


def test_oracle_gravity_matches_twin():
    shape = (5, 5, 8)
    prim = random_primitives(shape, 8)
    bcs = (P, P, P, P, W, W)
    o = pyoracle.Oracle(shape, 0.1, bcs, gamma=1.4, cfl=0.4, gravity=True, g=-0.1)
    o.set_primitives(prim)
    t = numpy_twin.TwinState(shape, 0.1, bcs, 1.4, 0.4, gravity=True, g=-0.1)
    for f in range(5):
        t.prim[f][...] = prim[f]
    t.calc_conserved()
    t._prim_ghosts(t.prim)
    for _ in range(3):
        assert o.step(1)[0] == t.compute_step()
    for f in range(5):
        np.testing.assert_array_equal(o.conserved()[f][INTERIOR], t.cons[f][INTERIOR])


C = 3   # conducting wall (the reference's CUDA variant)


def hot_gas(shape, seed):
    """Air-like state (rho ~ 1.2, p ~ 4e5, so t_in ~ 1200 K against the
    wall's 273 K) with smooth noise: the conducting walls cool it at a rate
    that stays small per step."""
    prim = random_primitives(shape, seed)
    return [prim[0] * 1.2, prim[1] * 50.0, prim[2] * 50.0, prim[3] * 50.0, prim[4] * 4e5]


@pytest.mark.parametrize("bcs", [(C, W, P, P, O, O), (W, C, C, C, P, P), (C,) * 6, (O, C, P, P, C, W)])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_oracle_conducting_wall_matches_numpy_twin_bitwise(bcs, dtype):
    shape = (6, 5, 7)
    prim = hot_gas(shape, 17)
    o = pyoracle.Oracle(shape, 0.05, bcs, gamma=1.4, cfl=0.4, limiter=1, dtype=dtype)
    o.set_primitives([a.astype(dtype) for a in prim])
    t = numpy_twin.TwinState(shape, 0.05, bcs, 1.4, 0.4, dtype=dtype, limiter=1)
    for f in range(5):
        t.prim[f][...] = prim[f].astype(dtype)
    t.calc_conserved()
    t._prim_ghosts(t.prim)
    for _ in range(3):
        assert o.step(1)[0] == t.compute_step()
    for f in range(5):
        np.testing.assert_array_equal(o.conserved()[f][INTERIOR], t.cons[f][INTERIOR])


def _one_step(bcs, prim, shape):
    o = pyoracle.Oracle(shape, 0.05, bcs, gamma=1.4, cfl=0.4, limiter=1)
    o.set_primitives(prim)
    dt = o.step(1)[0]
    cons = o.conserved()
    o.close()
    return dt, cons


def test_conducting_wall_heat_reaches_only_the_first_cells_of_a_lower_face():
    """One step: a conducting lower x face changes only the energy of the
    first interior plane, by dt ds^2 Q/V (cooling of the hot gas); an upper
    conducting face adds its heat on a ghost face (kernels.h:616-627 tests
    i == NX-2), so the interior equals the plain wall's bit for bit."""
    shape = (6, 5, 7)
    prim = hot_gas(shape, 3)
    dt_w, wall = _one_step((W, W, P, P, O, O), prim, shape)
    dt_c, lo = _one_step((C, W, P, P, O, O), prim, shape)
    dt_u, up = _one_step((W, C, P, P, O, O), prim, shape)
    assert dt_w == dt_c == dt_u
    for f in range(5):
        np.testing.assert_array_equal(up[f][INTERIOR], wall[f][INTERIOR])
    for f in range(4):
        np.testing.assert_array_equal(lo[f][INTERIOR], wall[f][INTERIOR])
    d = (lo[4] - wall[4])[INTERIOR]
    assert np.all(d[1:] == 0)
    assert np.all(d[0] < 0)   # the wall (273 K) cools the gas
    # size: dt ds ds (Q / V), Q from the ghost cell's extrapolated state,
    # bounded by the first cell's cell-centred temperature within the step
    ds = 0.05
    t_in = prim[4][2:-2, 2:-2, 2:-2][0] / (287.0 * prim[0][2:-2, 2:-2, 2:-2][0])
    q = (273.0 - t_in) * (ds * ds / (0.008 / 0.2 + 0.1)) / ds ** 3
    np.testing.assert_allclose(d[0], dt_c * ds * ds * q, rtol=0.05)


def test_golden_fixtures_reproduce():
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).parent / "golden"))
    import make_golden
    gold = np.load(Path(__file__).parent / "golden" / "oracle_cases.npz")
    for name, shape, bcs, lim, grav, steps, seed in make_golden.CASES:
        _, dts, cons = make_golden.run_case(shape, bcs, lim, grav, steps, seed)
        np.testing.assert_array_equal(dts, gold[f"{name}/dts"], err_msg=name)
        np.testing.assert_array_equal(cons, gold[f"{name}/cons"], err_msg=name)


def test_uniform_state_is_steady():
    shape = (6, 6, 6)
    n = tuple(s + 4 for s in shape)
    prim = [np.full(n, 1.3), np.full(n, 0.2), np.full(n, -0.1), np.full(n, 0.05), np.full(n, 0.7)]
    for bcs in BC_SETS[:2]:
        o = pyoracle.Oracle(shape, 0.1, bcs, gamma=1.4, cfl=0.4, limiter=1)
        o.set_primitives(prim)
        c0 = o.conserved()
        o.step(5)
        for f in range(5):
            np.testing.assert_allclose(o.conserved()[f][INTERIOR], c0[f][INTERIOR], rtol=1e-14, atol=1e-16)


def test_periodic_conservation():
    prim, ds, bcs = setups.kelvin_helmholtz(16, seed=2)
    o = pyoracle.Oracle((16, 16, 16), ds, bcs, gamma=1.4, cfl=0.4, limiter=1)
    o.set_primitives(prim)
    s0 = [c[INTERIOR].sum() for c in o.conserved()]
    o.step(20)
    s1 = [c[INTERIOR].sum() for c in o.conserved()]
    for f in (0, 1, 4):
        assert abs(s1[f] - s0[f]) <= 1e-12 * abs(s0[f])
    for f in (2, 3):   # near-zero totals: compare against the momentum scale
        assert abs(s1[f] - s0[f]) <= 1e-12 * abs(s0[1]) + 1e-15


def test_axis_permutation_symmetry():
    """A problem rotated x->y->z gives the rotated result (unsplit scheme)."""
    shape = (6, 7, 5)
    prim = random_primitives(shape, 21)
    bcs = (P, P, O, O, W, W)
    o1 = pyoracle.Oracle(shape, 0.1, bcs, gamma=1.4, cfl=0.4, limiter=1)
    o1.set_primitives(prim)
    o1.step(3)
    # rotate axes (x, y, z) -> (y, z, x): new array index (j, k, i)
    perm = (1, 2, 0)
    shape2 = tuple(shape[p] for p in perm)
    bcs2 = tuple(v for p in perm for v in (bcs[2 * p], bcs[2 * p + 1]))
    prim2 = [np.transpose(prim[0], perm), np.transpose(prim[2], perm), np.transpose(prim[3], perm),
             np.transpose(prim[1], perm), np.transpose(prim[4], perm)]
    o2 = pyoracle.Oracle(shape2, 0.1, bcs2, gamma=1.4, cfl=0.4, limiter=1)
    o2.set_primitives(prim2)
    o2.step(3)
    c1 = o1.conserved()
    c2 = o2.conserved()
    back = [c2[0], c2[3], c2[1], c2[2], c2[4]]
    for f in range(5):
        np.testing.assert_allclose(np.transpose(back[f], (2, 0, 1))[INTERIOR], c1[f][INTERIOR],
                                   rtol=1e-10, atol=1e-14)


def test_nan_gives_cfl_fallback_dt():
    """calc_timestep: a NaN anywhere makes min() fail and dt = CFL * 1.0
    (physics.rs:191-195)."""
    shape = (4, 4, 4)
    prim = random_primitives(shape, 3)
    prim[4][3, 3, 3] = -1.0   # negative pressure -> sqrt(negative) = NaN
    o = pyoracle.Oracle(shape, 0.1, (P,) * 6, gamma=1.4, cfl=0.4)
    o.set_primitives(prim)
    assert o.step(1)[0] == pytest.approx(0.4)


def test_setups_device_path_matches_numpy():
    """The torch path of the KH generator (used on the GPU for the learned
    workload's large states) gives the NumPy path's bits; Fourier modes
    agree to an FP64 unit in the last place."""
    pytest.importorskip("torch")
    for n in (12, 21):
        a, _, _ = setups.kelvin_helmholtz(n, seed=7, shear=0.4, ratio=3.0)
        b, _, _ = setups.kelvin_helmholtz(n, seed=7, shear=0.4, ratio=3.0, device="cpu")
        assert all(np.array_equal(x, y) for x, y in zip(a, b))
        a, _, _ = setups.fourier_modes(n, 5)
        b, _, _ = setups.fourier_modes(n, 5, device="cpu")
        assert all(np.allclose(x, y, rtol=0, atol=4 * np.finfo(np.float64).eps) for x, y in zip(a, b))
