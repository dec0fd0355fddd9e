"""Parity at the benchmark's full size (512^3, FP32) through properties that
hold at any size, so that the FP64 oracle only has to run small cases.

Sod along x (the benchmark's workload, 100 steps): the state never varies
along y and z, so every (y, z) row of the 512^3 result is one 1-D solution,
which the oracle computes on a 512 x 4 x 4 grid with the same faces; every
row must match it within the FP32 tolerance.  Isentropic vortex (periodic,
the second 512^3 workload): the FP64 totals are conserved, the tube stays
invariant along z, and rolling the initial state by any number of cells
rolls the result bit for bit (each cell's arithmetic depends only on its
neighbourhood, not on where the tiling puts it)."""
import numpy as np
import pytest

import pyoracle
from deepgreen import capi, setups

pytestmark = pytest.mark.gpu

N = 512
I3 = (slice(2, -2),) * 3


def _broadcast(fields, shape):
    return [np.ascontiguousarray(np.broadcast_to(np.asarray(f, np.float32), shape)) for f in fields]


def test_sod_512_rows_match_the_oracle():
    shape = (N + 4,) * 3
    prim1, ds, bcs = setups.sod(N, ny=4, nz=4)                  # ghosted (516, 8, 8)
    ctx = capi.Context((N,) * 3, ds, bcs, gamma=1.4, cfl=0.4, limiter=capi.LIMITER_MINMOD, precision=capi.F32)
    ctx.set_primitives(_broadcast([f[:, :1, :1] for f in prim1], shape))
    del prim1
    dts = ctx.compute_step(100)
    cons = ctx.get_conserved()
    ctx.close()
    prim_o, _, _ = setups.sod(N, ny=4, nz=4)
    o = pyoracle.Oracle((N, 4, 4), ds, bcs, gamma=1.4, cfl=0.4, limiter=1, threads=pyoracle.ALL_PARALLEL)
    o.set_primitives(prim_o)
    ref_dts = o.step(100)
    ref = o.conserved()
    np.testing.assert_allclose(dts, ref_dts, rtol=1e-6)
    rows = [(0, 0), (0, N - 1), (15, 31), (16, 32), (N // 2, 300), (N - 1, N - 1)]
    for f in range(5):
        r = np.asarray(ref[f], np.float64)[2:-2, 3, 4]
        den = np.abs(r).sum()
        tol = 1e-5 * den if den > 0 else 1e-12
        for (y, z) in rows:
            g = np.asarray(cons[f][2:-2, y + 2, z + 2], np.float64)
            assert np.abs(g - r).sum() <= tol, (f, y, z, np.abs(g - r).sum() / max(den, 1e-300))
        # every row of the 512^3 result is the same row
        a = cons[f][I3]
        assert np.array_equal(a, np.broadcast_to(a[:, :1, :1], a.shape)), f


def test_vortex_512_conservation_and_roll_invariance():
    shape = (N + 4,) * 3
    prim1, ds, bcs = setups.isentropic_vortex(N, nz=4)           # (516, 516, 8): the tube is z-invariant
    prim = _broadcast([f[:, :, :1] for f in prim1], shape)
    del prim1
    kw = dict(gamma=1.4, cfl=0.4, limiter=capi.LIMITER_MINMOD, precision=capi.F32)
    ctx = capi.Context((N,) * 3, ds, bcs, **kw)
    ctx.set_primitives(prim)
    s0 = np.array(ctx.conservation_sums())
    dts = ctx.compute_step(10)
    s1 = np.array(ctx.conservation_sums())
    a = [c[I3].copy() for c in ctx.get_conserved()]
    ctx.close()
    scale = np.abs(s0).max()
    assert np.all(np.abs(s1 - s0) <= 1e-6 * scale), (s0, s1)
    for f in range(5):
        assert np.array_equal(a[f], np.broadcast_to(a[f][:, :, :1], a[f].shape)), f
    # the same state rolled by (7, 5, 3) interior cells
    shift = (7, 5, 3)
    rolled = []
    for f in prim:
        g = f.copy()
        g[I3] = np.roll(f[I3], shift, axis=(0, 1, 2))
        rolled.append(g)
    del prim
    ctx = capi.Context((N,) * 3, ds, bcs, **kw)
    ctx.set_primitives(rolled)
    del rolled
    dts_r = ctx.compute_step(10)
    b = ctx.get_conserved()
    ctx.close()
    np.testing.assert_array_equal(dts, dts_r)
    for f in range(5):
        assert np.array_equal(b[f][I3], np.roll(a[f], shift, axis=(0, 1, 2))), f
