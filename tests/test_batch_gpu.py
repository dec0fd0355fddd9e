"""Batched stepping (dg_batch): many independent grids, one persistent launch
per step, per-grid CFL dt, CUDA-graph replay, autotuned tiling.

Every cell of a batched grid is computed by the same kernel code as in a
single-grid run, so batch results must equal single-grid results bit for
bit, whatever the tiling; against the FP64 oracle the FP32 tolerance holds.
"""
import numpy as np
import pytest

import pyoracle
from conftest import INTERIOR, rel_l1
from deepgreen import batch, capi, setups

pytestmark = pytest.mark.gpu

P, O, W = 0, 1, 2
SHAPES = [(17, 9, 40), (8, 33, 12), (21, 20, 19), (5, 6, 70), (30, 14, 9)]
BCS = [(O,) * 6, (P,) * 6, (W, W, O, O, P, P), (O, W, P, P, W, O), (P, P, W, W, O, O)]


def _batch():
    specs, prims = [], []
    for i, (sh, b) in enumerate(zip(SHAPES, BCS)):
        prim, ds, _ = setups.riemann_random(sh, 500 + i, bcs=b)
        specs.append({"shape": sh, "ds": ds, "bcs": b, "limiter": 1})
        prims.append(prim)
    bt = capi.Batch(specs)
    for i, p in enumerate(prims):
        bt.set_primitives(i, p)
    return bt, specs, prims


def _single(spec, prim, steps):
    ctx = capi.Context(spec["shape"], spec["ds"], spec["bcs"], gamma=1.4, cfl=0.4, limiter=1, precision=capi.F32)
    ctx.set_primitives(prim)
    dts = ctx.compute_step(steps)
    return dts, ctx.get_conserved()


@pytest.mark.parametrize("chunk", [0, 24])
def test_batch_equals_single_grid_runs_bitwise(chunk):
    bt, specs, prims = _batch()
    rows, _, _ = bt.tiling()
    bt.set_tiling(rows, chunk)
    steps = 7                      # odd: graph replay plus a single launch
    bt.step(steps)
    for i, (sp, pr) in enumerate(zip(specs, prims)):
        dts, cons = _single(sp, pr, steps)
        np.testing.assert_array_equal(bt.get_dts(i, steps), dts, err_msg=f"grid {i}")
        got = bt.get_conserved(i)
        for f in range(5):
            np.testing.assert_array_equal(got[f][INTERIOR], cons[f][INTERIOR], err_msg=f"grid {i} field {f}")


def test_batch_conducting_walls_equal_single_grid_bitwise():
    """A conducting-wall grid (DG_BC_CONDUCTING_WALL, hot gas) beside a plain
    one in a batch: both equal their single-grid runs bit for bit."""
    from conftest import random_primitives
    C = capi.CONDUCTING_WALL
    specs, prims = [], []
    for sh, b, seed in (((13, 11, 45), (C, W, C, O, C, C), 41), ((9, 12, 20), (O,) * 6, 42)):
        pr = random_primitives(sh, seed)
        prims.append([pr[0] * 1.2, pr[1] * 50.0, pr[2] * 50.0, pr[3] * 50.0, pr[4] * 4e5])
        specs.append({"shape": sh, "ds": 0.05, "bcs": b, "limiter": 1})
    bt = capi.Batch(specs)
    for i, p in enumerate(prims):
        bt.set_primitives(i, p)
    steps = 5
    bt.step(steps)
    for i, (sp, pr) in enumerate(zip(specs, prims)):
        dts, cons = _single(sp, pr, steps)
        np.testing.assert_array_equal(bt.get_dts(i, steps), dts, err_msg=f"grid {i}")
        got = bt.get_conserved(i)
        for f in range(5):
            np.testing.assert_array_equal(got[f][INTERIOR], cons[f][INTERIOR], err_msg=f"grid {i} field {f}")


def test_batch_matches_fp64_oracle():
    bt, specs, prims = _batch()
    bt.step(5)
    for i, (sp, pr) in enumerate(zip(specs, prims)):
        o = pyoracle.Oracle(sp["shape"], sp["ds"], sp["bcs"], gamma=1.4, cfl=0.4, limiter=1,
                            threads=pyoracle.ALL_PARALLEL)
        o.set_primitives(pr)
        ref_dts = o.step(5)
        got = bt.get_conserved(i)
        errs = [rel_l1(got[f], o.conserved()[f]) for f in range(5)]
        assert max(errs) <= 1e-5, (i, errs)
        np.testing.assert_allclose(bt.get_dts(i, 5), ref_dts, rtol=1e-5)


def test_per_grid_dt_differs_between_grids():
    bt, _, _ = _batch()
    bt.step(2)
    first = [bt.get_dts(i, 2)[0] for i in range(len(SHAPES))]
    assert len(set(first)) == len(first)


def test_autotune_leaves_the_state_unchanged():
    bt, specs, prims = _batch()
    rows0, _, _ = bt.tiling()
    rows, chunk, ms = bt.autotune(2)
    assert rows == rows0 and chunk > 0 and ms > 0
    bt.step(3)
    for i, (sp, pr) in enumerate(zip(specs, prims)):
        dts, cons = _single(sp, pr, 3)
        np.testing.assert_array_equal(bt.get_dts(i, 3), dts)
        got = bt.get_conserved(i)
        for f in range(5):
            np.testing.assert_array_equal(got[f][INTERIOR], cons[f][INTERIOR])


def test_batch_workload_generator_is_seeded():
    a = batch.grid_shapes(64, seed=7)
    b = batch.grid_shapes(64, seed=7)
    assert a == b and len(a) == 64
    assert all(32 <= x <= 160 for sh in a for x in sh)


@pytest.mark.parametrize("trial", range(4))
def test_random_batches_equal_single_grid_runs_bitwise(trial):
    """Seeded random batches: 2-8 grids of 2-60 cells per axis, every
    boundary type, both limiters, gravity on some, a random x-chunk; each
    grid equals its single-grid run bit for bit."""
    from conftest import random_primitives
    C = capi.CONDUCTING_WALL
    rng = np.random.default_rng(40000 + trial)
    specs, prims = [], []
    for i in range(int(rng.integers(2, 9))):
        shape = tuple(int(v) for v in rng.integers(2, 60, 3))
        bcs = []
        for _ in range(3):
            bcs += [P, P] if rng.random() < 0.3 else [int(rng.choice([O, W, C])), int(rng.choice([O, W, C]))]
        spec = {"shape": shape, "ds": 0.05, "bcs": tuple(bcs), "limiter": int(rng.integers(0, 2)),
                "gravity": bool(rng.random() < 0.4)}
        pr = random_primitives(shape, 50000 + 10 * trial + i)
        if C in bcs:
            pr = [pr[0] * 1.2, pr[1] * 50.0, pr[2] * 50.0, pr[3] * 50.0, pr[4] * 4e5]
        specs.append(spec)
        prims.append(pr)
    steps, chunk = int(rng.integers(1, 7)), int(rng.choice([0, 8, 16, 64]))
    bt = capi.Batch(specs)
    for i, pr in enumerate(prims):
        bt.set_primitives(i, pr)
    rows, _, _ = bt.tiling()
    bt.set_tiling(rows, chunk)
    bt.step(steps)
    for i, (sp, pr) in enumerate(zip(specs, prims)):
        ctx = capi.Context(sp["shape"], 0.05, sp["bcs"], gamma=1.4, cfl=0.4, gravity=sp["gravity"],
                           limiter=sp["limiter"], precision=capi.F32)
        ctx.set_primitives(pr)
        dts = ctx.compute_step(steps)
        cons = ctx.get_conserved()
        np.testing.assert_array_equal(bt.get_dts(i, steps), dts, err_msg=f"grid {i}")
        got = bt.get_conserved(i)
        for f in range(5):
            np.testing.assert_array_equal(got[f][INTERIOR], cons[f][INTERIOR], err_msg=f"grid {i} field {f}")



# Shapes whose tiles pad less in another axis order (z widths just over 64,
# wide y, a short z), a conducting x face that is stored along z, and a
# gravity grid.
RE_SHAPES = [(40, 9, 70), (8, 33, 12), (70, 20, 30), (5, 6, 70), (30, 66, 9), (9, 33, 8)]
RE_BCS = [(O,) * 6, (P,) * 6, (W, W, O, O, P, P), (O, W, P, P, W, O), (3, W, O, O, W, O), (P, P, O, O, W, W)]


def _re_batch(reorient):
    specs, prims = [], []
    for i, (sh, b) in enumerate(zip(RE_SHAPES, RE_BCS)):
        prim, ds, _ = setups.riemann_random(sh, 700 + i, bcs=b)
        if 3 in b:
            # a hot gas for the conducting face (p / (287 rho) ~ 1200 K), same Mach numbers
            scale = 287.0 * 1200.0
            prim = [prim[0]] + [v * np.sqrt(scale) for v in prim[1:4]] + [prim[4] * scale]
        specs.append({"shape": sh, "ds": ds, "bcs": b, "limiter": 1, "gravity": i == 5, "g": -0.5})
        prims.append(prim)
    bt = capi.Batch(specs, reorient=reorient)
    for i, p in enumerate(prims):
        bt.set_primitives(i, p)
    return bt, specs, prims


def test_reoriented_batch_layout_round_trip_bitwise():
    """DG_BATCH_REORIENT stores grids with permuted axes, keeps z for the
    gravity grid, and hands back exactly what the caller-order batch holds
    after setting the same primitives (ghosts included)."""
    ref, _, _ = _re_batch(False)
    bt, specs, _ = _re_batch(True)
    axes = [bt.orientation(i) for i in range(len(specs))]
    assert sum(a != (0, 1, 2) for a in axes) >= 3, axes
    assert axes[5][2] == 2
    for i in range(len(specs)):
        got, want = bt.get_conserved(i), ref.get_conserved(i)
        for f in range(5):
            np.testing.assert_array_equal(got[f], want[f], err_msg=f"grid {i} axes {axes[i]} field {f}")


def test_reoriented_batch_steps_match_oracle():
    """Seven steps of the reoriented batch: per grid within the FP32
    tolerance (rel-L1 1e-5) of the FP64 oracle run in the caller's order,
    and within rounding of the caller-order batch (the permuted flux balance
    adds the axes in another order)."""
    ref, _, _ = _re_batch(False)
    bt, specs, prims = _re_batch(True)
    steps = 7
    ref.step(steps)
    bt.step(steps)
    for i, (sp, pr) in enumerate(zip(specs, prims)):
        o = pyoracle.Oracle(sp["shape"], sp["ds"], sp["bcs"], gamma=1.4, cfl=0.4, limiter=1,
                            gravity=sp["gravity"], g=sp["g"], threads=pyoracle.ALL_PARALLEL)
        o.set_primitives(pr)
        odts = o.step(steps)
        truth = o.conserved()
        got, same = bt.get_conserved(i), ref.get_conserved(i)
        errs = [rel_l1(got[f], truth[f]) for f in range(5)]
        assert max(errs) <= 1e-5, (i, bt.orientation(i), errs)
        np.testing.assert_allclose(bt.get_dts(i, steps), odts, rtol=1e-6, err_msg=f"grid {i}")
        diff = [rel_l1(got[f], same[f]) for f in range(5)]
        assert max(diff) <= 1e-5, (i, diff)
