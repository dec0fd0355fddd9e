"""Snapshots on the GPU: the file holds exactly what dg_get_primitives and
dg_get_conserved return at the moment of dg_snapshot_begin, even when the
context keeps stepping before the file is written."""
import numpy as np
import pytest

from conftest import random_primitives
from deepgreen import capi, grid as dgrid, snapshot

pytestmark = pytest.mark.gpu

PRIM = ["rho", "vx", "vy", "vz", "pressure"]
CONS = ["mass", "momentum_x", "momentum_y", "momentum_z", "energy"]


@pytest.mark.parametrize("precision", [capi.F32, capi.F64])
def test_snapshot_is_the_state_at_begin(tmp_path, precision):
    shape = (20, 18, 16)
    bcs = [capi.PERIODIC, capi.PERIODIC, capi.OUTFLOW, capi.OUTFLOW, capi.WALL, capi.WALL]
    ctx = capi.Context(shape, 1.0 / 20, bcs, gamma=1.4, cfl=0.4, limiter=capi.LIMITER_MINMOD,
                       precision=precision)
    ctx.set_primitives(random_primitives(shape, 11))
    ctx.compute_step(3)
    prim, cons = ctx.get_primitives(), ctx.get_conserved()
    snap = snapshot.Snapshot(ctx)
    snap.begin()
    ctx.enqueue_steps(2)                      # the state moves on before the write
    path = tmp_path / "state.00001.dgsnap"
    snap.write(path)
    got = snapshot.read(path)
    assert got["meta"]["steps"] == 3
    assert got["meta"]["dtype"] == np.dtype(ctx.dtype).name
    assert got["meta"]["attrs"]["bcs"] == bcs and got["meta"]["attrs"]["ds"] == 1.0 / 20
    for name, a in zip(PRIM, prim):
        assert np.array_equal(got["primitives"][name], a), name
    for name, a in zip(CONS, cons):
        assert np.array_equal(got["conserved"][name], a), name
    after = ctx.get_conserved()
    assert not np.array_equal(after[0], cons[0])
    # a second capture with the same snapshot object
    snap.begin()
    snap.write(path)
    again = snapshot.read(path, mmap=False)
    assert again["meta"]["steps"] == 5
    assert np.array_equal(again["conserved"]["energy"], after[4])
    snap.close()
    ctx.close()


def test_conserved_only_snapshot(tmp_path):
    shape = (12, 12, 12)
    ctx = capi.Context(shape, 1.0 / 12, [capi.PERIODIC] * 6, gamma=1.4, cfl=0.4)
    ctx.set_primitives(random_primitives(shape, 5))
    snap = snapshot.Snapshot(ctx, groups=("conserved",))
    snap.begin()
    path = tmp_path / "c.dgsnap"
    snap.write(path)
    got = snapshot.read(path)
    assert set(got) == {"meta", "conserved"} and got["meta"]["steps"] == 0
    for name, a in zip(CONS, ctx.get_conserved()):
        assert np.array_equal(got["conserved"][name], a)
    snap.close()
    ctx.close()


def test_save_to_disk_mirrors_io_rs(tmp_path):
    info = dgrid.Simulation.new(12, 12, 12, 1.0 / 12, [capi.PERIODIC] * 6, periodicity=(True, True, True))
    g = dgrid.SimulationGrid.new(info)
    rng = np.random.default_rng(0)
    p = g.primitives
    p.rho[...] = 1.0 + 0.1 * rng.random(p.rho.shape)
    p.p[...] = 1.0
    dgrid.calc_conserved(g)
    dgrid.compute_step(info, g)
    fname = tmp_path / "state.00000.dgsnap"
    dgrid.save_to_disk(g, str(fname))
    got = snapshot.read(fname)
    assert set(got) == {"meta", "primitives", "conserved"}
    assert np.array_equal(got["conserved"]["mass"], g.conserved.mass)
    assert np.array_equal(got["primitives"]["rho"], g.primitives.rho)
