"""The reference-shaped Python API (deepgreen.grid: Simulation,
SimulationGrid, calc_conserved, compute_step) on a stand-in context (no
GPU): sizes stored with the ghosts as Simulation::new does, the host
primitives handed over by calc_conserved, the order main.rs uses enforced,
and the dt of each step returned."""
import numpy as np
import pytest

from deepgreen import capi, grid as G


class FakeContext:
    """Records what the grid hands to the library; steps return fixed dts."""

    def __init__(self, interior, ds, bcs, **kw):
        self.interior, self.ds, self.bcs, self.kw = interior, ds, bcs, kw
        self.prim = None
        self.steps = 0

    def set_primitives(self, fields):
        self.prim = [np.array(f) for f in fields]

    def compute_step(self, n):
        self.steps += n
        return np.full(n, 0.25 / self.steps)

    def get_primitives(self):
        return [f + 1.0 for f in self.prim]

    def get_conserved(self):
        return [2.0 * f for f in self.prim]


@pytest.fixture()
def fake(monkeypatch):
    monkeypatch.setattr(capi, "Context", FakeContext)


def test_simulation_new_adds_ghosts_and_checks_periodic_pairs():
    sim = G.Simulation.new(8, 6, 4, 0.1, (G.BoundaryType.PERIODIC,) * 2 + (G.BoundaryType.OUTFLOW,) * 4,
                           periodicity=(True, False, False))
    assert (sim.nx, sim.ny, sim.nz) == (12, 10, 8) and sim.interior == (8, 6, 4)
    assert sim.gamma == pytest.approx(5.0 / 3.0) and sim.cfl == pytest.approx(0.2)   # globals.rs
    with pytest.raises(AssertionError):
        G.Simulation.new(8, 6, 4, 0.1, (G.BoundaryType.OUTFLOW,) * 6, periodicity=(True, False, False))


def test_grid_hands_host_primitives_to_the_library(fake):
    sim = G.Simulation.new(4, 3, 2, 0.5, (G.BoundaryType.WALL,) * 6, gamma=1.4, cfl=0.4, limiter=1)
    grid = G.SimulationGrid.new(sim)
    ctx = grid.context
    assert ctx.interior == (4, 3, 2) and ctx.ds == 0.5 and ctx.kw["gamma"] == 1.4 and ctx.kw["limiter"] == 1
    prim = grid.primitives
    assert prim.rho.shape == (8, 7, 6) and prim.rho.dtype == np.float32 and not prim.rho.any()
    with pytest.raises(RuntimeError):
        G.compute_step(sim, grid)          # main.rs runs calc_conserved first
    for k, f in enumerate(prim.fields()):
        f[...] = k + 1
    G.calc_conserved(grid)
    assert [float(f[0, 0, 0]) for f in ctx.prim] == [1, 2, 3, 4, 5]
    # after calc_conserved the arrays come from the device state
    assert float(grid.primitives.vx[1, 1, 1]) == 3.0 and float(grid.conserved.energy[0, 0, 0]) == 10.0
    assert G.compute_step(sim, grid) == 0.25 and G.compute_step(sim, grid) == 0.125
    assert ctx.steps == 2


def test_double_precision_grid_uses_float64_host_arrays(fake):
    sim = G.Simulation.new(2, 2, 2, 1.0, (G.BoundaryType.PERIODIC,) * 6, precision=capi.F64)
    assert G.SimulationGrid.new(sim).primitives.p.dtype == np.float64
