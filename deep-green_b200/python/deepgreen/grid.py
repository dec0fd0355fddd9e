"""Host-side mirror of the reference's grid/state/step API over the C ABI.

Same names and argument meaning as deep-green's Rust path:
  BoundaryType            src/rs/src/grid.rs:23-28
  Simulation / new        src/rs/src/grid.rs:30-76
  SimulationGrid / new    src/rs/src/grid.rs:111-221
  calc_conserved          src/rs/src/physics.rs:143-175
  compute_step            src/rs/src/physics.rs:595-681
The difference is where the data lives: the state stays in GPU memory and
the host arrays are synchronised on demand (reading ``grid.conserved`` or
``grid.primitives`` copies the current device state back).
"""
from __future__ import annotations

from dataclasses import dataclass
from enum import IntEnum

import numpy as np

from . import capi


class BoundaryType(IntEnum):
    PERIODIC = capi.PERIODIC
    OUTFLOW = capi.OUTFLOW
    WALL = capi.WALL
    # the reference's CUDA variant only (src/cu/include/constants.h:44)
    CONDUCTING_WALL = capi.CONDUCTING_WALL


@dataclass
class Simulation:
    """grid.rs:30-76.  ``nx, ny, nz`` are stored WITH the ghosts added, as
    Simulation::new does; the constants the reference keeps as statics
    (globals.rs:3-8) are fields with the reference's values as defaults."""

    nx: int
    ny: int
    nz: int
    ds: float
    bcs: tuple
    nghosts: int = 2
    gravity: bool = False
    gamma: float = 5.0 / 3.0
    cfl: float = 0.2
    g: float = -0.1
    limiter: int = capi.LIMITER_NONE
    precision: int = capi.F32
    device: int = 0

    @classmethod
    def new(cls, nx, ny, nz, ds, bcs, periodicity=(False, False, False), nghosts=2, gravity=False, **kw):
        for axis, per in enumerate(periodicity):
            if per:
                assert bcs[2 * axis] == BoundaryType.PERIODIC and bcs[2 * axis + 1] == BoundaryType.PERIODIC
        return cls(nx + 2 * nghosts, ny + 2 * nghosts, nz + 2 * nghosts, ds, tuple(int(b) for b in bcs),
                   nghosts, gravity, **kw)

    @property
    def interior(self):
        g = self.nghosts
        return (self.nx - 2 * g, self.ny - 2 * g, self.nz - 2 * g)


@dataclass
class Primitives:
    rho: np.ndarray
    vx: np.ndarray
    vy: np.ndarray
    vz: np.ndarray
    p: np.ndarray

    def fields(self):
        return [self.rho, self.vx, self.vy, self.vz, self.p]


@dataclass
class Conserved:
    mass: np.ndarray
    momentum_x: np.ndarray
    momentum_y: np.ndarray
    momentum_z: np.ndarray
    energy: np.ndarray

    def fields(self):
        return [self.mass, self.momentum_x, self.momentum_y, self.momentum_z, self.energy]


class SimulationGrid:
    """grid.rs:111-221, with the state resident on the GPU.

    ``primitives`` starts as zeroed host arrays (as SimulationGrid::new
    allocates them) for the caller to fill before calc_conserved."""

    def __init__(self, info: Simulation):
        self.info = info
        shape = (info.nx, info.ny, info.nz)
        dt = np.float64 if info.precision == capi.F64 else np.float32
        self._host_prim = Primitives(*[np.zeros(shape, dtype=dt) for _ in range(5)])
        self._ctx = capi.Context(info.interior, info.ds, info.bcs, gamma=info.gamma, cfl=info.cfl, g=info.g,
                                 gravity=info.gravity, limiter=info.limiter, precision=info.precision,
                                 device=info.device)
        self._has_state = False

    @classmethod
    def new(cls, info: Simulation):
        return cls(info)

    @property
    def context(self) -> capi.Context:
        return self._ctx

    @property
    def primitives(self) -> Primitives:
        if not self._has_state:
            return self._host_prim
        return Primitives(*self._ctx.get_primitives())

    @property
    def conserved(self) -> Conserved:
        return Conserved(*self._ctx.get_conserved())


def calc_conserved(grid: SimulationGrid) -> None:
    """physics.rs:143-175: conserved state from the host primitives; from
    here on the state lives on the device."""
    grid._ctx.set_primitives(grid._host_prim.fields())
    grid._has_state = True


def compute_step(info: Simulation, grid: SimulationGrid) -> float:
    """physics.rs:595-681.  Returns the dt the step used (the reference
    writes it through its ``&mut f32`` argument)."""
    if not grid._has_state:
        raise RuntimeError("calc_conserved must run before compute_step (as in main.rs:50)")
    return float(grid._ctx.compute_step(1)[0])


def save_to_disk(grid: SimulationGrid, fname: str) -> None:
    """io.rs:5-196: the grid's primitive and conserved fields to fname, in
    the snapshot format of deepgreen.snapshot (HDF5 is not available; the
    gradient and flux intermediates are not stored by the fused step).  The
    capture and its copy to the host run on the device; the grid may step
    again as soon as this returns."""
    from . import snapshot
    if not grid._has_state:
        raise RuntimeError("calc_conserved must run before save_to_disk")
    snap = getattr(grid, "_snapshot", None)
    if snap is None:
        snap = grid._snapshot = snapshot.Snapshot(grid._ctx)
    snap.begin()
    snap.write(fname)
