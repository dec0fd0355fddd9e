"""deep-green B200: host side of the CUDA Euler step (C ABI binding, the
reference-shaped grid/step API, workload set-ups)."""
from . import capi, setups  # noqa: F401
from .grid import BoundaryType, Simulation, SimulationGrid, calc_conserved, compute_step  # noqa: F401
