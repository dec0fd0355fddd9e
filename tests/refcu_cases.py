"""Golden cases made by the reference's own CUDA kernels run on the host.

TEST INFRASTRUCTURE ONLY.  `oracle/refcu/` builds deep-green's
src/cu/include/kernels.h for the host, once per configuration header the
reference ships (its compile-time grid, boundaries and constants), and
`tests/golden/make_refcu_golden.py` runs those programs on the seeded states
of `tests/golden/refcu_state.py` and stores their outputs in
`tests/golden/refcu_cases.npz`.  This module holds what the tests need to
put the oracle and the CUDA kernels on the same footing:

* the configurations (grid with ghosts, ds, gamma, CFL, g, gravity,
  boundaries in the CUDA variant's face order x-, y-, z-, x+, y+, z+ and
  its enum PERIODIC, WALL, CONDUCTING_WALL, OUTFLOW; src/cu/include/
  constants.h:43-70, ini_files/sod.h, ini_files/trb.h), converted to this
  path's face order and enum;
* the CFL the reference's CUDA variant effectively uses: its timestep
  candidate is CFL * DELTA / (...) with CFL and DELTA float constants, so the
  product is rounded to float first (kernels.h:92-95), while the Rust path
  computes CFL * (ds / ...) (physics.rs:177-196).  cfl_eff = fl32(CFL * DELTA)
  / DELTA gives the Rust form the same step; it equals CFL when the product
  is exact (the KHI configuration, DELTA = 2^-7);
* the region where both variants compute the same thing: periodic axes are
  compared in full; on a wall axis the first interior layer is left out,
  because the CUDA variant applies no ghost rules to its gradients,
  predicted states or fluxes (physics.hpp:336-490 fills only primitive
  ghosts) while the Rust path does (boundaries.rs:5-407), so the two differ
  there by design;
* which differences the comparison allows: FP64 and the FP32 momenta and
  energy are bit for bit after one step; the FP32 mass may differ by one
  unit in the last place, because the CUDA mass flux scales its dissipation
  by a double literal (kernels.h:677, `0.5 * c_star`), which evaluates that
  line in double and rounds once.
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "refcu_cases.npz"

# CUDA-variant BC enum (constants.h:44) -> this path's (grid.rs:23-28 + 3).
CU_TO_DG = {0: 0, 1: 2, 2: 3, 3: 1}

# Each reference configuration header, as its `refcu_host info` prints it.
CONFIGS = {
    "khi": {"NX": 128, "NY": 6, "NZ": 128, "DELTA": 0.0078125, "GAMMA": 1.6666666269302368,
            "CFL": 0.20000000298023224, "G": 9.8100004196166992, "GRAVITY": 0, "bcs": [0] * 6},
    "sod": {"NX": 5000, "NY": 8, "NZ": 8, "DELTA": 0.00019999999494757503,
            "GAMMA": 1.6666666269302368, "CFL": 0.30000001192092896, "G": -9.8100004196166992,
            "GRAVITY": 0, "bcs": [1] * 6},
    "trb": {"NX": 128, "NY": 128, "NZ": 256, "DELTA": 1.0, "GAMMA": 1.6666666269302368,
            "CFL": 0.20000000298023224, "G": -9.8100004196166992, "GRAVITY": 1, "bcs": [1] * 6},
}

# name -> (configuration, precision in bytes, steps, seed)
CASES = {
    "khi_f64_1": ("khi", 8, 1, 1),
    "khi_f64_5": ("khi", 8, 5, 2),
    "khi_f32_1": ("khi", 4, 1, 1),
    "khi_f32_5": ("khi", 4, 5, 2),
    "sod_f64_1": ("sod", 8, 1, 3),
    "sod_f32_1": ("sod", 4, 1, 3),
    "trb_f64_1": ("trb", 8, 1, 4),
    "trb_f32_1": ("trb", 4, 1, 4),
}

SAMPLE = 2048  # stored cells per case (plus whole-region sums)


def grid_shape(cfg: dict) -> tuple[int, int, int]:
    """Cells including the two ghost layers per side (the CUDA variant's NX, NY, NZ)."""
    return (cfg["NX"], cfg["NY"], cfg["NZ"])


def bcs_dg(cfg: dict) -> list[int]:
    """Boundaries in this path's face order (x-, x+, y-, y+, z-, z+) and enum."""
    cu = cfg["bcs"]
    return [CU_TO_DG[cu[i]] for i in (0, 3, 1, 4, 2, 5)]


def cfl_eff(cfg: dict) -> float:
    return float(np.float32(cfg["CFL"]) * np.float32(cfg["DELTA"])) / cfg["DELTA"]


def region(cfg: dict) -> tuple[slice, slice, slice]:
    """Interior cells both variants compute alike (see the module docstring)."""
    cu = cfg["bcs"]
    out = []
    for axis, n in enumerate(grid_shape(cfg)):
        periodic = cu[axis] == 0 and cu[axis + 3] == 0
        m = 2 if periodic else 3
        out.append(slice(m, n - m))
    return tuple(out)


def sample_index(cfg: dict, seed: int) -> np.ndarray:
    """Flat indices (into the ghosted grid) of the stored cells: a fixed,
    sorted draw from the comparison region."""
    shape = grid_shape(cfg)
    reg = region(cfg)
    sub = np.arange(int(np.prod(shape))).reshape(shape)[reg].ravel()
    if sub.size <= SAMPLE:
        return sub
    step = sub.size / SAMPLE
    pick = (np.arange(SAMPLE) * step + (seed * 0.37 % 1.0) * step).astype(np.int64)
    return sub[np.minimum(pick, sub.size - 1)]


def load() -> dict:
    with np.load(GOLDEN, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


def case(golden: dict, name: str) -> dict:
    cfg_name, prec, steps, seed = CASES[name]
    return {
        "config": cfg_name, "cfg": CONFIGS[cfg_name], "prec": prec, "steps": steps, "seed": seed,
        "info": json.loads(str(golden[f"{name}.info"])),
        "dts": golden[f"{name}.dts"], "idx": golden[f"{name}.idx"],
        "cons": golden[f"{name}.cons"], "sum": golden[f"{name}.sum"],
    }


def region_sums(cons, cfg: dict) -> np.ndarray:
    """Per-field float64 sum over the comparison region (fixed order)."""
    reg = region(cfg)
    return np.array([np.asarray(c, dtype=np.float64)[reg].sum() for c in cons])
