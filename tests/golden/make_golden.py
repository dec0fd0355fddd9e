"""Generates tests/golden/oracle_cases.npz from the C oracle.

These fixtures are regression vectors of this project's oracle (the
reference ships none, so they do not pin parity to the reference): inputs
are regenerated from the stored seeds, outputs are the FP64 conserved
interior after `steps` steps and the dt of every step.

    python tests/golden/make_golden.py
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "deep-green_b200" / "python"))

import pyoracle  # noqa: E402
from conftest import random_primitives  # noqa: E402
from deepgreen import setups  # noqa: E402

P, O, W = 0, 1, 2
CASES = [
    # name, shape, bcs, limiter, gravity, steps, seed
    ("periodic", (6, 5, 7), (P,) * 6, 0, 0, 5, 11),
    ("outflow", (6, 5, 7), (O,) * 6, 0, 0, 5, 12),
    ("wall", (6, 5, 7), (W,) * 6, 0, 0, 5, 13),
    ("mixed_a", (5, 7, 6), (W, W, P, P, O, O), 0, 0, 5, 14),
    ("mixed_b", (7, 6, 5), (O, W, W, O, P, P), 1, 0, 5, 15),
    ("minmod_periodic", (6, 5, 7), (P,) * 6, 1, 0, 5, 16),
    ("minmod_wall", (6, 5, 7), (W,) * 6, 1, 0, 5, 17),
    ("gravity_wall_z", (5, 5, 8), (P, P, P, P, W, W), 0, 1, 5, 18),
    ("tiny_n2", (2, 3, 2), (O, W, P, P, W, O), 1, 0, 4, 19),
]


def run_case(shape, bcs, limiter, gravity, steps, seed, gamma=1.4, cfl=0.4, ds=0.1):
    prim = random_primitives(shape, seed)
    o = pyoracle.Oracle(shape, ds, bcs, gamma=gamma, cfl=cfl, limiter=limiter, gravity=gravity,
                        threads=pyoracle.SERIAL)
    o.set_primitives(prim)
    dts = o.step(steps)
    cons = np.stack([c[2:-2, 2:-2, 2:-2] for c in o.conserved()])
    return prim, dts, cons


def main():
    out = {}
    for name, shape, bcs, lim, grav, steps, seed in CASES:
        _, dts, cons = run_case(shape, bcs, lim, grav, steps, seed)
        out[f"{name}/cons"] = cons
        out[f"{name}/dts"] = dts
    # KH workload on a small grid: 16^3, minmod, 20 steps
    prim, ds, bcs = setups.kelvin_helmholtz(16, seed=3)
    o = pyoracle.Oracle((16, 16, 16), ds, bcs, gamma=1.4, cfl=0.4, limiter=1, threads=pyoracle.SERIAL)
    o.set_primitives(prim)
    out["kh16/dts"] = o.step(20)
    out["kh16/cons"] = np.stack([c[2:-2, 2:-2, 2:-2] for c in o.conserved()])
    np.savez_compressed(Path(__file__).with_name("oracle_cases.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    main()
