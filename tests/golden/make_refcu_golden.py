"""Generates tests/golden/refcu_cases.npz from the reference's own kernels.

TEST INFRASTRUCTURE ONLY.  Builds `oracle/refcu` (deep-green's
src/cu/include/kernels.h compiled for the host against the reference's
configuration headers; needs the reference checkout, REF below), runs each
case of tests/refcu_cases.py on its seeded input (tests/golden/refcu_state.py)
and stores, per case: the configuration the program reports, every step's
dt, a fixed sample of cells of the conserved state after the last step (in
the case's precision) and per-field sums over the whole comparison region.

    python tests/golden/make_refcu_golden.py [REF]
"""
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "tests"))
sys.path.insert(0, str(ROOT / "tests" / "golden"))

import refcu_cases as rc  # noqa: E402
import refcu_state  # noqa: E402

BIN = ROOT / "oracle" / "_ref" / "refcu"


def build(ref: str) -> None:
    subprocess.run(["make", "-C", str(ROOT / "oracle" / "refcu"), "-s", f"REF={ref}"], check=True)


def info(cfg_name: str) -> dict:
    return json.loads(subprocess.check_output([str(BIN / f"refcu_{cfg_name}"), "info"]))


def run(cfg_name: str, prim, prec: int, steps: int):
    """Runs the reference kernels; returns (dts, conserved [5, NX, NY, NZ])."""
    dtype = np.float32 if prec == 4 else np.float64
    shape = prim[0].shape
    with tempfile.TemporaryDirectory() as d:
        fin, fout = os.path.join(d, "in.bin"), os.path.join(d, "out.bin")
        np.concatenate([np.asarray(a, dtype).ravel() for a in prim]).tofile(fin)
        subprocess.run([str(BIN / f"refcu_{cfg_name}"), "run", str(prec), str(steps), fin, fout],
                       check=True)
        raw = Path(fout).read_bytes()
    dts = np.frombuffer(raw[:8 * steps], np.float64).copy()
    cons = np.frombuffer(raw[8 * steps:], dtype).reshape((5,) + shape).copy()
    return dts, cons


def main(ref: str) -> None:
    build(ref)
    out = {}
    for name, (cfg_name, prec, steps, seed) in rc.CASES.items():
        cfg = rc.CONFIGS[cfg_name]
        got = info(cfg_name)
        for k, v in cfg.items():
            assert got[k] == v, (cfg_name, k, got[k], v)
        prim = refcu_state.primitives(rc.grid_shape(cfg), seed)
        dts, cons = run(cfg_name, prim, prec, steps)
        idx = rc.sample_index(cfg, seed)
        out[f"{name}.info"] = np.array(json.dumps(got))
        out[f"{name}.dts"] = dts
        out[f"{name}.idx"] = idx.astype(np.int64)
        out[f"{name}.cons"] = np.stack([c.ravel()[idx] for c in cons])
        out[f"{name}.sum"] = rc.region_sums(cons, cfg)
        print(name, "dts", dts)
    np.savez_compressed(rc.GOLDEN, **out)
    print("wrote", rc.GOLDEN, rc.GOLDEN.stat().st_size, "bytes")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
