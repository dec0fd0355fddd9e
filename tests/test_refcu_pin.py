"""The oracle against the reference's own kernels.

Golden vectors (tests/golden/refcu_cases.npz) come from deep-green's CUDA
solver kernels (src/cu/include/kernels.h) compiled for the host and run on
the reference's own configuration headers (KHI 128x6x128 periodic; Sod
5000x8x8 walls; TRB 128x128x256 walls with gravity); tests/refcu_cases.py
explains the set-up and the two places where the CUDA variant rounds or
bounds differently from the Rust path the oracle restates.

What must hold, per case, over the cells both variants compute alike:
* with the reference's dt given, the oracle's FP64 state is bit for bit the
  reference's when ds is a power of two (KHI over 5 steps, TRB with gravity),
  and within 2e-15 of each field's scale when it is not (Sod: the CUDA
  gradient multiplies by 1/(2 ds), kernels.h:169-171, the Rust one divides by
  2 ds, physics.rs:206-208); in FP32 after one step momenta and energy are
  bit for bit and the mass within one unit in the last place (kernels.h:677
  evaluates the mass dissipation in double); every FP32 field within 1e-6
  of its scale after several steps;
* the oracle's own dt is within one unit in the last place of the
  reference's (the Rust form CFL * (ds / x) against the CUDA form
  fl32(CFL * DELTA) / x, with cfl_eff making the two agree in exact
  arithmetic).
"""
import subprocess
from pathlib import Path

import numpy as np
import pytest

import pyoracle
import refcu_cases as rc

HERE = Path(__file__).resolve().parent
BIN = HERE.parent / "oracle" / "_ref" / "refcu"

GOLD = rc.load()


def _state(c):
    import sys
    sys.path.insert(0, str(HERE / "golden"))
    import refcu_state
    return refcu_state.primitives(rc.grid_shape(c["cfg"]), c["seed"])


def _oracle(c):
    cfg = c["cfg"]
    dtype = np.float32 if c["prec"] == 4 else np.float64
    o = pyoracle.Oracle(tuple(n - 4 for n in rc.grid_shape(cfg)), cfg["DELTA"], rc.bcs_dg(cfg),
                        gamma=cfg["GAMMA"], cfl=rc.cfl_eff(cfg), limiter=0, gravity=bool(cfg["GRAVITY"]),
                        g=cfg["G"], dtype=dtype, threads=pyoracle.ALL_PARALLEL)
    o.set_primitives([np.asarray(a, dtype) for a in _state(c)])
    return o


def _pow2(x: float) -> bool:
    m, _ = np.frexp(x)
    return m == 0.5


def test_golden_configurations_are_the_reference_headers():
    for name in rc.CASES:
        c = rc.case(GOLD, name)
        for k, v in c["cfg"].items():
            assert c["info"][k] == v, (name, k)
        assert c["cons"].shape == (5, c["idx"].size) and c["dts"].size == c["steps"]


@pytest.mark.parametrize("name", list(rc.CASES))
def test_oracle_matches_reference_kernels_given_their_dt(name):
    c = rc.case(GOLD, name)
    o = _oracle(c)
    o.step_given_dts(c["dts"])
    cons = o.conserved()
    got = np.stack([f.ravel()[c["idx"]] for f in cons])
    ref = c["cons"]
    exact_grid = _pow2(c["cfg"]["DELTA"])
    if c["prec"] == 8 and exact_grid:
        np.testing.assert_array_equal(got, ref, err_msg=name)
        np.testing.assert_array_equal(rc.region_sums(cons, c["cfg"]), c["sum"], err_msg=name)
        return
    scale = np.abs(ref.astype(np.float64)).max(axis=1)
    err = np.abs(got.astype(np.float64) - ref.astype(np.float64)).max(axis=1) / scale
    if c["prec"] == 8:
        assert err.max() <= 2e-15, (name, err)
        return
    if c["steps"] == 1 and exact_grid:
        np.testing.assert_array_equal(got[1:], ref[1:], err_msg=name)
        ulp = np.spacing(np.abs(ref[0]))
        assert np.all(np.abs(got[0] - ref[0]) <= ulp), name
    assert err.max() <= 1e-6, (name, err)


@pytest.mark.parametrize("name", [n for n, v in rc.CASES.items() if v[2] == 1])
def test_oracle_timestep_within_an_ulp_of_reference_kernels(name):
    c = rc.case(GOLD, name)
    o = _oracle(c)
    dt = o.step(1)[0]
    ref = c["dts"][0]
    eps = np.finfo(np.float32 if c["prec"] == 4 else np.float64).eps
    assert abs(dt - ref) <= eps * ref, (name, dt, ref)


@pytest.mark.skipif(not (BIN / "refcu_khi").exists(),
                    reason="reference kernels not built here (make -C oracle/refcu needs the reference checkout)")
def test_live_reference_kernels_khi_whole_grid():
    """A fresh input (seed 9), two steps, FP64: the oracle equals the
    reference kernels on every interior cell."""
    import sys
    import tempfile
    sys.path.insert(0, str(HERE / "golden"))
    import refcu_state
    cfg = rc.CONFIGS["khi"]
    prim = refcu_state.primitives(rc.grid_shape(cfg), 9)
    with tempfile.TemporaryDirectory() as d:
        fin, fout = Path(d) / "in.bin", Path(d) / "out.bin"
        np.concatenate([a.ravel() for a in prim]).tofile(fin)
        subprocess.run([str(BIN / "refcu_khi"), "run", "8", "2", str(fin), str(fout)], check=True, timeout=120)
        raw = fout.read_bytes()
    dts = np.frombuffer(raw[:16], np.float64)
    ref = np.frombuffer(raw[16:], np.float64).reshape((5,) + rc.grid_shape(cfg))
    o = pyoracle.Oracle(tuple(n - 4 for n in rc.grid_shape(cfg)), cfg["DELTA"], rc.bcs_dg(cfg),
                        gamma=cfg["GAMMA"], cfl=rc.cfl_eff(cfg), limiter=0, dtype=np.float64,
                        threads=pyoracle.ALL_PARALLEL)
    o.set_primitives(prim)
    o.step_given_dts(dts)
    reg = rc.region(cfg)
    for f, got in enumerate(o.conserved()):
        np.testing.assert_array_equal(got[reg], ref[f][reg], err_msg=f"field {f}")
