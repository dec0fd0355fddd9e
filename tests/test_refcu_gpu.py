"""The CUDA step against the reference's own kernels (golden vectors).

The cases of tests/refcu_cases.py (deep-green's CUDA solver kernels run on
the host on its own configuration headers: KHI 128x6x128 periodic, Sod
5000x8x8 walls, TRB 128x128x256 walls with gravity) through the C ABI, each
kernel compared on the stored cells of the region both variants compute
alike:
* reference-rounding kernel, in the case's precision: dt within one unit in
  the last place of the reference's (the CUDA variant rounds CFL * DELTA to
  float; cfl_eff compensates in exact arithmetic), every field within
  1e-14 (FP64) / 1e-6 (FP32) of its scale;
* production kernels (fused arithmetic) against the FP64 golden: relative
  L1 per field <= 1e-12 (FP64 build) and <= 1e-5 (FP32).
"""
import sys
from pathlib import Path

import numpy as np
import pytest

import refcu_cases as rc
from deepgreen import capi

pytestmark = pytest.mark.gpu

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
import refcu_state  # noqa: E402

GOLD = rc.load()


def _run(c, precision, rounding):
    cfg = c["cfg"]
    ctx = capi.Context(tuple(n - 4 for n in rc.grid_shape(cfg)), cfg["DELTA"], rc.bcs_dg(cfg),
                       gamma=cfg["GAMMA"], cfl=rc.cfl_eff(cfg), g=cfg["G"], gravity=bool(cfg["GRAVITY"]),
                       limiter=capi.LIMITER_NONE, precision=precision, rounding=rounding)
    prim = refcu_state.primitives(rc.grid_shape(cfg), c["seed"])
    ctx.set_primitives([np.asarray(a, dtype=ctx.dtype) for a in prim])
    dts = ctx.compute_step(c["steps"])
    cons = ctx.get_conserved()
    return np.asarray(dts), np.stack([np.asarray(f).ravel()[c["idx"]] for f in cons])


@pytest.mark.parametrize("name", list(rc.CASES))
def test_reference_rounding_kernel_against_reference_kernels(name):
    c = rc.case(GOLD, name)
    precision = capi.F32 if c["prec"] == 4 else capi.F64
    dts, got = _run(c, precision, capi.ROUNDING_REFERENCE)
    eps = np.finfo(np.float32 if c["prec"] == 4 else np.float64).eps
    if c["steps"] == 1:
        assert abs(dts[0] - c["dts"][0]) <= eps * c["dts"][0], (name, dts, c["dts"])
    else:
        np.testing.assert_allclose(dts, c["dts"], rtol=1e-14 if c["prec"] == 8 else 1e-6, err_msg=name)
    ref = c["cons"].astype(np.float64)
    err = np.abs(got.astype(np.float64) - ref).max(axis=1) / np.abs(ref).max(axis=1)
    assert err.max() <= (1e-14 if c["prec"] == 8 else 1e-6), (name, err)


@pytest.mark.parametrize("name", [n for n, v in rc.CASES.items() if v[1] == 8])
@pytest.mark.parametrize("precision", [capi.F64, capi.F32])
def test_production_kernel_against_reference_kernels(name, precision):
    c = rc.case(GOLD, name)
    _, got = _run(c, precision, capi.ROUNDING_DEFAULT)
    ref = c["cons"]
    err = np.abs(got.astype(np.float64) - ref).sum(axis=1) / np.abs(ref).sum(axis=1)
    print(name, "FP64" if precision == capi.F64 else "FP32", "rel-L1 per field", err)
    assert err.max() <= (1e-12 if precision == capi.F64 else 1e-5), (name, err)
