"""The bounded-wait abort path of the step kernels, on the GPU.

Every wait of a step kernel for a staged plane is bounded; when it runs out
the kernel lets the copies it issued land, raises DG_STATUS_TIMEOUT and
returns, and the C ABI reports DG_ERR_TIMEOUT.  The reference has no such
path: its CUDA code abort()s on a failed CUDA call (src/cu/include/
matrix3d.hpp:65-68).  Here the wait is made to run out by the library's test
hook (a context created while DG_DEBUG_WAIT_BUDGET is set gives those waits
that many SM clocks; 0 = give up at the first unfinished one); nothing
faults, traps or hangs.  The tests check the error, the sticky status flag,
that the context refuses to step an invalid state, and that the device stays
usable: a context created afterwards computes the oracle's result.
"""
import numpy as np
import pytest

import pyoracle
from conftest import random_primitives, rel_l1
from deepgreen import capi

pytestmark = pytest.mark.gpu

SHAPE = (20, 14, 40)
DS = 0.05
BCS = (2, 2, 0, 0, 1, 1)


def _ctx(rounding, precision=capi.F32):
    return capi.Context(SHAPE, DS, BCS, gamma=1.4, cfl=0.4, limiter=capi.LIMITER_MINMOD, precision=precision,
                        rounding=rounding)


@pytest.mark.parametrize("precision, rounding", [(capi.F32, capi.ROUNDING_DEFAULT),
                                                 (capi.F32, capi.ROUNDING_REFERENCE),
                                                 (capi.F64, capi.ROUNDING_DEFAULT)])
def test_wait_that_runs_out_reports_timeout_and_the_device_stays_usable(monkeypatch, precision, rounding):
    prim = random_primitives(SHAPE, 77)
    monkeypatch.setenv("DG_DEBUG_WAIT_BUDGET", "0")
    bad = _ctx(rounding, precision)
    monkeypatch.delenv("DG_DEBUG_WAIT_BUDGET")
    bad.set_primitives([np.asarray(a, dtype=bad.dtype) for a in prim])   # set-up kernels do not wait
    with pytest.raises(capi.DgError) as err:
        bad.compute_step(2)
    assert err.value.code == capi.DG_ERR_TIMEOUT
    assert bad.status() & capi.STATUS_TIMEOUT
    # the state is invalid: the context refuses to step until a new one is set
    with pytest.raises(capi.DgError) as err2:
        bad.compute_step(1)
    assert err2.value.code == capi.DG_ERR_NO_STATE
    bad.close()

    # the device is still usable: a normal context matches the FP64 oracle
    good = _ctx(rounding, precision)
    good.set_primitives([np.asarray(a, dtype=good.dtype) for a in prim])
    dts = good.compute_step(3)
    cons = good.get_conserved()
    assert good.status() == 0
    good.close()
    o = pyoracle.Oracle(SHAPE, DS, BCS, gamma=1.4, cfl=0.4, limiter=1, threads=pyoracle.ALL_PARALLEL)
    o.set_primitives(prim)
    ref_dts = o.step(3)
    ref = o.conserved()
    o.close()
    tol = 1e-5 if precision == capi.F32 else 1e-12
    assert max(rel_l1(cons[f], ref[f]) for f in range(5)) <= tol
    np.testing.assert_allclose(dts, ref_dts, rtol=10 * tol)
