"""dg_compute_step_noalloc: one Euler step on device memory the caller owns.

Some callers must not let a library allocate GPU memory, for example a host
program whose device memory is owned by its own pool allocator sized at
start-up.  For them the library offers this entry point: the caller passes
the input and output states, and the step's scratch lives in a fixed array
inside the library.  These tests call it through the C ABI on buffers the
test owns and check it against the context entry point (dg_create +
dg_compute_step) on the same state, two calls in a row.  Both run the same
kernels on the same values (only the row pitch of the layout can differ),
so the outputs and dts must agree bit for bit; the parity tolerances used
elsewhere (1e-5 relative L1 for FP32, 1e-12 for FP64) are far looser.

The file is named to be collected last, so that a failure here does not
stop the rest of a `pytest -x` run.
"""
import ctypes

import numpy as np
import pytest

from conftest import INTERIOR, rel_l1, random_primitives
from deepgreen import capi

pytestmark = pytest.mark.gpu

TOL = {capi.F32: 1e-5, capi.F64: 1e-12}


def _noalloc(lib, info, src_ptr, dst_ptr):
    dt = ctypes.c_double(0.0)
    rc = lib.dg_compute_step_noalloc(ctypes.byref(info), ctypes.c_void_p(src_ptr), ctypes.c_void_p(dst_ptr),
                                     ctypes.byref(dt), None)
    assert rc == capi.DG_OK, lib.dg_last_error(None).decode()
    return dt.value


CASES = [
    # (precision, rounding, limiter): every kernel the entry point dispatches to
    (capi.F32, capi.ROUNDING_DEFAULT, capi.LIMITER_MINMOD),
    (capi.F32, capi.ROUNDING_DEFAULT, capi.LIMITER_NONE),
    (capi.F32, capi.ROUNDING_REFERENCE, capi.LIMITER_MINMOD),
    (capi.F64, capi.ROUNDING_DEFAULT, capi.LIMITER_MINMOD),
    (capi.F64, capi.ROUNDING_FAST, capi.LIMITER_MINMOD),
]
# (20, 18, 28): nz + 4 = 32, the same row pitch as a context; (13, 18, 40):
# ragged tiles along y and z and a row pitch (44) unlike the context's (64)
SHAPES = [(20, 18, 28), (13, 18, 40)]


@pytest.mark.parametrize("precision, rounding, limiter", CASES)
@pytest.mark.parametrize("bcs", [(0,) * 6, (2, 2, 1, 1, 0, 0)])
@pytest.mark.parametrize("shape", SHAPES)
def test_noalloc_matches_context_entry_point_two_calls(precision, rounding, limiter, bcs, shape):
    import torch

    ds = 0.05
    ctx = capi.Context(shape, ds, bcs, gamma=1.4, cfl=0.4, limiter=limiter, precision=precision, rounding=rounding)
    ctx.set_primitives(random_primitives(shape, 321))
    start = ctx.get_conserved()
    ref_dts, ref = [], []
    for _ in range(2):
        ref_dts.append(float(ctx.compute_step(1)[0]))
        ref.append(ctx.get_conserved())

    lib = capi.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    tdtype = torch.float64 if precision == capi.F64 else torch.float32
    a = torch.from_numpy(np.stack(start)).to(device=dev, dtype=tdtype).contiguous()
    b = torch.empty_like(a)
    c = torch.empty_like(a)
    dts = [_noalloc(lib, ctx.info, a.data_ptr(), b.data_ptr()),
           _noalloc(lib, ctx.info, b.data_ptr(), c.data_ptr())]
    outs = [b.cpu().numpy(), c.cpu().numpy()]
    flags = ctypes.c_uint32(99)
    assert lib.dg_noalloc_status(0, ctypes.byref(flags)) == capi.DG_OK
    assert flags.value == 0
    for call in range(2):
        for f in range(5):
            np.testing.assert_array_equal(outs[call][f][INTERIOR], ref[call][f][INTERIOR],
                                          err_msg=f"call {call} field {f}")
        assert dts[call] == ref_dts[call], (call, dts[call], ref_dts[call])
        errs = [rel_l1(outs[call][f], ref[call][f]) for f in range(5)]
        assert max(errs) <= TOL[precision], (call, errs)


def test_noalloc_without_dt_returns_at_once_and_reports_status():
    """dt_used NULL: no wait inside the call; after the caller synchronizes,
    dg_noalloc_status reads the step's flags; the current device is kept."""
    import torch

    shape = (16, 16, 28)
    ctx = capi.Context(shape, 0.05, (0,) * 6, gamma=1.4, cfl=0.4, limiter=capi.LIMITER_MINMOD, precision=capi.F32)
    ctx.set_primitives(random_primitives(shape, 9))
    start = ctx.get_conserved()
    ctx.compute_step(1)
    ref = ctx.get_conserved()
    lib = capi.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    a = torch.from_numpy(np.stack(start)).to(dev).contiguous()
    b = torch.empty_like(a)
    rc = lib.dg_compute_step_noalloc(ctypes.byref(ctx.info), ctypes.c_void_p(a.data_ptr()),
                                     ctypes.c_void_p(b.data_ptr()), None, None)
    assert rc == capi.DG_OK, lib.dg_last_error(None).decode()
    torch.cuda.synchronize()
    flags = ctypes.c_uint32(99)
    assert lib.dg_noalloc_status(0, ctypes.byref(flags)) == capi.DG_OK
    assert flags.value == 0
    assert torch.cuda.current_device() == 0
    out = b.cpu().numpy()
    for f in range(5):
        np.testing.assert_array_equal(out[f][INTERIOR], ref[f][INTERIOR])


def test_noalloc_rejects_grids_beyond_its_scratch():
    lib = capi.load()
    info = capi.SimInfo()
    info.nx, info.ny, info.nz = 4096, 4096, 4092   # far more blocks than the scratch holds
    info.nghosts = 2
    info.ds, info.gamma, info.cfl = 1e-3, 1.4, 0.4
    info.precision = capi.F32
    # rejected on size before any pointer is used
    rc = lib.dg_compute_step_noalloc(ctypes.byref(info), ctypes.c_void_p(256), ctypes.c_void_p(512), None, None)
    assert rc == capi.DG_ERR_INVALID
    assert b"scratch" in lib.dg_last_error(None)


def test_noalloc_status_rejects_a_bad_device():
    lib = capi.load()
    flags = ctypes.c_uint32(0)
    assert lib.dg_noalloc_status(-1, ctypes.byref(flags)) == capi.DG_ERR_NO_DEVICE
    assert lib.dg_noalloc_status(0, None) == capi.DG_ERR_INVALID


def test_noalloc_rejects_rows_that_break_tma_alignment():
    lib = capi.load()
    info = capi.SimInfo()
    info.nx, info.ny, info.nz = 8, 8, 9             # (9 + 4) * 4 bytes is not a multiple of 16
    info.nghosts = 2
    info.ds, info.gamma, info.cfl = 0.1, 1.4, 0.4
    info.precision = capi.F32
    rc = lib.dg_compute_step_noalloc(ctypes.byref(info), ctypes.c_void_p(256), ctypes.c_void_p(512), None, None)
    assert rc == capi.DG_ERR_INVALID
    assert b"16 bytes" in lib.dg_last_error(None)
