"""CPU checks of the C ABI boundary: the library is built, loads, and
exports every entry point include/deepgreen.h and include/deepgreen_net.h
declare (no compute call)."""
import re
import subprocess

import pytest

from deepgreen import capi


def header_symbols():
    text = capi.HEADER_PATH.read_text() + capi.NET_HEADER_PATH.read_text()
    return sorted(set(re.findall(r"^\s*(?:int32_t|const char \*|void \*)\s*(dg_\w+)\s*\(", text, re.M)))


def test_header_declares_expected_entry_points():
    syms = header_symbols()
    for must in ("dg_create", "dg_destroy", "dg_set_primitives", "dg_set_conserved", "dg_compute_step",
                 "dg_get_conserved", "dg_get_primitives", "dg_conservation_sums", "dg_status", "dg_last_error"):
        assert must in syms


def test_library_exports_every_declared_symbol():
    if not capi.LIB_PATH.exists():
        pytest.fail(f"{capi.LIB_PATH} missing: build with `make -C deep-green_b200`")
    out = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True, text=True,
                         check=True).stdout
    exported = set(re.findall(r"\bT (dg_\w+)", out))
    missing = [s for s in header_symbols() if s not in exported]
    assert not missing, missing


def test_library_loads_and_binds_signatures():
    lib = capi.load()
    assert lib.dg_abi_version() == 1
    for name in header_symbols():
        assert name in capi.SIGNATURES, f"{name} not bound in capi.SIGNATURES"


def test_create_rejects_bad_configurations_without_gpu_work():
    lib = capi.load()
    import ctypes
    info = capi.SimInfo()
    info.nx = info.ny = info.nz = 8
    info.nghosts = 3          # the reference asserts ghosts == 2 (physics.rs:14)
    info.ds, info.gamma, info.cfl = 0.1, 1.4, 0.4
    h = ctypes.c_void_p()
    assert lib.dg_create(ctypes.byref(info), ctypes.byref(h)) == capi.DG_ERR_INVALID
    assert b"nghosts" in lib.dg_last_error(None)
    info.nghosts = 2
    info.bcs[0], info.bcs[1] = capi.PERIODIC, capi.OUTFLOW   # unpaired periodic face (grid.rs:55-63)
    assert lib.dg_create(ctypes.byref(info), ctypes.byref(h)) == capi.DG_ERR_INVALID
    assert not h.value
