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
    info.bcs[0], info.bcs[1] = capi.PERIODIC, capi.CONDUCTING_WALL   # a conducting wall is no periodic face
    assert lib.dg_create(ctypes.byref(info), ctypes.byref(h)) == capi.DG_ERR_INVALID
    info.bcs[0], info.bcs[1] = 4, 4                                   # no such boundary type
    assert lib.dg_create(ctypes.byref(info), ctypes.byref(h)) == capi.DG_ERR_INVALID
    assert b"boundary" in lib.dg_last_error(None)
    assert not h.value


def _bad_info(**kw):
    info = capi.SimInfo()
    info.nx = info.ny = info.nz = 8
    info.nghosts = 2
    info.ds, info.gamma, info.cfl = 0.1, 1.4, 0.4
    for k, v in kw.items():
        setattr(info, k, v)
    return info


def test_creation_errors_are_per_thread():
    """dg_last_error(NULL) reports the calling thread's own failed create:
    two threads fail differently, and each reads its own message after both
    have failed."""
    import ctypes
    import threading
    lib = capi.load()
    barrier = threading.Barrier(2)
    seen = {}

    def worker(name, info):
        h = ctypes.c_void_p()
        rc = lib.dg_create(ctypes.byref(info), ctypes.byref(h))
        barrier.wait(timeout=30)
        seen[name] = (rc, lib.dg_last_error(None))

    infos = {"ghosts": _bad_info(nghosts=3), "constants": _bad_info(gamma=0.5)}
    threads = [threading.Thread(target=worker, args=item) for item in infos.items()]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=60)
    assert seen["ghosts"][0] == capi.DG_ERR_INVALID and b"nghosts" in seen["ghosts"][1]
    assert seen["constants"][0] == capi.DG_ERR_INVALID and b"gamma" in seen["constants"][1]


def test_batch_create_rejects_bad_grids_without_gpu_work():
    import ctypes
    lib = capi.load()
    h = ctypes.c_void_p()
    infos = (capi.SimInfo * 2)(_bad_info(), _bad_info(precision=capi.F64))
    assert lib.dg_batch_create(2, infos, ctypes.byref(h)) == capi.DG_ERR_INVALID
    assert b"FP32" in lib.dg_batch_last_error(None) and not h.value
    infos = (capi.SimInfo * 2)(_bad_info(), _bad_info(nx=1))
    assert lib.dg_batch_create(2, infos, ctypes.byref(h)) == capi.DG_ERR_INVALID
    assert b"grid 1" in lib.dg_batch_last_error(None)
    assert lib.dg_batch_create(0, infos, ctypes.byref(h)) == capi.DG_ERR_INVALID


def test_bench_traffic_figure_belongs_to_the_benchmarked_kernel():
    """The bench reports roofline.traffic only from a capture of the kernel
    it times; the committed summary must name that instantiation."""
    import json
    from pathlib import Path
    import bench
    d = json.loads((Path(__file__).resolve().parent.parent / "profiles" / "step_traffic.json").read_text())
    assert d["kernel"] == bench.STEP_KERNEL
    assert 40 <= d["interior_bytes_per_cell"] < 60 and 40 <= d["frame_bytes_per_cell"] < 70
    interior = 35 * 14 * 6 * 64 * 512          # 512^3: 35 x 6 interior tiles
    want = d["interior_bytes_per_cell"] * interior + d["frame_bytes_per_cell"] * (512 ** 3 - interior)
    assert bench.ncu_traffic_per_step(bench.STEP_KERNEL, 512) == want
    assert bench.step_launches(512) == 2 and bench.step_launches(128) == 1
    assert bench.ncu_traffic_per_step("another kernel", 512) is None


def test_resolution_norm_scales_only_the_output_scale():
    from deepgreen import learned
    from deepgreen.learned_workload import resolution_norm
    n = learned.Norm.identity()
    for c in range(16):
        n.in_mean[c], n.in_inv_std[c], n.out_std[c] = 0.1 * c, 1.0 + c, 2.0 + c
    r = resolution_norm(n, 128, 256)
    for c in range(16):
        assert r.in_mean[c] == n.in_mean[c] and r.in_inv_std[c] == n.in_inv_std[c]
        assert abs(r.out_std[c] - 0.25 * n.out_std[c]) <= 1e-6 * n.out_std[c]
    same = resolution_norm(n, 128, 128)
    assert all(same.out_std[c] == n.out_std[c] for c in range(16))

