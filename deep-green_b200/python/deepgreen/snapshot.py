"""Snapshots: the state groups of the reference's save_to_disk
(src/rs/src/io.rs:5-196) captured from a context and written as a
self-describing binary file (HDF5 is not available to this library).

File layout (written by libdeepgreen.so, dg_snapshot_write): the 8 bytes
"DGSNAP01", a little-endian uint64 header length, a JSON header, then the
datasets, each starting on a 4096-byte boundary, raw C-order values of the
header's dtype and shape.  Groups and names follow io.rs: "primitives/rho",
"primitives/vx", "primitives/vy", "primitives/vz", "primitives/pressure",
"conserved/mass", "conserved/momentum_x", "conserved/momentum_y",
"conserved/momentum_z", "conserved/energy".  The "gradients" and "fluxes"
groups of io.rs are step intermediates the fused kernels never store.
"""
from __future__ import annotations

import ctypes
import json
import os
import struct

import numpy as np

from . import capi

MAGIC = b"DGSNAP01"
GROUPS = {"primitives": capi.SNAP_PRIMITIVES, "conserved": capi.SNAP_CONSERVED}


def read_header(path: os.PathLike) -> dict:
    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise ValueError(f"{path}: not a deep-green snapshot")
        raw = f.read(8)
        if len(raw) != 8:
            raise ValueError(f"{path}: truncated header")
        (hl,) = struct.unpack("<Q", raw)
        text = f.read(hl)
        if len(text) != hl:
            raise ValueError(f"{path}: truncated header")
        return json.loads(text.decode())


def read(path: os.PathLike, mmap: bool = True) -> dict:
    """{"meta": header, group: {name: ndarray}}; the arrays are read-only
    memory maps unless mmap is False."""
    h = read_header(path)
    dt = np.dtype(h["dtype"]).newbyteorder("<")
    shape = tuple(h["shape"])
    size = os.path.getsize(path)
    want = int(np.prod(shape)) * dt.itemsize
    out = {"meta": h}
    for d in h["datasets"]:
        if d["nbytes"] != want or d["offset"] + want > size:
            raise ValueError(f"{path}: dataset {d['name']} is truncated or does not match the header's shape")
        group, name = d["name"].split("/", 1)
        if mmap:
            a = np.memmap(path, dtype=dt, mode="r", offset=d["offset"], shape=shape)
        else:
            with open(path, "rb") as f:
                f.seek(d["offset"])
                a = np.frombuffer(f.read(d["nbytes"]), dtype=dt).reshape(shape)
        out.setdefault(group, {})[name] = a
    return out


def write_host(path: os.PathLike, arrays: dict, steps: int = 0, attrs: dict | None = None) -> None:
    """Write host arrays {"group/name": ndarray} (one 3-D shape, float32 or
    float64) with the library's writer (dg_snapshot_write_host)."""
    lib = capi.load()
    names = list(arrays)
    arrs = [np.ascontiguousarray(arrays[n]) for n in names]
    dt = arrs[0].dtype
    if any(a.dtype != dt or a.shape != arrs[0].shape for a in arrs) or arrs[0].ndim != 3:
        raise ValueError("arrays must share one 3-D shape and dtype")
    dtype = {np.dtype(np.float32): capi.F32, np.dtype(np.float64): capi.F64}[dt]
    shape = (ctypes.c_int32 * 3)(*arrs[0].shape)
    cnames = (ctypes.c_char_p * len(names))(*[n.encode() for n in names])
    data = (ctypes.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    rc = lib.dg_snapshot_write_host(os.fsencode(path), dtype, shape, len(names), cnames, data, int(steps),
                                    json.dumps(attrs).encode() if attrs is not None else None)
    if rc != capi.DG_OK:
        raise capi.DgError(rc, lib.dg_snapshot_last_error(None).decode())


class Snapshot:
    """dg_snapshot on a capi.Context: begin() captures the current state
    without stopping the context, write(path) waits for the copy and writes
    the file."""

    def __init__(self, ctx: capi.Context, groups=("primitives", "conserved")):
        self.lib = ctx.lib
        self.ctx = ctx
        bits = 0
        for g in groups:
            bits |= GROUPS[g]
        h = ctypes.c_void_p()
        self._check(self.lib.dg_snapshot_create(ctx.h, bits, ctypes.byref(h)))
        self.h = h

    def _check(self, rc):
        if rc != capi.DG_OK:
            raise capi.DgError(rc, self.lib.dg_snapshot_last_error(None).decode())

    def begin(self):
        self._check(self.lib.dg_snapshot_begin(self.h))

    def write(self, path: os.PathLike):
        self._check(self.lib.dg_snapshot_write(self.h, os.fsencode(path)))

    def wait(self) -> int:
        """Wait for the last capture; the pinned host buffer's address."""
        p = ctypes.c_void_p()
        self._check(self.lib.dg_snapshot_wait(self.h, ctypes.byref(p)))
        return p.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.dg_snapshot_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
