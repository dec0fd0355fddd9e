"""ctypes wrapper of the C oracle (libdg_oracle.so).

TEST INFRASTRUCTURE ONLY: loaded by the tests, the smoke check and the
CPU-baseline leg of the benchmark, as the checker; never by the product.
Parity: pinned against the reference's own kernels (see dg_oracle.h).
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libdg_oracle.so"

PRIM, XTR, CONS, GRAD, FLUX = range(5)
SERIAL, RUST_LIKE, ALL_PARALLEL = 0, 1, 2


class Info(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("bcs", ctypes.c_int32 * 6), ("gravity", ctypes.c_int32), ("limiter", ctypes.c_int32),
                ("ds", ctypes.c_double), ("gamma", ctypes.c_double), ("cfl", ctypes.c_double),
                ("g", ctypes.c_double)]


_lib = None


def build():
    subprocess.run(["make", "-C", str(HERE), "-s"], check=True)


def load():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        lib = ctypes.CDLL(str(LIB))
        lib.dgo_create.argtypes = [ctypes.POINTER(Info), ctypes.c_int32]
        lib.dgo_create.restype = ctypes.c_void_p
        lib.dgo_destroy.argtypes = [ctypes.c_void_p]
        lib.dgo_set_threads.argtypes = [ctypes.c_void_p, ctypes.c_int32]
        lib.dgo_field.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32]
        lib.dgo_field.restype = ctypes.c_void_p
        for n in ("dgo_calc_conserved", "dgo_calc_primitives", "dgo_update_primitive_ghost_cells"):
            getattr(lib, n).argtypes = [ctypes.c_void_p]
        lib.dgo_calc_timestep.argtypes = [ctypes.c_void_p]
        lib.dgo_calc_timestep.restype = ctypes.c_double
        lib.dgo_compute_step.argtypes = [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
        lib.dgo_compute_step.restype = ctypes.c_int32
        lib.dgo_compute_step_given_dts.argtypes = [ctypes.c_void_p, ctypes.c_int32,
                                                   ctypes.POINTER(ctypes.c_double)]
        lib.dgo_compute_step_given_dts.restype = ctypes.c_int32
        _lib = lib
    return _lib


class Oracle:
    """One ghosted grid of the restated reference path (float or double)."""

    def __init__(self, shape, ds, bcs, gamma=5.0 / 3.0, cfl=0.2, limiter=0, gravity=False, g=-0.1,
                 dtype=np.float64, threads=RUST_LIKE):
        self.lib = load()
        info = Info()
        info.nx, info.ny, info.nz = (int(s) for s in shape)
        for i, b in enumerate(bcs):
            info.bcs[i] = int(b)
        info.gravity = int(bool(gravity))
        info.limiter = int(limiter)
        info.ds, info.gamma, info.cfl, info.g = float(ds), float(gamma), float(cfl), float(g)
        self.dtype = np.dtype(dtype)
        self.n = tuple(int(s) + 4 for s in shape)
        self.h = self.lib.dgo_create(ctypes.byref(info), 8 if self.dtype == np.float64 else 4)
        if not self.h:
            raise ValueError("oracle rejected the configuration")
        self.lib.dgo_set_threads(self.h, threads)

    def close(self):
        if self.h:
            self.lib.dgo_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def field(self, group, f):
        """Live NumPy view of an internal array."""
        ptr = self.lib.dgo_field(self.h, group, f)
        shape = self.n + ((3,) if group in (GRAD, FLUX) else ())
        ctype = ctypes.c_double if self.dtype == np.float64 else ctypes.c_float
        buf = (ctype * int(np.prod(shape))).from_address(ptr)
        return np.frombuffer(buf, dtype=self.dtype).reshape(shape)

    def set_primitives(self, prim):
        for f in range(5):
            self.field(PRIM, f)[...] = np.asarray(prim[f], dtype=self.dtype)
        self.lib.dgo_calc_conserved(self.h)
        self.lib.dgo_update_primitive_ghost_cells(self.h)

    def set_conserved(self, cons):
        for f in range(5):
            self.field(CONS, f)[...] = np.asarray(cons[f], dtype=self.dtype)

    def step(self, nsteps=1):
        dts = np.zeros(max(nsteps, 1), dtype=np.float64)
        self.lib.dgo_compute_step(self.h, int(nsteps), dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        return dts[:nsteps]

    def step_given_dts(self, dts):
        """Steps with the given dt per step in place of calc_timestep's."""
        d = np.ascontiguousarray(dts, dtype=np.float64)
        rc = self.lib.dgo_compute_step_given_dts(self.h, int(d.size), d.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        if rc != 0:
            raise ValueError("dgo_compute_step_given_dts failed")

    def conserved(self):
        return [self.field(CONS, f).copy() for f in range(5)]

    def primitives(self):
        return [self.field(PRIM, f).copy() for f in range(5)]
