"""ctypes binding of libdeepgreen.so (include/deepgreen.h).

Loads the in-tree library built by ``make -C deep-green_b200``.  There is no
fallback: if the library or a CUDA device is missing, calls raise.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

PKG_ROOT = Path(__file__).resolve().parents[2]          # deep-green_b200/
LIB_PATH = PKG_ROOT / "lib" / "libdeepgreen.so"
HEADER_PATH = PKG_ROOT.parent / "include" / "deepgreen.h"
NET_HEADER_PATH = PKG_ROOT.parent / "include" / "deepgreen_net.h"

DG_OK = 0
DG_ERR_INVALID = -1
DG_ERR_CUDA = -2
DG_ERR_NO_STATE = -3
DG_ERR_TIMEOUT = -4
DG_ERR_NO_DEVICE = -5

PERIODIC, OUTFLOW, WALL = 0, 1, 2
CONDUCTING_WALL = 3   # DG_BC_CONDUCTING_WALL: a wall with the heat source of the reference's CUDA variant
LIMITER_NONE, LIMITER_MINMOD = 0, 1
F32, F64 = 0, 1
ROUNDING_DEFAULT, ROUNDING_REFERENCE, ROUNDING_FAST = 0, 1, 2
BATCH_REORIENT = 1  # dg_batch_create_ex flag
STATUS_NONFINITE = 0x1
STATUS_TIMEOUT = 0x2
SNAP_PRIMITIVES, SNAP_CONSERVED = 0x1, 0x2


class SimInfo(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("nghosts", ctypes.c_int32),
        ("ds", ctypes.c_double), ("gamma", ctypes.c_double), ("cfl", ctypes.c_double),
        ("g", ctypes.c_double),
        ("bcs", ctypes.c_int32 * 6),
        ("gravity", ctypes.c_int32), ("limiter", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("device", ctypes.c_int32),
        ("rounding", ctypes.c_int32),
    ]


class DgError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"deepgreen error {code}: {msg}")
        self.code = code


_lib = None

# (name, argtypes) of every entry point the header declares
_P = ctypes.c_void_p
_I = ctypes.c_int32
_PP5 = ctypes.c_void_p * 5
SIGNATURES = {
    "dg_abi_version": [],
    "dg_create": [ctypes.POINTER(SimInfo), ctypes.POINTER(ctypes.c_void_p)],
    "dg_destroy": [_P],
    "dg_set_primitives": [_P, _PP5],
    "dg_set_conserved": [_P, _PP5],
    "dg_compute_step": [_P, _I, ctypes.POINTER(ctypes.c_double)],
    "dg_get_conserved": [_P, _PP5],
    "dg_get_primitives": [_P, _PP5],
    "dg_conservation_sums": [_P, ctypes.POINTER(ctypes.c_double)],
    "dg_set_conserved_device": [_P, _PP5],
    "dg_get_conserved_device": [_P, _PP5],
    "dg_enqueue_steps": [_P, _I],
    "dg_get_dts": [_P, _I, ctypes.POINTER(ctypes.c_double)],
    "dg_synchronize": [_P],
    "dg_get_stream": [_P, ctypes.POINTER(ctypes.c_void_p)],
    "dg_step_launch_shape": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "dg_set_chunk": [_P, _I],
    "dg_status": [_P, ctypes.POINTER(ctypes.c_uint32)],
    "dg_last_error": [_P],
    "dg_compute_step_dt": [_P, ctypes.c_double],
    "dg_next_dt": [_P, ctypes.POINTER(ctypes.c_double)],
    "dg_compute_step_noalloc": [ctypes.POINTER(SimInfo), _P, _P, ctypes.POINTER(ctypes.c_double), _P],
    "dg_noalloc_status": [_I, ctypes.POINTER(ctypes.c_uint32)],
    "dg_snapshot_create": [_P, ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)],
    "dg_snapshot_destroy": [_P],
    "dg_snapshot_begin": [_P],
    "dg_snapshot_wait": [_P, ctypes.POINTER(ctypes.c_void_p)],
    "dg_snapshot_write": [_P, ctypes.c_char_p],
    "dg_snapshot_write_host": [ctypes.c_char_p, _I, ctypes.POINTER(_I), _I, ctypes.POINTER(ctypes.c_char_p),
                               ctypes.POINTER(ctypes.c_void_p), ctypes.c_uint64, ctypes.c_char_p],
    "dg_snapshot_last_error": [_P],
    "dg_batch_create": [_I, ctypes.POINTER(SimInfo), ctypes.POINTER(ctypes.c_void_p)],
    "dg_batch_create_ex": [_I, ctypes.POINTER(SimInfo), ctypes.c_uint32, ctypes.POINTER(ctypes.c_void_p)],
    "dg_batch_get_orientation": [_P, _I, ctypes.POINTER(_I)],
    "dg_batch_destroy": [_P],
    "dg_batch_set_primitives": [_P, _I, _PP5],
    "dg_batch_step": [_P, _I],
    "dg_batch_enqueue": [_P, _I],
    "dg_batch_get_dts": [_P, _I, _I, ctypes.POINTER(ctypes.c_double)],
    "dg_batch_get_conserved": [_P, _I, _PP5],
    "dg_batch_set_tiling": [_P, _I, _I],
    "dg_batch_get_tiling": [_P, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(_I)],
    "dg_batch_autotune": [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I), ctypes.POINTER(ctypes.c_double)],
    "dg_batch_get_stream": [_P, ctypes.POINTER(ctypes.c_void_p)],
    "dg_batch_last_error": [_P],
    # learned correction (deepgreen_net.h)
    "dg_net_create": [_P, ctypes.POINTER(ctypes.c_void_p)],
    "dg_net_destroy": [_P],
    "dg_net_set_layer": [_P, _I, _P, _P],
    "dg_net_get_layer": [_P, _I, _P, _P],
    "dg_net_get_grad": [_P, _I, _P, _P],
    "dg_net_forward": [_P, _P, _I, _I, _I, _I, _P],
    "dg_net_forward_backward": [_P, _P, _P, _I, _I, _I, _I, ctypes.POINTER(ctypes.c_double)],
    "dg_net_forward_backward_flux": [_P, _P, _P, _I, _I, _I, _I, _I, ctypes.POINTER(ctypes.c_double)],
    "dg_net_adam_step": [_P, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float],
    "dg_net_get_tensor": [_P, _I, _I, _P, ctypes.c_uint64],
    "dg_coarsen": [_P, _P],
    "dg_learned_features": [_P, _P, _P, _I, ctypes.c_double, ctypes.c_double, _I, _I, _I, _I, _P, _P],
    "dg_learned_targets": [_P, _P, _P, _I, ctypes.c_double, _I, _I, _I, _I, _P, _P],
    "dg_corrector_create": [_P, _P, _P, ctypes.POINTER(ctypes.c_void_p)],
    "dg_corrector_destroy": [_P],
    "dg_corrector_set_tolerance": [_P, ctypes.c_double],
    "dg_corrector_step": [_P, _I],
    "dg_corrector_stats": [_P, _P],
    "dg_corrector_last_error": [_P],
    "dg_net_synchronize": [_P],
    "dg_net_get_stream": [_P],
    "dg_net_last_error": [_P],
}

_RESTYPES = {
    "dg_last_error": ctypes.c_char_p,
    "dg_batch_last_error": ctypes.c_char_p,
    "dg_net_last_error": ctypes.c_char_p,
    "dg_corrector_last_error": ctypes.c_char_p,
    "dg_snapshot_last_error": ctypes.c_char_p,
    "dg_net_get_stream": ctypes.c_void_p,
}


def load(path: os.PathLike | None = None):
    """Load libdeepgreen.so once and declare every signature."""
    global _lib
    if _lib is not None:
        return _lib
    # DEEPGREEN_LIB names another build of the library (e.g. one compiled
    # with different tile sizes); the default is the in-tree build
    p = Path(path) if path else Path(os.environ.get("DEEPGREEN_LIB", LIB_PATH))
    if not p.exists():
        raise FileNotFoundError(f"{p} not built; run `make -C {PKG_ROOT}` (no CPU fallback exists)")
    lib = ctypes.CDLL(str(p))
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPES.get(name, ctypes.c_int32)
    _lib = lib
    return lib


def _ptrs(arrays):
    return _PP5(*[a.ctypes.data for a in arrays])


class Context:
    """Owner of one dg_ctx (one grid on one device)."""

    def __init__(self, shape, ds, bcs, gamma=5.0 / 3.0, cfl=0.2, g=-0.1, gravity=False,
                 limiter=LIMITER_NONE, precision=F32, device=0, rounding=ROUNDING_DEFAULT):
        self.lib = load()
        self.shape = tuple(int(s) for s in shape)
        self.n = tuple(s + 4 for s in self.shape)
        self.dtype = np.float64 if precision == F64 else np.float32
        info = SimInfo()
        info.nx, info.ny, info.nz = self.shape
        info.nghosts = 2
        info.ds, info.gamma, info.cfl, info.g = float(ds), float(gamma), float(cfl), float(g)
        for i, b in enumerate(bcs):
            info.bcs[i] = int(b)
        info.gravity = int(bool(gravity))
        info.limiter = int(limiter)
        info.precision = int(precision)
        info.device = int(device)
        info.rounding = int(rounding)
        self.info = info
        h = ctypes.c_void_p()
        rc = self.lib.dg_create(ctypes.byref(info), ctypes.byref(h))
        if rc != DG_OK:
            raise DgError(rc, self.lib.dg_last_error(None).decode())
        self.h = h

    # -- helpers -------------------------------------------------------------
    def _check(self, rc):
        if rc != DG_OK:
            raise DgError(rc, self.lib.dg_last_error(self.h).decode())

    def _fields(self, fields):
        out = []
        for a in fields:
            a = np.ascontiguousarray(a, dtype=self.dtype)
            if a.shape != self.n:
                raise ValueError(f"field shape {a.shape} != {self.n}")
            out.append(a)
        return out

    def close(self):
        if getattr(self, "h", None):
            self.lib.dg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- state ---------------------------------------------------------------
    def set_primitives(self, prim):
        prim = self._fields(prim)
        self._check(self.lib.dg_set_primitives(self.h, _ptrs(prim)))

    def set_conserved(self, cons):
        cons = self._fields(cons)
        self._check(self.lib.dg_set_conserved(self.h, _ptrs(cons)))

    def get_conserved(self):
        out = [np.empty(self.n, dtype=self.dtype) for _ in range(5)]
        self._check(self.lib.dg_get_conserved(self.h, _ptrs(out)))
        return out

    def get_primitives(self):
        out = [np.empty(self.n, dtype=self.dtype) for _ in range(5)]
        self._check(self.lib.dg_get_primitives(self.h, _ptrs(out)))
        return out

    def set_conserved_device(self, ptrs):
        self._check(self.lib.dg_set_conserved_device(self.h, _PP5(*ptrs)))

    def get_conserved_device(self, ptrs):
        self._check(self.lib.dg_get_conserved_device(self.h, _PP5(*ptrs)))

    # -- stepping ------------------------------------------------------------
    def compute_step(self, nsteps=1):
        dts = np.zeros(max(nsteps, 1), dtype=np.float64)
        self._check(self.lib.dg_compute_step(self.h, int(nsteps),
                                             dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return dts[:nsteps]

    def next_dt(self) -> float:
        """dt of the coming step (dg_next_dt)."""
        v = ctypes.c_double()
        self._check(self.lib.dg_next_dt(self.h, ctypes.byref(v)))
        return v.value

    def compute_step_dt(self, dt):
        """One step with the given dt (dg_compute_step_dt)."""
        self._check(self.lib.dg_compute_step_dt(self.h, float(dt)))

    def enqueue_steps(self, nsteps):
        self._check(self.lib.dg_enqueue_steps(self.h, int(nsteps)))

    def get_dts(self, nsteps):
        dts = np.zeros(max(nsteps, 1), dtype=np.float64)
        self._check(self.lib.dg_get_dts(self.h, int(nsteps), dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return dts[:nsteps]

    def synchronize(self):
        self._check(self.lib.dg_synchronize(self.h))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.dg_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0

    def launch_shape(self):
        b, t, c = _I(), _I(), _I()
        self._check(self.lib.dg_step_launch_shape(self.h, ctypes.byref(b), ctypes.byref(t), ctypes.byref(c)))
        return b.value, t.value, c.value

    def set_chunk(self, chunk):
        self._check(self.lib.dg_set_chunk(self.h, int(chunk)))

    def conservation_sums(self):
        out = np.zeros(5, dtype=np.float64)
        self._check(self.lib.dg_conservation_sums(self.h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def status(self) -> int:
        f = ctypes.c_uint32()
        self._check(self.lib.dg_status(self.h, ctypes.byref(f)))
        return f.value


class Batch:
    """Owner of one dg_batch: independent grids stepped by one launch per
    step.  ``specs`` is a list of dicts with keys shape, ds, bcs and
    optionally gamma, cfl, limiter, g, gravity.  ``reorient``: let the
    library store each grid with its axes in the order that pads its tiles
    least (DG_BATCH_REORIENT); inputs and outputs keep the caller's layout."""

    def __init__(self, specs, device=0, reorient=False):
        self.lib = load()
        self.n = len(specs)
        arr = (SimInfo * self.n)()
        self.shapes = []
        for i, sp in enumerate(specs):
            inf = arr[i]
            inf.nx, inf.ny, inf.nz = (int(x) for x in sp["shape"])
            inf.nghosts = 2
            inf.ds = float(sp["ds"])
            inf.gamma = float(sp.get("gamma", 1.4))
            inf.cfl = float(sp.get("cfl", 0.4))
            inf.g = float(sp.get("g", -0.1))
            for f, bc in enumerate(sp["bcs"]):
                inf.bcs[f] = int(bc)
            inf.gravity = int(bool(sp.get("gravity", False)))
            inf.limiter = int(sp.get("limiter", LIMITER_MINMOD))
            inf.precision = F32
            inf.device = int(device)
            inf.rounding = ROUNDING_DEFAULT
            self.shapes.append(tuple(int(x) + 4 for x in sp["shape"]))
        self.infos = arr
        h = ctypes.c_void_p()
        rc = self.lib.dg_batch_create_ex(self.n, arr, BATCH_REORIENT if reorient else 0, ctypes.byref(h))
        if rc != DG_OK:
            raise DgError(rc, self.lib.dg_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != DG_OK:
            raise DgError(rc, self.lib.dg_batch_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.dg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_primitives(self, i, prim):
        prim = [np.ascontiguousarray(a, dtype=np.float32) for a in prim]
        for a in prim:
            if a.shape != self.shapes[i]:
                raise ValueError(f"grid {i}: field shape {a.shape} != {self.shapes[i]}")
        self._check(self.lib.dg_batch_set_primitives(self.h, int(i), _ptrs(prim)))

    def step(self, nsteps=1):
        self._check(self.lib.dg_batch_step(self.h, int(nsteps)))

    def enqueue(self, nsteps):
        self._check(self.lib.dg_batch_enqueue(self.h, int(nsteps)))

    def get_dts(self, i, nsteps):
        dts = np.zeros(max(nsteps, 1), dtype=np.float64)
        self._check(self.lib.dg_batch_get_dts(self.h, int(i), int(nsteps),
                                              dts.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return dts[:nsteps]

    def get_conserved(self, i):
        out = [np.empty(self.shapes[i], dtype=np.float32) for _ in range(5)]
        self._check(self.lib.dg_batch_get_conserved(self.h, int(i), _ptrs(out)))
        return out

    def orientation(self, i):
        """Caller axes (0 x, 1 y, 2 z) of grid i's stored x, y, z."""
        axes = (_I * 3)()
        self._check(self.lib.dg_batch_get_orientation(self.h, int(i), axes))
        return tuple(axes)

    def set_tiling(self, tile_rows, chunk=0):
        self._check(self.lib.dg_batch_set_tiling(self.h, int(tile_rows), int(chunk)))

    def tiling(self):
        r, c, n = _I(), _I(), _I()
        self._check(self.lib.dg_batch_get_tiling(self.h, ctypes.byref(r), ctypes.byref(c), ctypes.byref(n)))
        return r.value, c.value, n.value

    def autotune(self, steps=3):
        r, c, ms = _I(), _I(), ctypes.c_double()
        self._check(self.lib.dg_batch_autotune(self.h, int(steps), ctypes.byref(r), ctypes.byref(c), ctypes.byref(ms)))
        return r.value, c.value, ms.value

    def stream(self) -> int:
        s = ctypes.c_void_p()
        self._check(self.lib.dg_batch_get_stream(self.h, ctypes.byref(s)))
        return s.value or 0
