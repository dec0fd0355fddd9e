"""ctypes binding of the correction network (include/deepgreen_net.h).

Device tensors are passed as torch CUDA tensors (torch provides the device
memory); all arithmetic runs in libdeepgreen.so's kernels.  Layouts:
features BF16 [n][x][y][z][16], outputs and targets FP32
[n][x-8][y-8][z-8][16], channels last.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import capi

IO_CHANNELS = 16
HIDDEN = 32
LAYERS = 4


class NetInfo(ctypes.Structure):
    _fields_ = [
        ("inputs", ctypes.c_int32), ("outputs", ctypes.c_int32), ("device", ctypes.c_int32),
        ("pad", ctypes.c_int32), ("seed", ctypes.c_uint64), ("out_scale", ctypes.c_double),
    ]


def layer_shape(layer: int, inputs: int, outputs: int):
    cin = inputs if layer == 0 else HIDDEN
    cout = outputs if layer == LAYERS - 1 else HIDDEN
    return cout, cin


class Net:
    """Owner of one dg_net."""

    def __init__(self, inputs: int, outputs: int, seed: int = 0, out_scale: float = 0.1, device: int = 0):
        self.lib = capi.load()
        self.inputs, self.outputs = int(inputs), int(outputs)
        info = NetInfo(self.inputs, self.outputs, int(device), 0, int(seed), float(out_scale))
        h = ctypes.c_void_p()
        rc = self.lib.dg_net_create(ctypes.byref(info), ctypes.byref(h))
        if rc != capi.DG_OK:
            raise capi.DgError(rc, self.lib.dg_net_last_error(None).decode())
        self.h = h

    def _check(self, rc):
        if rc != capi.DG_OK:
            raise capi.DgError(rc, self.lib.dg_net_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.dg_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- parameters ------------------------------------------------------------
    def shape(self, layer):
        return layer_shape(layer, self.inputs, self.outputs)

    def set_layer(self, layer, w, b):
        co, ci = self.shape(layer)
        w = np.ascontiguousarray(w, dtype=np.float32).reshape(co, ci, 3, 3, 3)
        b = np.ascontiguousarray(b, dtype=np.float32).reshape(co)
        self._check(self.lib.dg_net_set_layer(self.h, layer, w.ctypes.data, b.ctypes.data))

    def get_layer(self, layer):
        co, ci = self.shape(layer)
        w = np.empty((co, ci, 3, 3, 3), np.float32)
        b = np.empty(co, np.float32)
        self._check(self.lib.dg_net_get_layer(self.h, layer, w.ctypes.data, b.ctypes.data))
        return w, b

    def get_grad(self, layer):
        co, ci = self.shape(layer)
        w = np.empty((co, ci, 3, 3, 3), np.float32)
        b = np.empty(co, np.float32)
        self._check(self.lib.dg_net_get_grad(self.h, layer, w.ctypes.data, b.ctypes.data))
        return w, b

    def params(self):
        return [self.get_layer(l) for l in range(LAYERS)]

    def set_params(self, params):
        for l, (w, b) in enumerate(params):
            self.set_layer(l, w, b)

    # -- compute ---------------------------------------------------------------
    @staticmethod
    def _dims(feat):
        import torch
        if feat.dtype != torch.bfloat16 or feat.dim() != 5 or feat.shape[-1] != IO_CHANNELS or not feat.is_contiguous():
            raise ValueError("features must be a contiguous BF16 tensor [n][x][y][z][16]")
        return tuple(int(s) for s in feat.shape[:4])

    def forward(self, feat, out=None):
        import torch
        n, x, y, z = self._dims(feat)
        if out is None:
            out = torch.empty((n, x - 8, y - 8, z - 8, IO_CHANNELS), dtype=torch.float32, device=feat.device)
        self._check(self.lib.dg_net_forward(self.h, feat.data_ptr(), n, x, y, z, out.data_ptr()))
        return out

    def forward_backward(self, feat, target):
        import torch
        n, x, y, z = self._dims(feat)
        if target.dtype != torch.float32 or tuple(target.shape) != (n, x - 8, y - 8, z - 8, IO_CHANNELS):
            raise ValueError("target must be FP32 [n][x-8][y-8][z-8][16]")
        loss = ctypes.c_double()
        self._check(self.lib.dg_net_forward_backward(self.h, feat.data_ptr(), target.data_ptr(), n, x, y, z,
                                                     ctypes.byref(loss)))
        return loss.value

    def forward_backward_flux(self, feat, target, balance=False):
        """Flux-form loss (dg_net_forward_backward_flux): cubic feat of
        extent x, target FP32 [n][x-9]^3[16]; `balance` weighs every batch
        entry by the inverse power of its target."""
        import torch
        n, x, y, z = self._dims(feat)
        if target.dtype != torch.float32 or tuple(target.shape) != (n, x - 9, y - 9, z - 9, IO_CHANNELS):
            raise ValueError("target must be FP32 [n][x-9][y-9][z-9][16]")
        loss = ctypes.c_double()
        self._check(self.lib.dg_net_forward_backward_flux(self.h, feat.data_ptr(), target.data_ptr(), n, x, y, z,
                                                          int(bool(balance)), ctypes.byref(loss)))
        return loss.value

    def adam_step(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self._check(self.lib.dg_net_adam_step(self.h, lr, beta1, beta2, eps))

    def synchronize(self):
        self._check(self.lib.dg_net_synchronize(self.h))

    def stream(self):
        return self.lib.dg_net_get_stream(self.h)

    def get_tensor(self, layer, which, shape):
        """Intermediate of the last forward_backward: which 0 activation, 1
        pre-activation, 3 pre-activation gradient (BF16, returned as float32),
        2 the output (FP32)."""
        count = int(np.prod(shape))
        if which == 2:
            out = np.empty(shape, np.float32)
            self._check(self.lib.dg_net_get_tensor(self.h, layer, which, out.ctypes.data, out.nbytes))
            return out
        raw = np.empty(count, np.uint16)
        self._check(self.lib.dg_net_get_tensor(self.h, layer, which, raw.ctypes.data, raw.nbytes))
        return (raw.astype(np.uint32) << 16).view(np.float32).reshape(shape)
