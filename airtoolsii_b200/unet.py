"""U-Net warm start (no counterpart in the reference; its output is used as
the x0 argument of sirt, sirt/sirt.m:5).

Thin host wrapper over libairt's airt_unet_* entry points.  Device buffers
are torch tensors (memory plumbing only); every kernel is libairt's.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check, lib


class UNet:
    """levels-level U-Net on H x W images, widths base*2^l."""

    def __init__(self, H, W, base=32, levels=4, max_batch=16, seed=0):
        self.H, self.W, self.base, self.levels, self.max_batch = H, W, base, levels, max_batch
        h = C.c_void_p()
        check(lib().airt_unet_create(H, W, base, levels, max_batch, seed, C.byref(h)))
        self._h = h
        n = C.c_int64()
        check(lib().airt_unet_num_params(h, C.byref(n)))
        self.num_params = int(n.value)

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                lib().airt_unet_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(lib().airt_unet_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        check(lib().airt_unet_get_params(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        assert p.size == self.num_params
        check(lib().airt_unet_set_params(self._h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def get_grads(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        check(lib().airt_unet_get_grads(self._h, out.ctypes.data_as(C.POINTER(C.c_float))))
        return out

    def forward(self, d_in, d_out, B: int) -> None:
        """d_in, d_out: device float32 buffers of B images (x(:) order)."""
        check(lib().airt_unet_forward(self._h, C.c_void_p(d_in), C.c_void_p(d_out), int(B)))

    def forward_f64(self, d_in, d_out, B: int, stream=0) -> None:
        """d_in, d_out: device float64 buffers of B images, any B; ordered on
        the CUDA stream `stream` (0: the network's own stream)."""
        check(lib().airt_unet_forward_f64(self._h, C.c_void_p(d_in), C.c_void_p(d_out), int(B),
                                          C.c_void_p(stream or None)))

    def gradients(self, d_in, d_tgt, B: int) -> float:
        loss = C.c_float()
        check(lib().airt_unet_gradients(self._h, C.c_void_p(d_in), C.c_void_p(d_tgt), int(B),
                                        C.byref(loss)))
        return float(loss.value)

    def train_step(self, d_in, d_tgt, B: int, lr: float) -> float:
        loss = C.c_float()
        check(lib().airt_unet_train_step(self._h, C.c_void_p(d_in), C.c_void_p(d_tgt), int(B),
                                         float(lr), C.byref(loss)))
        return float(loss.value)
