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


def _bf16_rne(w: np.ndarray) -> np.ndarray:
    """FP32 -> BF16 bit patterns (uint16), round to nearest even."""
    u = np.ascontiguousarray(w, dtype=np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint16)


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

    def layer_shapes(self):
        """(cin, cout) of every 3x3 convolution in the order of the flattened
        parameters: encoder levels 0..L-1, then decoder levels L-2..0."""
        b, L = self.base, self.levels
        shapes = []
        for lv in range(L):
            shapes += [(1 if lv == 0 else b << (lv - 1), b << lv), (b << lv, b << lv)]
        for lv in range(L - 2, -1, -1):
            shapes += [((b << (lv + 1)) + (b << lv), b << lv), (b << lv, b << lv)]
        return shapes

    def _weight_mask(self) -> np.ndarray:
        """True for convolution weights, False for biases and the 1x1 head."""
        mask = np.zeros(self.num_params, bool)
        off = 0
        for cin, cout in self.layer_shapes():
            mask[off:off + 9 * cin * cout] = True
            off += 9 * cin * cout + cout
        assert off + self.base + 1 == self.num_params
        return mask

    def save(self, path, **meta) -> None:
        """Checkpoint for inference: 3x3 convolution weights as BF16 (the
        values the tensor cores use, so inference from the file is identical),
        biases and head in FP32, plus metadata."""
        p = self.get_params()
        mask = self._weight_mask()
        np.savez_compressed(path, w_bf16=_bf16_rne(p[mask]), rest_f32=p[~mask],
                            H=self.H, W=self.W, base=self.base, levels=self.levels,
                            meta=np.array(repr(meta)))

    def load(self, path) -> dict:
        """Load a checkpoint written by save (shape must match); returns its
        metadata."""
        z = np.load(path)
        if (int(z["H"]), int(z["W"]), int(z["base"]), int(z["levels"])) != (
                self.H, self.W, self.base, self.levels):
            raise ValueError("checkpoint was made for a different network shape")
        mask = self._weight_mask()
        p = np.zeros(self.num_params, np.float32)
        p[mask] = (z["w_bf16"].astype(np.uint32) << 16).view(np.float32)
        p[~mask] = z["rest_f32"]
        self.set_params(p)
        import ast
        return ast.literal_eval(str(z["meta"]))

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


def _timing_main():
    """python -m airtoolsii_b200.unet [--batch B] [--reps R] [--conv tap|halo|rows|rows1|stack]
    [--forward-only]: device time per image of the forward pass and of one
    Adam training step of the N=256, 4-level, base-32 network (random
    inputs), CUDA events on its stream; --conv picks the operand form of the
    TMA 3x3 convolutions (default: row runs where they apply; rows1: row runs
    with one strip per input row for 64-byte pixel rows; stack: row runs with
    the kernel rows stacked along N)."""
    import argparse
    import torch
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--conv", choices=["default", "tap", "halo", "rows", "rows1", "stack"], default="default")
    ap.add_argument("--forward-only", action="store_true")
    a = ap.parse_args()
    if a.conv != "default":
        f = lib().airt_test_conv_halo
        f.restype, f.argtypes = C.c_int, [C.c_int]
        check(f({"tap": 0, "halo": 1, "rows": 2, "rows1": 6, "stack": 3}[a.conv]))
    B = a.batch
    net = UNet(256, 256, 32, 4, B, 0)
    u = torch.rand(B, 65536, device="cuda")
    t = torch.rand_like(u)
    o = torch.empty_like(u)
    torch.cuda.synchronize()
    for _ in range(2):
        net.forward(u.data_ptr(), o.data_ptr(), B)
        if not a.forward_only:
            net.train_step(u.data_ptr(), t.data_ptr(), B, 1e-4)
    torch.cuda.synchronize()
    s = torch.cuda.ExternalStream(net.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    for _ in range(a.reps):
        net.forward(u.data_ptr(), o.data_ptr(), B)
    e1.record(s)
    torch.cuda.synchronize()
    fwd = e0.elapsed_time(e1) / a.reps / B
    if a.forward_only:
        print({"conv": a.conv, "forward_ms_per_image": round(fwd, 5)})
        return
    e0.record(s)
    for _ in range(a.reps):
        net.train_step(u.data_ptr(), t.data_ptr(), B, 1e-4)
    e1.record(s)
    torch.cuda.synchronize()
    print({"conv": a.conv, "forward_ms_per_image": round(fwd, 5),
           "train_ms_per_image": round(e0.elapsed_time(e1) / a.reps / B, 5)})


if __name__ == "__main__":
    _timing_main()
