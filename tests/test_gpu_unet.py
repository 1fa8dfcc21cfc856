"""U-Net kernels (tcgen05 GEMM convolutions, pooling, upsampling, head, Adam)
against the FP64 NumPy restatement in oracle/unet_oracle.py, which rounds to
BF16 at the same points.  Tolerances: loss 1e-3 relative, every gradient
tensor 2e-2 relative Frobenius error (BF16 rounding of masked gradients can
flip on FP32-order differences), forward output 1e-2."""
import numpy as np
import pytest

import airtoolsii_b200 as airt
from oracle import unet_oracle as UO

pytestmark = pytest.mark.gpu


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).cuda()


def _set_gemm_path(path):
    import ctypes as C
    f = airt._lib.lib().airt_test_gemm_path
    f.restype, f.argtypes = C.c_int, [C.c_int]
    assert f(path) == 0


@pytest.mark.parametrize("path", [0, 1], ids=["tma", "cpasync"])
@pytest.mark.parametrize("levels,base", [(2, 8), (3, 8), (2, 32)])
def test_unet_gradients_vs_oracle(levels, base, path):
    """base 8: channel widths 8 (cp.async gathers), 16 and 32 (TMA, 32- and
    64-byte swizzle); base 32: widths 32, 64 and 96 (64- and 128-byte
    swizzle); 16x16 and 8x8 images exercise pixel boxes of one and two
    images."""
    _set_gemm_path(path)
    try:
        _check_gradients(levels, base)
    finally:
        _set_gemm_path(0)


def _check_gradients(levels, base):
    import torch
    H = W = 16
    B = 2
    net = airt.UNet(H, W, base, levels, max_batch=B, seed=7)
    rng = np.random.default_rng(levels)
    x = rng.random((B, H * W)).astype(np.float32)
    t = rng.random((B, H * W)).astype(np.float32)
    dx, dt = _dev(x), _dev(t)
    loss = net.gradients(dx.data_ptr(), dt.data_ptr(), B)
    torch.cuda.synchronize()
    g = net.get_grads().astype(np.float64)
    p = net.get_params()
    lo, go, out_o = UO.forward_backward(p.astype(np.float64), x.astype(np.float64), t.astype(np.float64), base, levels, H, W)
    assert abs(loss - lo) <= 1e-3 * lo
    off = 0
    for cin, cout in UO.layer_shapes(base, levels):
        for n in (cout * 9 * cin, cout):
            a, r = g[off:off + n], go[off:off + n]
            assert np.linalg.norm(a - r) <= 2e-2 * np.linalg.norm(r) + 1e-12, (cin, cout, n)
            off += n
    a, r = g[off:], go[off:]
    assert np.linalg.norm(a - r) <= 2e-2 * np.linalg.norm(r)
    # forward output in image order
    dout = torch.zeros(B * H * W, dtype=torch.float32, device="cuda")
    net.forward(dx.data_ptr(), dout.data_ptr(), B)
    torch.cuda.synchronize()
    out = dout.cpu().numpy().reshape(B, W, H).transpose(0, 2, 1)
    assert np.linalg.norm(out - out_o) <= 1e-2 * np.linalg.norm(out_o)


def test_unet_params_roundtrip_and_training_reduces_loss():
    import torch
    H = W = 32
    net = airt.UNet(H, W, 8, 3, max_batch=4, seed=3)
    p = net.get_params()
    net.set_params(p)
    assert np.array_equal(net.get_params(), p)
    rng = np.random.default_rng(0)
    x = rng.random((4, H * W)).astype(np.float32)
    t = (0.5 * x + 0.1).astype(np.float32)
    dx, dt = _dev(x), _dev(t)
    l0 = net.train_step(dx.data_ptr(), dt.data_ptr(), 4, 1e-3)
    for _ in range(60):
        l1 = net.train_step(dx.data_ptr(), dt.data_ptr(), 4, 1e-3)
    assert np.isfinite(l1) and l1 < 0.5 * l0


def test_unet_full_size_forward():
    import torch
    net = airt.UNet(256, 256, 32, 4, max_batch=2, seed=1)
    x = _dev(np.random.default_rng(1).random((2, 256 * 256)))
    out = torch.zeros(2 * 256 * 256, dtype=torch.float32, device="cuda")
    net.forward(x.data_ptr(), out.data_ptr(), 2)
    torch.cuda.synchronize()
    assert torch.isfinite(out).all()
    loss = net.train_step(x.data_ptr(), x.data_ptr(), 2, 1e-4)
    assert np.isfinite(loss)
