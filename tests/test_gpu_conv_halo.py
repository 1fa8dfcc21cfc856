"""The halo-strip forms of the TMA 3x3 convolution (images whose rows hold
whole 128-pixel tiles: one 130-pixel strip per kernel row, the three taps
read it through shifted descriptors; per output row, per run of output
rows with the weights resident, or per run with the three kernel rows
stacked along N) against the nine-tap-box form on the same
network, inputs and weights: forward output, loss and every gradient
tensor.  The two forms add the same products in a different order for
inputs of more than one channel chunk, so the bar is the BF16-level one of
the oracle tests (1e-2 forward, 2e-2 gradients)."""
import ctypes as C

import numpy as np
import pytest

import airtoolsii_b200 as airt

pytestmark = pytest.mark.gpu


def _hook(name, v):
    f = getattr(airt._lib.lib(), name)
    f.restype, f.argtypes = C.c_int, [C.c_int]
    assert f(v) == 0


def _run(net, x, t, B):
    import torch
    dx = torch.from_numpy(x).cuda()
    dt = torch.from_numpy(t).cuda()
    out = torch.empty_like(dx)
    net.forward(dx.data_ptr(), out.data_ptr(), B)
    loss = net.gradients(dx.data_ptr(), dt.data_ptr(), B)
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64), loss, net.get_grads().astype(np.float64)


@pytest.mark.parametrize("mode", [1, 2, 6, 3], ids=["halo", "rows", "rows_one_strip", "stacked"])
@pytest.mark.parametrize("H,W,base,levels,B", [(256, 256, 32, 2, 2), (128, 256, 16, 2, 2),
                                               (128, 128, 32, 2, 2), (100, 128, 32, 2, 16)])
def test_halo_conv_matches_tap_boxes(mode, H, W, base, levels, B):
    # (100, 128) with 16 images: runs of 8 rows, the last run of each column 4 rows
    net = airt.UNet(H, W, base, levels, max_batch=B, seed=11)
    rng = np.random.default_rng(H + W + base)
    x = rng.random((B, H * W)).astype(np.float32)
    t = rng.random((B, H * W)).astype(np.float32)
    try:
        _hook("airt_test_conv_halo", 0)
        o0, l0, g0 = _run(net, x, t, B)
        _hook("airt_test_conv_halo", mode)
        o1, l1, g1 = _run(net, x, t, B)
    finally:
        _hook("airt_test_conv_halo", 3)      # the library default
    assert np.linalg.norm(o1 - o0) <= 1e-2 * np.linalg.norm(o0)
    assert abs(l1 - l0) <= 1e-3 * abs(l0)
    off = 0
    for cin, cout in net.layer_shapes():
        for n in (cout * 9 * cin, cout):
            a, r = g1[off:off + n], g0[off:off + n]
            assert np.linalg.norm(a - r) <= 2e-2 * np.linalg.norm(r) + 1e-12, (cin, cout, n)
            off += n
