"""Learned warm start: the GPU phantom rasterizer against the oracle's
ellipse rasterisation, and what a trained U-Net gains over plain SIRT from
zero (fewer iterations to the DP stop at no worse relative error)."""
import math

import numpy as np
import pytest

from oracle import airt_oracle as O

pytestmark = pytest.mark.gpu


def ws_single_dp(ws, b, taudelta):
    from airtoolsii_b200.solvers import cimmino
    return cimmino(ws.A, b, 2000, None, {"stoprule": {"type": "DP", "taudelta": taudelta},
                                         "rho": ws.rho})


@pytest.fixture(scope="module")
def ws():
    from airtoolsii_b200.warmstart import WarmStart
    return WarmStart(N=64, theta=np.arange(0.0, 180.0, 6.0), base=16, levels=3, max_batch=16,
                     seed=2)


def test_gpu_phantoms_match_oracle_rasterisation(ws):
    from airtoolsii_b200.warmstart import ellipse_params
    seeds = [3, 4, 5]
    xs = ws.phantoms(seeds).cpu().numpy()
    prm = ellipse_params(seeds)
    for k in range(len(seeds)):
        ell = [(a, ea, eb, x0, y0, math.atan2(s, c)) for a, ea, eb, x0, y0, c, s in prm[k]]
        ref = O.ellipse_image(64, ell, clip_hi=1.0).ravel(order="F")
        assert np.mean(xs[k] != ref) < 2e-3      # rounding of cos/sin at ellipse edges only
        assert np.abs(xs[k] - ref).sum() / ref.sum() < 1e-2


def test_warm_start_beats_plain_sirt(ws):
    train = ws.prepare(list(range(1000, 1640)), eta=0.02)
    hist = ws.train(train["u"], train["target"], epochs=4, batch=16, lr=2e-3)
    assert hist[-1] < hist[0]
    test = ws.prepare(list(range(50_000, 50_032)), eta=0.02)
    r = ws.compare_batched(test)
    assert np.all(r["plain_iters"] == test["iters"])           # same batch, same stop
    for k in (0, 17):                                           # batch == single-problem GPU SIRT
        _, info = ws_single_dp(ws, test["b"][k].cpu().numpy(), test["taudelta"][k])
        assert info["finaliter"] == test["iters"][k]
    assert np.mean(r["x0_relerr"]) < 0.5                        # x0 is far better than zero
    assert np.mean(r["warm_iters"]) < 0.75 * np.mean(r["plain_iters"])
    assert np.mean(r["warm_relerr"]) <= 1.05 * np.mean(r["plain_relerr"])


def test_checkpoint_roundtrip(tmp_path):
    """The committed checkpoint loads, saves and reloads to identical
    parameters and an identical forward pass."""
    import torch
    from airtoolsii_b200 import warmstart as W
    from airtoolsii_b200.unet import UNet
    a = UNet(256, 256, 32, 4, max_batch=2, seed=5)
    meta = a.load(W.checkpoint_path())
    assert meta["epochs"] == W.C5["epochs"]
    a.save(tmp_path / "c.npz", **meta)
    b = UNet(256, 256, 32, 4, max_batch=2, seed=6)
    b.load(tmp_path / "c.npz")
    assert np.array_equal(a.get_params(), b.get_params())
    x = torch.rand(2 * 256 * 256, device="cuda")
    ya, yb = torch.empty_like(x), torch.empty_like(x)
    a.forward(x.data_ptr(), ya.data_ptr(), 2)
    b.forward(x.data_ptr(), yb.data_ptr(), 2)
    torch.cuda.synchronize()
    assert torch.equal(ya, yb)


def test_checkpoint_cuts_dp_iterations():
    """What the trained network gains on held-out N=256 problems (seeds never
    used in training): far fewer cimmino iterations to the DP stop, at a
    relative error no worse than plain SIRT from zero."""
    from airtoolsii_b200 import warmstart as W
    ws = W.c5_warmstart(max_batch=16, chunk=16)
    ws.net.load(W.checkpoint_path())
    te = ws.prepare(list(range(700_000, 700_016)), eta=W.C5["eta"])
    r = ws.compare_batched(te)
    assert np.mean(r["warm_iters"]) < 0.4 * np.mean(r["plain_iters"])
    assert np.mean(r["warm_relerr"]) <= 1.02 * np.mean(r["plain_relerr"])
    assert np.mean(r["x0_relerr"]) < 1.1 * np.mean(r["plain_relerr"])
    # the multi-batch pipeline (network of batch i+1 overlapping the solve of
    # batch i) solves the same problems to the same stop iterations
    ws16 = W.c5_warmstart(max_batch=16, chunk=8)
    ws16.net.load(W.checkpoint_path())
    t = ws16.time_to_dp(te, 8)
    np.testing.assert_array_equal(t["plain_iters"], r["plain_iters"])
    np.testing.assert_array_equal(t["warm_iters"], r["warm_iters"])
    np.testing.assert_allclose(t["warm_relerr"], r["warm_relerr"], rtol=1e-6)
