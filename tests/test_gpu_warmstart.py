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
