"""train_relaxpar / train_dpme (train/train_relaxpar.m, train/train_dpme.m)
on the GPU solvers against the oracle's branch-for-branch port, with rho and
the noise matrix fixed so both see the same inputs."""
import numpy as np
import pytest

import airtoolsii_b200 as airt
from airtoolsii_b200 import train as T
from oracle import airt_oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def prob():
    theta = np.arange(0.0, 180.0, 3.0)
    A_ref = O.paralleltomo_matrix(32, theta)
    A, *_ = airt.paralleltomo(32, theta)
    x = airt.random_ellipses(32, 6, seed=41)
    b_ex = A_ref @ x
    b, en = airt.add_noise(b_ex, 0.03, seed=42)
    return A, A_ref, x, b_ex, b, en


@pytest.mark.parametrize("method,batched", [("cimmino", True), ("cimmino", False),
                                            ("sart", True), ("drop", True), ("kaczmarz", False)])
def test_train_relaxpar(prob, method, batched):
    """batched: the golden-section probes of the next three steps run as one
    multi-right-hand-side solve; the decisions, and so the result, are those
    of the sequential search."""
    A, A_ref, x, _, b, _ = prob
    opts = {}
    if method in ("cimmino", "drop"):
        _, io, _ = O.sirt(method, A_ref, b, [1])
        opts["rho"] = io["rho"]
    r_gpu = T.train_relaxpar(A, b, x, method, 60, opts, batched=batched)
    r_ref = O.train_relaxpar(A_ref, b, x, method, 60, opts)
    assert 0 < r_ref < 2 / (opts.get("rho", 1.0) if method != "kaczmarz" else 1.0)
    assert abs(r_gpu - r_ref) <= 1e-9 * r_ref


def test_train_relaxpar_columnaction(prob):
    """train_relaxpar.m:90 runs CART through the ART branch (relaxpar 0.25 to
    find kopt, golden section on (0, 2)); the oracle uses the FP32-rounded
    matrix so that both take the same flagging decisions."""
    A, A_ref, x, _, b, _ = prob
    R = A_ref.copy().tocsc()
    R.data = R.data.astype(np.float32).astype(np.float64)
    r_gpu = T.train_relaxpar(A, b, x, "columnaction", 30, {})
    r_ref = O.train_relaxpar(R, b, x, "columnaction", 30, {})
    assert 0 < r_ref < 2
    assert abs(r_gpu - r_ref) <= 1e-9 * r_ref


@pytest.mark.parametrize("rule,batched", [("DP", True), ("ME", True), ("DP", False)])
def test_train_dpme(prob, rule, batched):
    """batched: the replicas run together on the multi-right-hand-side
    engine with every iterate saved."""
    A, A_ref, x, b_ex, _, en = prob
    _, io, _ = O.sirt("cimmino", A_ref, b_ex, [1])
    opts = {"rho": io["rho"]}
    E = np.random.default_rng(7).standard_normal((A_ref.shape[0], 5))
    t_gpu = T.train_dpme(A, b_ex, x, "cimmino", rule, en, 5, 40, opts, E=E, batched=batched)
    t_ref = O.train_dpme(A_ref, b_ex, x, "cimmino", rule, en, E, 40, opts)
    assert t_ref > 0.5
    assert abs(t_gpu - t_ref) <= 1e-6 * t_ref
