"""Custom SIRT weights given as full matrices (auxil/get_mfun_dfun.m:252-307,
Mflag/Dflag = 2) on the GPU, against the FP64 oracle, and the reference
demo invariant of demos/demo_custom_sirt.m:36-74: custom SIRT with the full
weight matrix M = ((1/w)Delta + L')^-1 ((2/w - 1)Delta) ((1/w)Delta + L)^-1
(AA' = L + Delta + L') is symmetric Kaczmarz with relaxpar w, one SIRT
iteration per symmetric sweep pair.

Tolerance: relative iterate error <= 1e-5 (FP32 matrix values, FP64
arithmetic; measured ~1e-8)."""
import numpy as np
import pytest

import airtoolsii_b200 as airt
from oracle import airt_oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def demo():
    """demo_custom_sirt.m:17-25: N=50, theta = 0:5:175, p=75, zero rows
    removed (purge_rows), Shepp-Logan phantom, noise-free b."""
    A = O.paralleltomo_matrix(50, np.arange(0.0, 180.0, 5.0), 75).tocsr()
    A = A[np.flatnonzero(np.diff(A.indptr) > 0)].tocsc()
    b = A @ O.shepplogan(50)
    omega = 1.3
    AAT = (A @ A.T).toarray()
    L = np.tril(AAT, -1)
    Dl = np.diag(np.diag(AAT))
    T1 = np.linalg.solve((1 / omega) * Dl + L.T, (2 / omega - 1) * Dl)
    M = np.linalg.solve(((1 / omega) * Dl + L).T, T1.T).T
    return A, b, M, omega


def test_custom_full_M_equals_symmetric_kaczmarz(demo):
    A, b, M, omega = demo
    op = airt.afun_matrix(A)
    Xsym, _ = airt.symkaczmarz(op, b, list(range(2, 21, 2)), None, {"relaxpar": omega})
    Xc, info = airt.sirt({"M": M}, op, b, list(range(1, 11)), None, {"relaxpar": 1.0})
    assert Xc.shape == Xsym.shape == (A.shape[1], 10)
    Xo, _, _ = O.sirt({"M": M}, A, b, list(range(1, 11)), None, {"relaxpar": 1.0})
    for k in range(10):
        assert relerr(Xc[:, k], Xo[:, k]) <= RTOL
        assert relerr(Xc[:, k], Xsym[:, k]) <= RTOL
    assert abs(info["rho"] - 1.0) <= 1e-4           # eigs gives 0.99999999885 here


def test_custom_full_D_and_line_search(demo):
    """A full, non-diagonal D (with a full M) under constant, line-search and
    psi2 relaxation, box constraints and the DP rule."""
    A, b, M, _ = demo
    n = A.shape[1]
    rng = np.random.default_rng(8)
    Q = rng.standard_normal((n, 6))
    D = np.diag(rng.uniform(0.5, 1.5, n)) + 0.02 * (Q @ Q.T) / 6
    op = airt.afun_matrix(A)
    for opts in ({"relaxpar": 0.5}, {"relaxpar": "line"}, {"relaxpar": "psi2"},
                 {"relaxpar": 0.5, "lbound": 0.0, "ubound": 0.8}):
        meth = {"M": M, "D": D}
        Xo, io, _ = O.sirt(meth, A, b, [3, 12], None, dict(opts, rho=1.2))
        X, info = airt.sirt(meth, op, b, [3, 12], None, dict(opts, rho=1.2))
        assert info["finaliter"] == io["finaliter"] == 12
        for k in range(2):
            assert relerr(X[:, k], Xo[:, k]) <= RTOL, (opts, k, relerr(X[:, k], Xo[:, k]))
    # D alone full (M the identity), DP stop
    en = 0.02 * np.linalg.norm(b)
    Xo, io, _ = O.sirt({"D": D}, A, b, [200], None,
                       {"rho": 1.0e3, "relaxpar": 1e-3, "stoprule": {"type": "DP", "taudelta": en}})
    X, info = airt.sirt({"D": D}, op, b, [200], None,
                        {"rho": 1.0e3, "relaxpar": 1e-3, "stoprule": {"type": "DP", "taudelta": en}})
    assert info["finaliter"] == io["finaliter"] and info["stoprule"] == io["stoprule"]
    assert relerr(X[:, -1], Xo[:, -1]) <= RTOL


def test_custom_full_rho_matches_oracle(demo):
    """rho of D*A'*M*A for full weights (power iteration on the device)
    against the oracle's eigs (calc_relaxpar.m:91-103)."""
    A, b, M, _ = demo
    n = A.shape[1]
    rng = np.random.default_rng(9)
    Q = rng.standard_normal((n, 4))
    D = np.diag(rng.uniform(0.5, 1.5, n)) + 0.05 * (Q @ Q.T) / 4
    op = airt.afun_matrix(A)
    for meth in ({"M": M}, {"D": D}, {"M": M, "D": D}):
        _, io, _ = O.sirt(meth, A, b, [1])
        _, info = airt.sirt(meth, op, b, [1])
        assert abs(info["rho"] - io["rho"]) <= 1e-4 * abs(io["rho"]), (info["rho"], io["rho"])
