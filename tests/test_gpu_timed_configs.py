"""Parity at the configurations the benchmark times, against the FP64 C
oracle on the identical matrix (traced by the C restatement of
paralleltomo.m / fanlineartomo.m):

* C2: paralleltomo N=512, 360 angles x 724 rays (m=260,640, n=262,144,
  120 M nonzeros), 30-ellipse phantom, 0.5% noise.  cimmino 200 iterations
  with box [0,1] on the stored matrix; cav, drop, sart 10 iterations each;
  cimmino 5 iterations on the matrix-free projector.
* C4-shaped batch: 12 instances, N in {96,128,192,256}, 120-180 angles, 1-3%
  noise, cimmino and drop to the per-instance DP stop (the > 128 lane class
  and active-tile lists spanning many 2048-segment tiles run here).
* C3 fan: fanlineartomo N=1024, 1448 detectors, source at 2N, 36 of the 720
  half-degree angles, matrix-free SART to the DP stop (tau = 1.02, 1% noise).

Bar: relative iterate error <= 1e-5 after K iterations (sirt/sirt.m:198-261
run in FP64), identical DP stopping iterations.  The relaxation parameter is
passed explicitly so that the eigs tolerance is not part of the comparison.
"""
import numpy as np
import pytest

import airtoolsii_b200 as airt
from oracle import airt_oracle as O
from oracle import cbind

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def gpu_rho(op, method):
    """rho of the method's D*A'*M*A on the device (airt_rho)."""
    import ctypes as C
    from airtoolsii_b200 import _lib
    r = C.c_double()
    _lib.check(_lib.lib().airt_rho(op.handle, _lib.METHODS[method], None, None, 1e-7, 200,
                                   C.byref(r)))
    return float(r.value)


@pytest.fixture(scope="module")
def c2():
    theta = np.arange(360) * 0.5
    th, p, d, ct, st, off = O.parallel_geometry(512, theta, 724)
    rows, cols, vals = cbind.trace_coo(512, list(O.parallel_rays(512, ct, st, off)), True)
    Rm = O.coo_to_csc(rows, cols, vals, len(th) * p, 512 * 512)
    del rows, cols, vals
    A, *_ = airt.paralleltomo(512, theta, 724)
    assert A.nnz == Rm.nnz == 120_154_640
    x = O.random_ellipses(512, 30, seed=100)
    b, _ = O.add_noise(Rm @ x, 0.005, seed=200)
    return A, Rm, b, theta


def test_c2_cimmino_200_box(c2):
    """The benchmark's own workload: cimmino, 200 iterations, box [0,1]."""
    A, Rm, b, _ = c2
    M, D, _, _ = O.get_mfun_dfun("cimmino", Rm)
    lam = 1.9 / gpu_rho(A, "cimmino")
    X, info = airt.cimmino(A, b, [200], None, {"relaxpar": lam, "lbound": 0.0, "ubound": 1.0})
    assert info["finaliter"] == 200
    xo, k, _ = cbind.sirt_csr(Rm, b, M, D, lam, 0.0, 1.0, None, 200)
    assert k == 200
    assert relerr(X[:, -1], xo) <= RTOL, relerr(X[:, -1], xo)


@pytest.mark.parametrize("method,lam", [("cav", 1.0), ("drop", 1.0), ("sart", 1.9)])
def test_c2_methods_10_iterations(c2, method, lam):
    A, Rm, b, _ = c2
    M, D, _, _ = O.get_mfun_dfun(method, Rm)
    X, info = airt.sirt(method, A, b, [10], None, {"relaxpar": lam, "lbound": 0.0, "ubound": 1.0})
    xo, _, _ = cbind.sirt_csr(Rm, b, M, D, lam, 0.0, 1.0, None, 10)
    assert relerr(X[:, -1], xo) <= RTOL, (method, relerr(X[:, -1], xo))


def test_c2_matrix_free_cimmino_5_iterations(c2):
    A, Rm, b, theta = c2
    Amf, *_ = airt.paralleltomo(512, theta, 724, None, 0, 0)
    assert Amf.matrix_free
    M, D, _, _ = O.get_mfun_dfun("cimmino", Rm)
    lam = 1.9 / gpu_rho(A, "cimmino")
    X, _ = airt.cimmino(Amf, b, [5], None, {"relaxpar": lam, "lbound": 0.0, "ubound": 1.0})
    xo, _, _ = cbind.sirt_csr(Rm, b, M, D, lam, 0.0, 1.0, None, 5)
    assert relerr(X[:, -1], xo) <= RTOL, relerr(X[:, -1], xo)


@pytest.fixture(scope="module")
def c4_batch():
    rng = np.random.default_rng(44)
    Ns = [96, 128, 192, 256, 96, 128, 192, 256, 256, 192, 128, 96]
    nAs = [int(a) for a in rng.integers(120, 181, len(Ns))]
    etas = rng.uniform(0.01, 0.03, len(Ns))
    thetas = [np.arange(a) * (180.0 / a) for a in nAs]
    B = airt.ParallelBatch(Ns, thetas)
    mats, bs, tds = [], [], []
    for k, N in enumerate(Ns):
        th, p, d, ct, st, off = O.parallel_geometry(N, thetas[k], None)
        rows, cols, vals = cbind.trace_coo(N, list(O.parallel_rays(N, ct, st, off)), True)
        A = O.coo_to_csc(rows, cols, vals, len(th) * p, N * N)
        x = O.random_ellipses(N, 10, seed=10_000 + k)
        b, en = O.add_noise(A @ x, float(etas[k]), seed=20_000 + k)
        mats.append(A)
        bs.append(b)
        tds.append(1.02 * en)
    return B, mats, bs, np.array(tds)


def test_c4_batch_exercises_long_segments(c4_batch):
    """Mean row and column lengths above 128 for the N=256 instances, and a
    batch spanning many 2048-segment tiles."""
    B, mats, *_ = c4_batch
    big = [A for A in mats if A.shape[1] == 256 * 256]
    assert big and all(A.nnz / A.shape[0] > 128 and A.nnz / A.shape[1] > 128 for A in big)
    assert B.m // 2048 > 50 and B.n // 2048 > 50
    assert list(B.inst_nnz()) == [A.nnz for A in mats]


@pytest.mark.parametrize("method", ["cimmino", "drop"])
def test_c4_batch_dp_per_instance(c4_batch, method):
    B, mats, bs, tds = c4_batch
    rho = B.rho(method)
    xs, info = B.sirt(method, bs, 2000, taudelta=tds, rho=rho, lbound=0.0)
    for k, A in enumerate(mats):
        M, D, _, _ = O.get_mfun_dfun(method, A)
        xo, ko, _ = cbind.sirt_csr(A, bs[k], M, D, 1.9 / rho[k], 0.0, None, tds[k], 2000)
        assert info["finaliter"][k] == ko, (k, info["finaliter"][k], ko)
        assert info["stoprule"][k] == (2 if ko < 2000 else 0)
        assert relerr(xs[k], xo) <= RTOL, (k, relerr(xs[k], xo))


def test_c3_fan_matrix_free_sart_to_dp():
    """fanlineartomo N=1024, 1448 detectors, R = 2N, every 20th of the 720
    half-degree angles (36 projections), matrix-free SART (relaxpar 1.9,
    rho = 1 for sart) to the DP stop, against the C-traced FP64 matrix."""
    N = 1024
    theta = (np.arange(720) * 0.5)[::20]
    th, p, R, _, _, ct, st, cw, sw = O.fan_geometry(N, theta, 1448, 2.0)
    rows, cols, vals = cbind.trace_coo(N, list(O.fan_rays(N, R, ct, st, cw, sw)), False)
    Rm = O.coo_to_csc(rows, cols, vals, len(th) * p, N * N)
    del rows, cols, vals
    Af, *_ = airt.fanlineartomo(N, theta, 1448, 2.0, None, None, 0, 0)
    assert Af.matrix_free and Af.shape == Rm.shape
    x = O.random_ellipses(N, 10, seed=300)
    b, en = O.add_noise(Rm @ x, 0.01, seed=301)
    td = 1.02 * en
    X, info = airt.sart(Af, b, [1000], None, {"stoprule": {"type": "DP", "taudelta": td}})
    M, D, _, _ = O.get_mfun_dfun("sart", Rm)
    xo, ko, _ = cbind.sirt_csr(Rm, b, M, D, 1.9, None, None, td, 1000)
    assert 0 < ko < 1000
    assert info["finaliter"] == ko and info["stoprule"] == 2
    assert relerr(X[:, -1], xo) <= RTOL, relerr(X[:, -1], xo)
