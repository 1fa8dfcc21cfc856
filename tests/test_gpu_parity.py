"""GPU parity tests: libairt through its C-ABI against the FP64 oracle.

Tolerances: the generated system matrix is bit-exact (pattern, and values
equal to the FP64 trace rounded to FP32); SIRT/ART iterates agree with the
FP64 oracle to a relative error <= 1e-5 after K iterations (rho passed
explicitly so that the eigs tolerance is not part of the comparison).
"""
import os

import numpy as np
import pytest
import scipy.sparse as sp

import airtoolsii_b200 as airt
from oracle import airt_oracle as O
from oracle import cbind

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
RTOL = 1e-5


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def same_matrix(A_gpu, A_ref):
    E = A_gpu.to_scipy()
    R = sp.csc_matrix(A_ref)
    assert E.shape == R.shape
    assert np.array_equal(E.indptr, R.indptr)
    assert np.array_equal(E.indices, R.indices)
    assert np.array_equal(E.data, R.data.astype(np.float32).astype(np.float64))


# ------------------------------------------------------------ matrix generation
def test_golden_parallel_matrix():
    g = np.load(os.path.join(GOLD, "paralleltomo_N16_30ang.npz"))
    A, b, x, *_ = airt.paralleltomo(16, g["theta"])
    R = sp.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=tuple(g["shape"]))
    same_matrix(A, R)
    np.testing.assert_allclose(b, R @ g["x"], rtol=1e-6)


def test_golden_widened_rows():
    """libairt against widened_N16.npz: seismictomo and sphericaltomo matrices
    bit-exact, CART columnaction iterates (1e-9) and fbp (1e-10)."""
    g = np.load(os.path.join(GOLD, "paralleltomo_N16_30ang.npz"))
    w = np.load(os.path.join(GOLD, "widened_N16.npz"))
    As, *_ = airt.seismictomo(12, 6, 10)
    same_matrix(As, sp.csc_matrix((w["seis_data"], w["seis_indices"], w["seis_indptr"]),
                                  shape=tuple(w["seis_shape"])))
    Aq, *_ = airt.sphericaltomo(10, np.arange(0.0, 360.0, 30.0), 8)
    same_matrix(Aq, sp.csc_matrix((w["sph_data"], w["sph_indices"], w["sph_indptr"]),
                                  shape=tuple(w["sph_shape"])))
    A = airt.afun_matrix(sp.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=tuple(g["shape"])))
    opts = {"lbound": 0.0, "Kbegin": 2, "Nunflag": 2, "THR": 1e-2, "seed": 5}
    X, info = airt.columnaction(A, g["b"], [2, 6], None, opts)
    assert relerr(X, w["cart_X"]) <= 1e-9 and info["finaliter"] == int(w["cart_finaliter"])
    assert relerr(airt.fbp(A, g["b"], g["theta"], "hamming"), w["fbp_hamming"]) <= 1e-10
    assert relerr(airt.fbp(A, g["b"], g["theta"], "ram-lak"), w["fbp_ramlak"]) <= 1e-10


def test_golden_fan_matrix():
    g = np.load(os.path.join(GOLD, "fanlineartomo_N12_30ang.npz"))
    A, *_ = airt.fanlineartomo(12, np.arange(0.0, 360.0, 12.0), 17)
    same_matrix(A, sp.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=tuple(g["shape"])))


def test_c1_matrix_bit_exact():
    """N=64, 180 angles, p=91 (the CPU-runnable configuration)."""
    A, *_ = airt.paralleltomo(64)
    assert A.shape == (16380, 4096) and A.nnz == 938572
    same_matrix(A, O.paralleltomo_matrix(64))


@pytest.mark.parametrize("N,theta,p,d", [
    (15, np.arange(0.0, 180.0, 7.5), 21, 18.5),
    (12, np.array([0, 45, 90, 135, 180, 225, 270, 315.0]), 17, None),
    (1, np.array([0.0, 30.0]), 3, None),
])
def test_parallel_edge_geometries(N, theta, p, d):
    A, *_ = airt.paralleltomo(N, theta, p, d)
    same_matrix(A, O.paralleltomo_matrix(N, theta, p, d))


def test_fan_matrix_vs_c_oracle():
    N = 40
    th, p, R, _, _, ct, st, cw, sw = O.fan_geometry(N, np.arange(0.0, 360.0, 4.0))
    rows, cols, vals = cbind.trace_coo(N, list(O.fan_rays(N, R, ct, st, cw, sw)), False)
    Rm = O.coo_to_csc(rows, cols, vals, len(th) * p, N * N)
    A, *_ = airt.fanlineartomo(N, np.arange(0.0, 360.0, 4.0))
    same_matrix(A, Rm)


@pytest.mark.parametrize("N,theta,p,R,d", [(40, np.arange(0.0, 360.0, 4.0), None, None, None),
                                          (33, np.arange(0.0, 360.0, 7.5), 45, 1.5, 60.0)])
def test_fancurved_matrix_vs_c_oracle(N, theta, p, R, d):
    """fancurvedtomo (arc detector): bit-exact against the C tracer fed with
    the oracle's fancurvedtomo.m tables; matrix-free products agree."""
    th, pp, Rabs, dd, ct, st, cw, sw = O.fancurved_geometry(N, theta, p, 2.0 if R is None else R, d)
    rows, cols, vals = cbind.trace_coo(N, list(O.fan_rays(N, Rabs, ct, st, cw, sw)), False)
    Rm = O.coo_to_csc(rows, cols, vals, len(th) * pp, N * N)
    A, b, x, th2, p2, R2, d2 = airt.fancurvedtomo(N, theta, p, R, d)
    assert p2 == pp and abs(d2 - dd) == 0 and R2 == Rabs / N
    same_matrix(A, Rm)
    Amf, *_ = airt.fancurvedtomo(N, theta, p, R, d, 0, 0)
    v = np.random.default_rng(N).random(N * N)
    y = Amf(v, "notransp")
    assert np.linalg.norm(y - Rm @ v) <= 1e-6 * np.linalg.norm(Rm @ v)


@pytest.mark.parametrize("N,s,p", [(48, None, None), (31, 9, 40), (10, 1, 1)])
def test_seismic_matrix_vs_c_oracle(N, s, p):
    """seismictomo: bit-exact against the C tracer fed with the oracle's
    source/receiver tables (horizontal rays included); b is A*x of the
    tectonic phantom; matrix-free products agree."""
    s_, p_, x0, y0, xp, yp = O.seismic_geometry(N, s, p)
    rows, cols, vals = cbind.trace_coo(N, list(O.seismic_rays(x0, y0, xp, yp)), False)
    Rm = O.coo_to_csc(rows, cols, vals, s_ * p_, N * N)
    A, b, x, s2, p2 = airt.seismictomo(N, s, p)
    assert (s2, p2) == (s_, p_)
    same_matrix(A, Rm)
    np.testing.assert_array_equal(x, O.tectonic(N).ravel(order="F"))
    R32 = Rm.copy()
    R32.data = R32.data.astype(np.float32).astype(np.float64)
    np.testing.assert_allclose(b, R32 @ x, rtol=1e-12, atol=1e-12)
    Amf, *_ = airt.seismictomo(N, s, p, 0, 0)
    v = np.random.default_rng(N).random(N * N)
    y = Amf(v, "notransp")
    assert np.linalg.norm(y - Rm @ v) <= 1e-6 * np.linalg.norm(Rm @ v)
    u = np.random.default_rng(N + 1).random(s_ * p_)
    assert np.linalg.norm(Amf(u, "transp") - Rm.T @ u) <= 1e-6 * np.linalg.norm(Rm.T @ u)


@pytest.mark.parametrize("N,angles,nc", [(16, None, None), (33, [0.0, 45.0, 97.5, 200.0], 7),
                                         (40, np.arange(0.0, 360.0, 24.0), None)])
def test_spherical_matrix_vs_oracle(N, angles, nc):
    """sphericaltomo: bit-exact against the oracle's unique/histc restatement
    (same circle-sample tables); matrix-free products within the FP32 entry
    rounding, matrix-free SIRT weights equal to the stored matrix's."""
    Ro = O.sphericaltomo_matrix(N, angles, nc)
    A, b, x, ang, nc2 = airt.sphericaltomo(N, angles, nc)
    assert nc2 == Ro.shape[0] // len(ang)
    same_matrix(A, Ro)
    R32 = Ro.copy()
    R32.data = R32.data.astype(np.float32).astype(np.float64)
    np.testing.assert_allclose(b, R32 @ x, rtol=1e-12, atol=1e-12)
    Amf, *_ = airt.sphericaltomo(N, angles, nc, 0, 0)
    assert Amf.matrix_free
    v = np.random.default_rng(N).random(N * N)
    assert np.linalg.norm(Amf(v, "notransp") - Ro @ v) <= 1e-6 * np.linalg.norm(Ro @ v)
    u = np.random.default_rng(N + 1).random(Ro.shape[0])
    assert np.linalg.norm(Amf(u, "transp") - Ro.T @ u) <= 1e-6 * np.linalg.norm(Ro.T @ u)
    for meth in ("cimmino", "cav", "drop", "sart"):
        Ms, Ds = A.weights(meth)
        Mm, Dm = Amf.weights(meth)
        np.testing.assert_allclose(Mm, Ms, rtol=1e-12)
        np.testing.assert_allclose(Dm, Ds, rtol=1e-12)
    Xs, info = airt.cimmino(A, b, 20)
    Xm, _ = airt.cimmino(Amf, b, 20, None, {"rho": info["rho"]})
    assert relerr(Xm, Xs) <= 1e-5


def test_c2_matrix_bit_exact_sampled_angles():
    """N=512, p=724 on 24 of the 360 half-degree angles (full-size rays)."""
    theta = (np.arange(360) * 0.5)[::15]
    th, p, d, ct, st, off = O.parallel_geometry(512, theta, 724)
    rows, cols, vals = cbind.trace_coo(512, list(O.parallel_rays(512, ct, st, off)), True)
    Rm = O.coo_to_csc(rows, cols, vals, len(th) * p, 512 * 512)
    A, *_ = airt.paralleltomo(512, theta, 724)
    same_matrix(A, Rm)


def test_csc_upload_roundtrip_and_apply():
    rng = np.random.default_rng(0)
    R = sp.random(300, 200, density=0.05, random_state=1, format="csc")
    R.data = rng.standard_normal(R.nnz)
    op = airt.afun_matrix(R)
    same_matrix(op, R)
    x = rng.standard_normal(200)
    y = rng.standard_normal(300)
    R32 = R.copy()
    R32.data = R32.data.astype(np.float32).astype(np.float64)
    np.testing.assert_allclose(op(x, "notransp"), R32 @ x, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(op(y, "transp"), R32.T @ y, rtol=1e-12, atol=1e-12)
    assert list(op(None, "size")) == [300, 200]


def test_csc_with_unsorted_or_duplicate_rows_is_rejected():
    """airt_problem_from_csc takes MATLAB's canonical sparse form only: a
    column whose row indices repeat or decrease is an argument error."""
    import ctypes as C
    from airtoolsii_b200 import _lib
    L = _lib.lib()
    h = C.c_void_p()
    jc = np.array([0, 2, 3], np.uint64)
    pr = np.array([1.0, 2.0, 3.0])
    for ir in (np.array([1, 1, 0], np.uint64), np.array([2, 0, 1], np.uint64)):
        st = L.airt_problem_from_csc(3, 2, _lib.u64ptr(jc), _lib.u64ptr(ir), _lib.dptr(pr),
                                     C.byref(h))
        assert st == _lib.AIRT_ERR_ARG
        assert b"strictly increasing" in L.airt_last_error()
    ir = np.array([0, 2, 1], np.uint64)
    assert L.airt_problem_from_csc(3, 2, _lib.u64ptr(jc), _lib.u64ptr(ir), _lib.dptr(pr),
                                   C.byref(h)) == _lib.AIRT_OK
    L.airt_destroy(h)


def test_empty_and_degenerate_matrices():
    op = airt.afun_matrix(sp.csc_matrix((5, 4)))
    assert op.nnz == 0
    np.testing.assert_array_equal(op(np.ones(4), "notransp"), np.zeros(5))
    np.testing.assert_array_equal(op(np.ones(5), "transp"), np.zeros(4))


# ------------------------------------------------------------ matrix-free
@pytest.mark.parametrize("geo", ["parallel", "fan"])
def test_matrix_free_equals_stored(geo):
    rng = np.random.default_rng(3)
    if geo == "parallel":
        As, *_ = airt.paralleltomo(48, np.arange(0.0, 180.0, 2.0), None, None, 0, 1)
        Am, *_ = airt.paralleltomo(48, np.arange(0.0, 180.0, 2.0), None, None, 0, 0)
    else:
        As, *_ = airt.fanlineartomo(40, np.arange(0.0, 360.0, 5.0), None, None, None, None, 0, 1)
        Am, *_ = airt.fanlineartomo(40, np.arange(0.0, 360.0, 5.0), None, None, None, None, 0, 0)
    assert Am.matrix_free
    x = rng.random(As.n)
    y = rng.random(As.m)
    np.testing.assert_allclose(Am(x, "notransp"), As(x, "notransp"), rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(Am(y, "transp"), As(y, "transp"), rtol=1e-12, atol=1e-11)
    for meth in ("cimmino", "cav", "drop", "sart"):
        Ms, Ds = As.weights(meth)
        Mm, Dm = Am.weights(meth)
        np.testing.assert_allclose(Mm, Ms, rtol=1e-12)
        np.testing.assert_allclose(Dm, Ds, rtol=1e-12)


@pytest.mark.parametrize("geo", ["parallel", "fan"])
def test_matrix_free_adjoint_is_bitwise_repeatable(geo):
    """The matrix-free back projection accumulates in fixed point, so two
    calls (and two SIRT solves on the matrix-free operator) agree bit for
    bit, whatever order the rays' terms arrive in."""
    if geo == "parallel":
        Am, b, *_ = airt.paralleltomo(96, np.arange(0.0, 180.0, 1.0), None, None, 0, 0)
    else:
        Am, b, *_ = airt.fanlineartomo(80, np.arange(0.0, 360.0, 2.0), None, None, None, None, 0, 0)
    y = np.random.default_rng(7).standard_normal(Am.m)
    g1 = Am(y, "transp")
    g2 = Am(y, "transp")
    assert np.array_equal(g1, g2)
    X1, _ = airt.sart(Am, b, 5)
    X2, _ = airt.sart(Am, b, 5)
    assert np.array_equal(X1, X2)


def test_matrix_free_sart_equals_stored_sart():
    """demos/demo_matrixfree.m: SART on the matrix and on the matrix-free
    operator give the same iterates."""
    As, b, *_ = airt.paralleltomo(40, np.arange(0.0, 180.0, 3.0))
    Am, *_ = airt.paralleltomo(40, np.arange(0.0, 180.0, 3.0), None, None, 0, 0)
    Xs, _ = airt.sart(As, b, 30)
    Xm, _ = airt.sart(Am, b, 30)
    assert relerr(Xm, Xs) <= 1e-6


# ------------------------------------------------------------ SIRT
@pytest.fixture(scope="module")
def c1():
    A_ref = O.paralleltomo_matrix(64)
    A, *_ = airt.paralleltomo(64)
    x = airt.random_ellipses(64, 10, seed=11)
    b, enorm = airt.add_noise(A_ref @ x, 0.01, seed=12)
    return A, A_ref, b, enorm, x


@pytest.mark.parametrize("method", ["landweber", "cimmino", "cav", "drop", "sart"])
def test_sirt_methods_c1(c1, method):
    """C1: 50 iterations, default relaxpar, nonneg=true."""
    A, A_ref, b, _, _ = c1
    Xo, io, _ = O.sirt(method, A_ref, b, [10, 50], options={"lbound": 0.0})
    X, info = airt.sirt(method, A, b, [10, 50], None, {"lbound": 0.0, "rho": io["rho"]})
    assert X.shape == Xo.shape and info["finaliter"] == 50
    assert relerr(X[:, 0], Xo[:, 0]) <= RTOL
    assert relerr(X[:, 1], Xo[:, 1]) <= RTOL
    assert list(info["itersaved"]) == [10, 50]
    assert abs(info["relaxpar"] - io["relaxpar"]) <= 1e-12 * abs(io["relaxpar"])


@pytest.mark.parametrize("method", ["landweber", "cimmino", "cav", "drop"])
def test_rho_power_iteration_vs_eigs(c1, method):
    A, A_ref, b, _, _ = c1
    _, io, _ = O.sirt(method, A_ref, b, [1])
    _, info = airt.sirt(method, A, b, [1])
    assert abs(info["rho"] - io["rho"]) <= 1e-4 * io["rho"]


def test_sirt_weights_vs_oracle(c1):
    A, A_ref, *_ = c1
    for meth in ("landweber", "cimmino", "cav", "drop", "sart"):
        M, D = A.weights(meth)
        Mo, Do, _, _ = O.get_mfun_dfun(meth, A_ref)
        np.testing.assert_allclose(M, Mo, rtol=1e-6)
        np.testing.assert_allclose(D, Do, rtol=1e-6)


def test_sirt_box_vector_bounds_x0(c1):
    A, A_ref, b, _, x = c1
    n = A.n
    lb = np.zeros(n)
    ub = np.full(n, 0.8)
    ub[::7] = 0.3
    x0 = 0.5 * x
    opts = {"lbound": lb, "ubound": ub, "rho": 1.0}
    Xo, _, _ = O.sirt("sart", A_ref, b, [3, 7, 20], x0, opts)
    X, _ = airt.sart(A, b, [3, 7, 20], x0, opts)
    assert relerr(X, Xo) <= RTOL
    assert X.min() >= 0 and np.all(X <= ub[:, None] + 0)


@pytest.mark.parametrize("rule", ["line", "psi1", "psi1mod", "psi2", "psi2mod"])
def test_sirt_relaxation_strategies(c1, rule):
    A, A_ref, b, _, _ = c1
    _, io, _ = O.sirt("cimmino", A_ref, b, [1])
    opts = {"relaxpar": rule, "rho": io["rho"], "lbound": 0.0}
    Xo, io2, _ = O.sirt("cimmino", A_ref, b, [5, 25], options=opts)
    X, info = airt.cimmino(A, b, [5, 25], None, opts)
    assert relerr(X, Xo) <= RTOL
    assert abs(info["relaxpar"] - io2["relaxpar"]) <= 1e-6 * abs(io2["relaxpar"])


def test_sirt_dp_stop(c1):
    A, A_ref, b, enorm, _ = c1
    _, io, _ = O.sirt("cimmino", A_ref, b, [1])
    opts = {"stoprule": {"type": "DP", "taudelta": 1.02 * enorm}, "rho": io["rho"]}
    Xo, io2, _ = O.sirt("cimmino", A_ref, b, [5, 1000], options=opts)
    X, info = airt.cimmino(A, b, [5, 1000], None, opts)
    assert io2["stoprule"] == 2
    assert info["stoprule"] == 2 and info["finaliter"] == io2["finaliter"]
    assert relerr(X, Xo) <= RTOL
    np.testing.assert_allclose(info["resnorms"][1:], io2["resnorms"], rtol=1e-5)
    assert abs(info["resnorms"][0] - np.linalg.norm(b)) <= 1e-6 * np.linalg.norm(b)


def test_sirt_me_stop(c1):
    A, A_ref, b, enorm, _ = c1
    opts = {"stoprule": {"type": "ME", "taudelta": 1.02 * enorm}, "rho": 1.0}
    Xo, io, _ = O.sirt("sart", A_ref, b, [500], options=opts)
    X, info = airt.sart(A, b, [500], None, opts)
    assert info["stoprule"] == io["stoprule"] == 3
    assert info["finaliter"] == io["finaliter"]
    assert relerr(X, Xo) <= RTOL


@pytest.mark.parametrize("method,dims,smooth", [("cimmino", "2d", 2), ("sart", "2d", 4),
                                                ("cimmino", "1d", 2), ("drop", "2d", 3)])
def test_sirt_ncp_stop(c1, method, dims, smooth):
    """NCP (check_stoprules.m:97-150) on the C1 problem: res_dims = [p, nA]
    (column-wise periodograms of the sinogram) or a scalar (the whole
    residual as one signal); same stop iteration and iterates as the oracle."""
    A, A_ref, b, _, _ = c1
    rd = [91, 180] if dims == "2d" else A.m
    opts = {"stoprule": {"type": "NCP", "res_dims": rd, "ncp_smooth": smooth}}
    if method != "sart":
        _, io, _ = O.sirt(method, A_ref, b, [1])
        opts["rho"] = io["rho"]
    Xo, io2, _ = O.sirt(method, A_ref, b, [5, 800], options=opts)
    X, info = airt.sirt(method, A, b, [5, 800], None, opts)
    assert io2["stoprule"] == 1
    assert info["stoprule"] == 1 and info["finaliter"] == io2["finaliter"]
    assert relerr(X, Xo) <= RTOL


@pytest.mark.parametrize("method,smooth", [("kaczmarz", 2), ("symkaczmarz", 2), ("kaczmarz", 3)])
def test_art_ncp_stop(c1, method, smooth):
    """NCP for ART (art.m calls check_stoprules after every sweep): same stop
    sweep and saved iterates as the oracle."""
    A, A_ref, b, _, _ = c1
    opts = {"stoprule": {"type": "NCP", "res_dims": [91, 180], "ncp_smooth": smooth}}
    K = list(range(1, 31)) if method == "kaczmarz" else list(range(2, 31, 2))
    Xo, io = O.art(method, A_ref, b, K, None, opts)
    X, info = getattr(airt, method)(A, b, K, None, opts)
    assert io["stoprule"] == 1
    assert info["stoprule"] == 1 and info["finaliter"] == io["finaliter"]
    assert X.shape == Xo.shape
    for k in range(X.shape[1]):
        assert relerr(X[:, k], Xo[:, k]) <= RTOL


def test_sirt_ncp_reaches_kmax(c1):
    """NCP with kmax below its stop: stoprule 0 at kmax, as the reference."""
    A, A_ref, b, _, _ = c1
    opts = {"stoprule": {"type": "NCP", "res_dims": [91, 180]}, "rho": 1.0}
    Xo, io, _ = O.sirt("sart", A_ref, b, [7], options=opts)
    X, info = airt.sart(A, b, [7], None, opts)
    assert info["stoprule"] == io["stoprule"] == 0 and info["finaliter"] == 7
    assert relerr(X, Xo) <= RTOL


def test_sirt_dp_at_k0_returns_empty(c1):
    A, _, b, _, _ = c1
    X, info = airt.cimmino(A, b, [10], None, {"stoprule": {"type": "DP", "taudelta": 1e12}})
    assert X.shape == (A.n, 0) and info["finaliter"] == 0 and list(info["itersaved"]) == [0]


def test_sirt_custom_weights(c1):
    A, A_ref, b, _, _ = c1
    rn = np.asarray(A_ref.multiply(A_ref).sum(axis=1)).ravel()
    Mc = np.where(rn > 0, 1.0 / np.where(rn > 0, rn, 1), 0.0)
    Dc = np.linspace(0.5, 1.5, A.n)
    meth = {"M": sp.diags(Mc), "D": Dc}
    Xo, io, _ = O.sirt(meth, A_ref, b, [20])
    X, info = airt.sirt(meth, A, b, [20], None, {"rho": io["rho"]})
    assert relerr(X, Xo) <= RTOL
    _, info2 = airt.sirt(meth, A, b, [1])
    assert abs(info2["rho"] - io["rho"]) <= 1e-4 * io["rho"]
    Xe, _ = airt.sirt({}, A, b, [20], None, {"rho": 20000.0})
    Xl, _ = airt.landweber(A, b, [20], None, {"rho": 20000.0})
    np.testing.assert_array_equal(Xe, Xl)


def test_sirt_matrix_free_vs_oracle():
    N = 32
    theta = np.arange(0.0, 180.0, 4.0)
    A_ref = O.paralleltomo_matrix(N, theta)
    Am, *_ = airt.paralleltomo(N, theta, None, None, 0, 0)
    b, _ = airt.add_noise(A_ref @ O.shepplogan(N), 0.02, seed=4)
    for meth in ("cimmino", "drop"):
        Xo, io, _ = O.sirt(meth, A_ref, b, [15], options={"lbound": 0.0})
        X, _ = airt.sirt(meth, Am, b, [15], None, {"lbound": 0.0, "rho": io["rho"]})
        assert relerr(X, Xo) <= RTOL


def test_sirt_input_errors(c1):
    A, _, b, _, _ = c1
    with pytest.raises(ValueError, match="size of A and b"):
        airt.cimmino(A, b[:-1], 5)
    with pytest.raises(ValueError, match="strictly increasing"):
        airt.cimmino(A, b, [5, 5])
    with pytest.raises(ValueError, match="taudelta"):
        airt.cimmino(A, b, 5, None, {"stoprule": {"type": "DP"}})
    with pytest.raises(ValueError, match="only available for SIRT"):
        airt.kaczmarz(A, b, 2, None, {"stoprule": {"type": "ME", "taudelta": 1.0}})
    with pytest.raises(ValueError, match="SIRT method not defined"):
        airt.sirt("nosuch", A, b, 5)
    with pytest.raises(ValueError, match="res_dims must be specified"):
        airt.cimmino(A, b, 5, None, {"stoprule": {"type": "NCP"}})
    with pytest.raises(ValueError, match="RESHAPE"):
        airt.cimmino(A, b, 5, None, {"stoprule": {"type": "NCP", "res_dims": [90, 180]}})
    with pytest.raises(ValueError, match="1D and 2D"):
        airt.cimmino(A, b, 5, None, {"stoprule": {"type": "NCP", "res_dims": [91, 90, 2]}})
    with pytest.warns(UserWarning, match="ncp_smooth"):
        airt.cimmino(A, b, 2, None, {"stoprule": {"type": "NONE", "ncp_smooth": 3}})


# ------------------------------------------------------------ ART
@pytest.fixture(scope="module")
def small():
    g = np.load(os.path.join(GOLD, "paralleltomo_N16_30ang.npz"))
    A_ref = sp.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=tuple(g["shape"]))
    return airt.afun_matrix(A_ref), A_ref, g["b"]


def test_golden_sirt_and_kaczmarz(small):
    A, A_ref, b = small
    s = np.load(os.path.join(GOLD, "solvers_N16_30ang.npz"))
    for meth in ("landweber", "cimmino", "cav", "drop", "sart"):
        X, _ = airt.sirt(meth, A, b, [5, 20], None,
                         {"lbound": 0.0, "ubound": 1.0, "rho": float(s[meth + "_rho"])})
        assert relerr(X, s[meth + "_X"]) <= RTOL
    X, info = airt.kaczmarz(A, b, [2, 5], None, {"lbound": 0.0})
    assert relerr(X, s["kaczmarz_X"]) <= RTOL
    X, info = airt.symkaczmarz(A, b, [4])
    assert relerr(X, s["symkaczmarz_X"]) <= RTOL and info["finaliter"] == 4


@pytest.mark.parametrize("method", ["kaczmarz", "symkaczmarz"])
def test_art_vs_oracle_with_options(small, method):
    A, A_ref, b = small
    opts = {"lbound": 0.0, "ubound": 0.6, "damp": 0.05, "relaxpar": 0.8}
    K = [2, 4, 6]
    Xo, io = O.art(method, A_ref, b, K, 0.3 * np.ones(A.n), opts)
    X, info = airt.art(method, A, b, K, 0.3 * np.ones(A.n), opts)
    assert relerr(X, Xo) <= RTOL
    assert info["finaliter"] == io["finaliter"] and list(info["itersaved"]) == list(io["itersaved"])


def test_art_custom_order_and_lambda_handle(small):
    A, A_ref, b = small
    order = np.arange(A.m)[::-1]
    lam = lambda j: 1.0 / np.sqrt(j) + 0.5  # noqa: E731
    Xo, io = O.art(order, A_ref, b, [3], options={"relaxpar": lam})
    X, info = airt.art(order, A, b, [3], None, {"relaxpar": lam})
    assert relerr(X, Xo) <= RTOL
    rn = np.asarray(A_ref.multiply(A_ref).sum(axis=1)).ravel()
    last = order[rn[order] > 0][-1]
    assert abs(info["relaxpar"] - lam(2 * A.m + int(last) + 1)) <= 1e-15


def test_randkaczmarz_stream(small):
    A, A_ref, b = small
    rn = np.asarray(A_ref.multiply(A_ref).sum(axis=1)).ravel()
    stream = O.RandStream(21)
    I = np.flatnonzero(rn > 0)
    rows = np.stack([O.art_sweep_rows(I, rn, True, stream, A.m)[0] for _ in range(4)])
    Xo = np.zeros(A.n)
    for k in range(4):
        Xo, _ = O.art(rows[k], A_ref, b, [1], Xo)
        Xo = Xo[:, 0]
    X, info = airt.randkaczmarz(A, b, [4], None, {"row_stream": rows})
    assert relerr(X[:, 0], Xo) <= RTOL


def test_art_dp_stop_c3_sized():
    """kaczmarz on N=64 with the DP rule, compared sweep by sweep."""
    A_ref = O.paralleltomo_matrix(64, np.arange(0.0, 180.0, 2.0))
    A = airt.afun_matrix(A_ref)
    b, enorm = airt.add_noise(A_ref @ O.shepplogan(64), 0.02, seed=2)
    opts = {"stoprule": {"type": "DP", "taudelta": 1.5 * enorm}}
    Xo, io = O.art("kaczmarz", A_ref, b, list(range(1, 11)), None, opts)
    X, info = airt.kaczmarz(A, b, list(range(1, 11)), None, opts)
    assert info["finaliter"] == io["finaliter"] and info["stoprule"] == io["stoprule"]
    for k in range(X.shape[1]):
        assert relerr(X[:, k], Xo[:, k]) <= RTOL


@pytest.fixture(scope="module")
def c3art():
    """C3-ART: paralleltomo N=256, 180 angles, p=362 (m=65,160, n=65,536), a
    10-ellipse phantom with 1% noise; the FP64 CSR from the C tracer."""
    theta = np.arange(180.0)
    th, p, d, ct, st, off = O.parallel_geometry(256, theta, None)
    rows, cols, vals = cbind.trace_coo(256, list(O.parallel_rays(256, ct, st, off)), True)
    Rm = O.coo_to_csc(rows, cols, vals, len(th) * p, 256 * 256).tocsr()
    A, *_ = airt.paralleltomo(256, theta)
    x = airt.random_ellipses(256, 10, seed=31)
    b, _ = airt.add_noise(Rm @ x, 0.01, seed=32)
    nrm = np.asarray(Rm.multiply(Rm).sum(axis=1)).ravel()
    return A, Rm, b, nrm


@pytest.mark.parametrize("method", ["kaczmarz", "symkaczmarz"])
def test_art_c3_sized_iterate_by_iterate(c3art, method):
    """20 sweeps of kaczmarz / symkaczmarz (art.m:188-191 row orders, the
    last row of the symmetric sweep applied twice) against the C oracle,
    every sweep's iterate within 1e-5."""
    A, Rm, b, nrm = c3art
    I = np.flatnonzero(nrm > 0)
    order = I if method == "kaczmarz" else np.concatenate([I, I[::-1]])
    K = list(range(1, 21)) if method == "kaczmarz" else list(range(2, 21, 2))
    X, info = getattr(airt, method)(A, b, K, None, {"lbound": 0.0})
    assert info["finaliter"] == 20 and X.shape[1] == len(K)
    x = np.zeros(A.n)
    for j in range(len(K)):
        x = cbind.kaczmarz(Rm, b, nrm, order, 1.0, 0.0, None, 1, x0=x)
        assert relerr(X[:, j], x) <= RTOL, (method, K[j], relerr(X[:, j], x))


# ------------------------------------------------------------ CART
def _f32(A):
    """A with its values rounded to FP32, as the GPU stores them: the CART
    oracle runs on it so that both sides take the same flagging decisions."""
    R = sp.csc_matrix(A, copy=True)
    R.data = R.data.astype(np.float32).astype(np.float64)
    return R


CART_TOL = 1e-9


@pytest.mark.parametrize("opts", [
    {},
    {"lbound": 0.0, "ubound": 1.0, "relaxpar": 0.5, "Kbegin": 2, "Nunflag": 2, "THR": 5e-3},
    {"damp": 0.1, "relaxpar": 1.2, "Kbegin": 1, "Nunflag": 3, "THR": 2e-2, "seed": 7},
])
def test_cart_vs_oracle(small, opts):
    """cart.m columnaction: saved iterates, finaliter and itersaved against
    the oracle, with flagging and unflagging active in the last two cases."""
    A, A_ref, b = small
    K = [1, 3, 8, 15]
    Xo, io = O.cart("columnaction", _f32(A_ref), b, K, None, opts)
    X, info = airt.columnaction(A, b, K, None, opts)
    assert X.shape == Xo.shape
    assert relerr(X, Xo) <= CART_TOL
    assert info["finaliter"] == io["finaliter"] == 15
    assert list(info["itersaved"]) == list(io["itersaved"])
    assert info["relaxpar"] == opts.get("relaxpar", 0.25)


def test_cart_running_max_rescans(small):
    """x0 above the upper bound: the clipped steps keep lowering the entry
    that holds max(abs(x)), and with THR = 0.05 from the first sweep on the
    flag of every column depends on that maximum before its step."""
    A, A_ref, b = small
    x0 = np.random.default_rng(5).uniform(0.0, 3.0, A.n)
    opts = {"lbound": 0.0, "ubound": 1.0, "Kbegin": 1, "THR": 0.05, "Nunflag": 2, "seed": 3}
    K = list(range(1, 7))
    Xo, _ = O.cart("columnaction", _f32(A_ref), b, K, x0, opts)
    X, _ = airt.columnaction(A, b, K, x0, opts)
    for j in range(len(K)):
        assert relerr(X[:, j], Xo[:, j]) <= CART_TOL, (K[j], relerr(X[:, j], Xo[:, j]))


def test_cart_custom_order_and_stop_rules(small, c1):
    A, A_ref, b = small
    n = A.n
    order = np.concatenate([np.arange(n)[::-1], np.arange(12), [5, 5, 7]])
    opts = {"Kbegin": 2, "Nunflag": 2, "THR": 1e-2}
    Xo, io = O.cart(order, _f32(A_ref), b, [2, 6], None, opts)
    X, info = airt.cart(order, A, b, [2, 6], None, opts)
    assert relerr(X, Xo) <= CART_TOL
    # DP: stop at the sweep whose residual first falls below taudelta
    Ac, Ac_ref, bc, enorm, _ = c1
    tau = 1.02 * enorm
    dp = {"stoprule": {"type": "DP", "taudelta": tau}}
    Xo, io = O.cart(None, _f32(Ac_ref), bc, 60, None, dp)
    X, info = airt.cart(None, Ac, bc, 60, None, dp)
    assert info["finaliter"] == io["finaliter"] and info["stoprule"] == io["stoprule"]
    assert relerr(X, Xo) <= CART_TOL
    assert info["resnorms"][-1] <= tau < info["resnorms"][-2] or info["finaliter"] == 60
    # NCP on the projections (res_dims = [rays, angles])
    ncp = {"stoprule": {"type": "NCP", "res_dims": [91, 180]}}
    Xo, io = O.cart("columnaction", _f32(Ac_ref), bc, 40, None, ncp)
    X, info = airt.columnaction(Ac, bc, 40, None, ncp)
    assert info["finaliter"] == io["finaliter"] and info["stoprule"] == io["stoprule"]
    assert relerr(X, Xo) <= CART_TOL


def test_cart_input_errors(small):
    A, A_ref, b = small
    with pytest.raises(ValueError):
        airt.cart("rowaction", A, b, 2)
    with pytest.raises(ValueError):
        airt.columnaction(A, b, 2, None, {"relaxpar": lambda k: 0.5})
    with pytest.raises(ValueError):
        airt.columnaction(A, b, 2, None, {"stoprule": {"type": "ME", "taudelta": 1.0}})
    Amf, *_ = airt.paralleltomo(16, np.arange(0.0, 180.0, 6.0), None, None, 0, 0)
    with pytest.raises(airt.AirtError):
        airt.columnaction(Amf, Amf(np.ones(256), "notransp"), 2)


# ------------------------------------------------------------ fbp
@pytest.mark.parametrize("filt", ["ram-lak", "shepp-logan", "cosine", "hamming", "hann", "none"])
def test_fbp_vs_oracle(c1, filt):
    """auxil/fbp.m: the FP64 direct convolution with real(ifft(filter)) on the
    GPU against the oracle's zero-pad / FFT / filter / IFFT / crop, both with
    the FP32-rounded matrix."""
    A, A_ref, b, _, x = c1
    theta = np.arange(0.0, 180.0, 1.0)
    xo = O.fbp(_f32(A_ref), b, theta, filt)
    xg = airt.fbp(A, b, theta, filt)
    assert relerr(xg, xo) <= 1e-10
    if filt == "ram-lak":
        assert relerr(xg, x) < 0.5           # a usable reconstruction of the phantom


def test_fbp_matrix_free_and_batch():
    import torch
    theta = np.arange(0.0, 180.0, 3.0)
    A, b, x, *_ = airt.paralleltomo(48, theta)
    Amf, *_ = airt.paralleltomo(48, theta, None, None, 0, 0)
    xs = airt.fbp(A, b, theta, "hamming")
    assert relerr(airt.fbp(Amf, b, theta, "hamming"), xs) <= 1e-10
    with pytest.raises(ValueError):
        airt.fbp(A, b, theta, "bogus")
    # a batch of instances with the same rays and different angle sets
    thetas = [theta, np.arange(0.0, 180.0, 5.0), np.arange(10.0, 170.0, 4.0)]
    Bt = airt.ParallelBatch([48] * 3, thetas)
    bs = []
    for th in thetas:
        Ak, bk, *_ = airt.paralleltomo(48, th)
        bs.append(bk)
    db = torch.from_numpy(np.concatenate(bs)).cuda()
    dx = torch.empty(Bt.n, dtype=torch.float64, device="cuda")
    Bt.fbp_device(db.data_ptr(), dx.data_ptr(), "hamming")
    got = Bt.split_cols(dx.cpu().numpy())
    for k, th in enumerate(thetas):
        Ak, *_ = airt.paralleltomo(48, th)
        assert relerr(got[k], airt.fbp(Ak, bs[k], th, "hamming")) <= 1e-10


def test_cart_residual_in_global_memory():
    """N=128, 180 angles: a residual of 32,580 rows does not fit in shared
    memory, so the sweep runs on the 256-thread CTA kernel; flagging and
    unflagging active."""
    theta = np.arange(0.0, 180.0, 1.0)
    A_ref = O.paralleltomo_matrix(128, theta)
    A, *_ = airt.paralleltomo(128, theta)
    assert A.m == 32580
    x = airt.random_ellipses(128, 8, seed=5)
    b = A_ref @ x
    opts = {"lbound": 0.0, "Kbegin": 2, "Nunflag": 2, "THR": 1e-2}
    Xo, io = O.cart("columnaction", _f32(A_ref), b, [2, 4], None, opts)
    X, info = airt.columnaction(A, b, [2, 4], None, opts)
    assert relerr(X, Xo) <= CART_TOL
    assert info["finaliter"] == io["finaliter"] == 4


@pytest.mark.gpu
@pytest.mark.parametrize("geo", ["parallel_c2", "parallel_odd", "fan", "seismic"])
def test_split_trace_has_the_whole_trace_entries(geo):
    """The matrix-free kernels trace a long ray on two threads, each from one
    side of a clean crossing near its middle.  For every ray, the union of
    the two halves' merged entries must be the whole trace's entries, pixel
    and FP64 value bits (count plus an order-independent hash), and most
    long rays must actually be split."""
    import ctypes as C
    from airtoolsii_b200._lib import lib
    if geo == "parallel_c2":
        A, *_ = airt.paralleltomo(512, np.arange(360) * 0.5, 724, None, 0, 0)
    elif geo == "parallel_odd":
        A, *_ = airt.paralleltomo(255, np.arange(0.0, 180.0, 0.7), 301, None, 0, 0)
    elif geo == "fan":
        A, *_ = airt.fanlineartomo(384, np.arange(0.0, 360.0, 1.0), None, None, None, None, 0, 0)
    else:
        A, *_ = airt.seismictomo(256, None, None, 0, 0)
    bad, split = C.c_int64(-1), C.c_int64(0)
    assert lib().airt_test_split_trace(A.handle, C.byref(bad), C.byref(split)) == 0
    assert bad.value == 0
    assert split.value > A.m // 2, (split.value, A.m)
