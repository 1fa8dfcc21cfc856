"""CPU tests of the FP64 oracle: golden fixtures, analytic known answers of
the ray tracer, agreement of the NumPy and C restatements, and the reference
demos' invariants (demos/demo_matrixfree.m, demos/demo_custom_all.m,
demos/demo_constraints.m)."""
import math
import os

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import airt_oracle as O
from oracle import cbind

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _load(name):
    return np.load(os.path.join(GOLD, name))


# ---------------------------------------------------------------- golden
def test_golden_paralleltomo_matrix():
    g = _load("paralleltomo_N16_30ang.npz")
    A = O.paralleltomo_matrix(16, g["theta"])
    assert np.array_equal(A.indptr, g["indptr"])
    assert np.array_equal(A.indices, g["indices"])
    assert np.array_equal(A.data, g["data"])
    assert np.array_equal(O.shepplogan(16), g["x"])


def test_golden_fanlineartomo_matrix():
    g = _load("fanlineartomo_N12_30ang.npz")
    F = O.fanlineartomo_matrix(12, np.arange(0.0, 360.0, 12.0), 17)
    assert np.array_equal(F.indptr, g["indptr"])
    assert np.array_equal(F.indices, g["indices"])
    assert np.array_equal(F.data, g["data"])


def test_golden_widened():
    """widened_N16.npz: seismictomo and sphericaltomo matrices, CART and fbp
    on the N=16 problem (FP32-rounded values) reproduce exactly."""
    g = _load("paralleltomo_N16_30ang.npz")
    w = _load("widened_N16.npz")
    S = O.seismictomo_matrix(12, 6, 10)
    Q = O.sphericaltomo_matrix(10, np.arange(0.0, 360.0, 30.0), 8)
    for M, k in ((S, "seis"), (Q, "sph")):
        assert np.array_equal(M.indptr, w[k + "_indptr"])
        assert np.array_equal(M.indices, w[k + "_indices"])
        assert np.array_equal(M.data, w[k + "_data"])
    R = sp.csc_matrix((g["data"].astype(np.float32).astype(np.float64), g["indices"], g["indptr"]),
                      shape=tuple(g["shape"]))
    opts = {"lbound": 0.0, "Kbegin": 2, "Nunflag": 2, "THR": 1e-2, "seed": 5}
    Xc, ic = O.cart("columnaction", R, g["b"], [2, 6], None, opts)
    np.testing.assert_allclose(Xc, w["cart_X"], rtol=1e-12, atol=1e-13)
    assert ic["finaliter"] == int(w["cart_finaliter"])
    np.testing.assert_allclose(O.fbp(R, g["b"], g["theta"], "hamming"), w["fbp_hamming"], rtol=1e-12)
    np.testing.assert_allclose(O.fbp(R, g["b"], g["theta"], "ram-lak"), w["fbp_ramlak"], rtol=1e-12)


def test_golden_solvers():
    g = _load("paralleltomo_N16_30ang.npz")
    s = _load("solvers_N16_30ang.npz")
    A = sp.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=tuple(g["shape"]))
    b = g["b"]
    for meth in ("landweber", "cimmino", "cav", "drop", "sart"):
        X, info, _ = O.sirt(meth, A, b, [5, 20], options={"lbound": 0.0, "ubound": 1.0,
                                                          "rho": float(s[meth + "_rho"])})
        np.testing.assert_allclose(X, s[meth + "_X"], rtol=1e-12, atol=1e-13)
    Xk, _ = O.art("kaczmarz", A, b, [2, 5], options={"lbound": 0.0})
    np.testing.assert_allclose(Xk, s["kaczmarz_X"], rtol=1e-12, atol=1e-13)


# ---------------------------------------------------------------- tracer KATs
def _trace(N, theta, offsets):
    ct, st = O.cosd(theta), O.sind(theta)
    rows, cols, vals = O.trace_coo(N, O.parallel_rays(N, ct, st, np.asarray(offsets, float)), True)
    return O.coo_to_csc(rows, cols, vals, len(theta) * len(offsets), N * N).tocsr()


def test_axis_aligned_rays_have_unit_lengths():
    N = 6
    offs = np.arange(N) - (N - 1) / 2.0          # pixel centres
    for th in (0.0, 90.0, 180.0, 270.0):
        A = _trace(N, [th], offs)
        for r in range(N):
            row = A.getrow(r)
            assert row.nnz == N
            np.testing.assert_array_equal(row.data, np.ones(N))
    # theta = 0 is a vertical ray: the pixels of one image column (column-major)
    A = _trace(N, [0.0], offs)
    assert sorted(A.getrow(0).indices) == list(range(0, N))


def test_diagonal_ray_through_corners():
    N = 8
    A = _trace(N, [45.0], [0.0])
    row = A.getrow(0)
    assert row.nnz == N                          # corner points merged (1e-10 rule)
    np.testing.assert_allclose(row.data, math.sqrt(2.0), rtol=0, atol=1e-12)


def test_boundary_ray_exclusion():
    """paralleltomo.m:255-256: a ray on the top/right edge is dropped, the
    bottom/left edge is kept."""
    N = 4
    A = _trace(N, [0.0, 90.0], [-2.0, 2.0])
    nnz = np.diff(A.indptr)
    assert list(nnz) == [4, 0, 4, 0]


def _chord(N, x0, y0, a, b):
    h = N / 2.0
    lo, hi = -np.inf, np.inf
    for p, d in ((x0, a), (y0, b)):
        if d == 0:
            if not (-h <= p <= h):
                return 0.0
            continue
        t1, t2 = (-h - p) / d, (h - p) / d
        lo, hi = max(lo, min(t1, t2)), min(hi, max(t1, t2))
    return max(0.0, hi - lo) * math.hypot(a, b)


def test_row_sums_equal_chord_lengths():
    rng = np.random.default_rng(7)
    N = 20
    theta = rng.uniform(0, 360, 25)
    offs = rng.uniform(-14, 14, 9)
    A = _trace(N, theta, offs)
    sums = np.asarray(A.sum(axis=1)).ravel()
    ct, st = O.cosd(theta), O.sind(theta)
    for r, x0t, y0t, a, b in O.parallel_rays(N, ct, st, offs):
        assert abs(sums[r] - _chord(N, x0t, y0t, a, b)) <= 1e-9


def test_fan_rows_pass_through_source():
    N = 10
    th, p, R, _, _, ct, st, cw, sw = O.fan_geometry(N, np.arange(0.0, 360.0, 30.0), 15)
    rays = list(O.fan_rays(N, R, ct, st, cw, sw))
    rows, cols, vals = O.trace_coo(N, rays, False)
    A = O.coo_to_csc(rows, cols, vals, len(th) * p, N * N).tocsr()
    sums = np.asarray(A.sum(axis=1)).ravel()
    for r, x0t, y0t, a, b in rays:
        assert abs(math.hypot(x0t, y0t) - R) < 1e-9
        assert abs(sums[r] - _chord(N, x0t, y0t, a, b)) <= 1e-9


def test_trig_tables_exact_at_right_angles():
    th = np.array([0, 90, 180, 270, 360, -90, 450], float)
    np.testing.assert_array_equal(O.cosd(th), [1, 0, -1, 0, 1, 0, 0])
    np.testing.assert_array_equal(O.sind(th), [0, 1, 0, -1, 0, -1, 1])
    np.testing.assert_allclose(O.cosd([30.0, 60.0, 1.5]), np.cos(np.deg2rad([30, 60, 1.5])),
                               rtol=1e-15)


# ---------------------------------------------------------------- NumPy vs C
@pytest.mark.parametrize("N,theta,p,d", [
    (64, None, None, None),
    (15, np.arange(0.0, 180.0, 7.5), 21, 18.5),
    (12, np.array([0, 45, 90, 135, 180, 225, 270, 315.0]), 17, None),
])
def test_c_tracer_matches_numpy_parallel(N, theta, p, d):
    th, p_, d_, ct, st, off = O.parallel_geometry(N, theta, p, d)
    rays = list(O.parallel_rays(N, ct, st, off))
    A1 = O.coo_to_csc(*cbind.trace_coo(N, rays, True), len(th) * p_, N * N)
    A0 = O.coo_to_csc(*O.trace_coo(N, rays, True), len(th) * p_, N * N)
    assert np.array_equal(A1.indptr, A0.indptr)
    assert np.array_equal(A1.indices, A0.indices)
    assert np.array_equal(A1.data, A0.data)


def test_c1_config_size():
    """The CPU-runnable configuration: N=64, 180 angles, p=91 (16380 x 4096)."""
    th, p, d, ct, st, off = O.parallel_geometry(64)
    rows, cols, vals = cbind.trace_coo(64, list(O.parallel_rays(64, ct, st, off)), True)
    A = O.coo_to_csc(rows, cols, vals, len(th) * p, 64 * 64)
    assert A.shape == (16380, 4096)
    assert A.nnz == 938572
    assert int((np.diff(A.tocsr().indptr) == 0).sum()) == 1694


def test_c_tracer_matches_numpy_fan():
    N = 24
    th, p, R, _, _, ct, st, cw, sw = O.fan_geometry(N, np.arange(0.0, 360.0, 10.0))
    rays = list(O.fan_rays(N, R, ct, st, cw, sw))
    A1 = O.coo_to_csc(*cbind.trace_coo(N, rays, False), len(th) * p, N * N)
    A0 = O.coo_to_csc(*O.trace_coo(N, rays, False), len(th) * p, N * N)
    assert (A1 != A0).nnz == 0


@pytest.mark.parametrize("N,s,p", [(24, None, None), (17, 5, 9), (10, 1, 1)])
def test_c_tracer_matches_numpy_seismic(N, s, p):
    """seismictomo rays include horizontal ones (b = 0, all y-crossings at
    t = +-inf) whenever a left-edge receiver sits level with a source."""
    s_, p_, x0, y0, xp, yp = O.seismic_geometry(N, s, p)
    rays = list(O.seismic_rays(x0, y0, xp, yp))
    A1 = O.coo_to_csc(*cbind.trace_coo(N, rays, False), s_ * p_, N * N)
    A0 = O.coo_to_csc(*O.trace_coo(N, rays, False), s_ * p_, N * N)
    assert (A1 != A0).nnz == 0
    assert np.array_equal(A1.indices, A0.indices)


def test_seismic_rows_are_source_receiver_distances():
    """Sources and receivers lie on the boundary, so the traced length of
    every ray is the source-receiver distance."""
    N = 16
    s, p, x0, y0, xp, yp = O.seismic_geometry(N)
    assert (s, p) == (16, 32)
    rays = list(O.seismic_rays(x0, y0, xp, yp))
    assert sum(1 for r in rays if r[4] == 0.0) == 16      # one level receiver per source
    A = O.seismictomo_matrix(N).tocsr()
    sums = np.asarray(A.sum(axis=1)).ravel()
    for r, x0t, y0t, a, b in rays:
        assert abs(sums[r] - math.hypot(a, b)) <= 1e-9


def test_sphere_rows_count_in_image_samples():
    """Every sample of a circle that lands in the image adds 2*pi*r/nPhi to its
    row (sphericaltomo.m:224-234): the row sum is that times the number of
    in-image samples, counted here with scalar MATLAB rounding."""
    N = 12
    angles = np.array([0.0, 90.0, 225.0])
    A = O.sphericaltomo_matrix(N, angles).tocsr()
    ang, nc, radii, nphi, dphi, center, dx = O.sphere_geometry(N, angles)
    ck, sk = O.sphere_circle_tables(nphi, dphi)
    off = np.concatenate([[0], np.cumsum(nphi + 1)])
    sums = np.asarray(A.sum(axis=1)).ravel()
    for m, a in enumerate(ang):
        xc, yc = O.cosd(a)[0], O.sind(a)[0]
        for n in range(nc):
            hits = 0
            for k in range(off[n], off[n + 1]):
                col = O.mround((xc + radii[n] * ck[k]) / dx + center)
                row = O.mround((yc + radii[n] * sk[k]) / dx + center)
                hits += (1 <= col <= N) and (1 <= row <= N)
            want = (2 * math.pi * radii[n] / nphi[n]) * hits
            assert abs(sums[m * nc + n] - want) <= 1e-12 * max(1.0, want)
    assert A.nnz > 0 and np.all(A.data > 0)


def test_cart_diagonal_known_answer():
    """For a diagonal A, one columnaction sweep with relaxpar 1 solves A x = b
    exactly (each column's step is b_j/a_jj), and the box clips it."""
    d = np.array([2.0, 0.5, 4.0, 1.0, 8.0])
    b = np.array([1.0, -3.0, 2.0, 5.0, 0.25])
    A = sp.diags(d).tocsc()
    X, info = O.cart("columnaction", A, b, [1, 2], None, {"relaxpar": 1.0})
    np.testing.assert_array_equal(X[:, 0], b / d)
    np.testing.assert_array_equal(X[:, 1], b / d)
    assert info["finaliter"] == 2
    X, _ = O.cart("columnaction", A, b, [1], None, {"relaxpar": 1.0, "lbound": 0.0, "ubound": 2.0})
    np.testing.assert_array_equal(X[:, 0], np.clip(b / d, 0.0, 2.0))


def test_cart_randi_draws():
    draws = [O.cart_randi(11, k, j, 4) for k in range(1, 50) for j in range(40)]
    assert min(draws) == 1 and max(draws) == 4
    assert draws == [O.cart_randi(11, k, j, 4) for k in range(1, 50) for j in range(40)]
    counts = np.bincount(draws)[1:]
    assert np.all(np.abs(counts / len(draws) - 0.25) < 0.03)
    assert O.cart_randi(11, 1, 0, 1) == 1


# ---------------------------------------------------------------- invariants
@pytest.fixture(scope="module")
def small():
    g = _load("paralleltomo_N16_30ang.npz")
    A = sp.csc_matrix((g["data"], g["indices"], g["indptr"]), shape=tuple(g["shape"]))
    return A, g["b"], g["theta"]


def test_matrix_free_equals_matrix(small):
    A, b, theta = small
    ct, st = O.cosd(theta), O.sind(theta)
    th, p, d, _, _, off = O.parallel_geometry(16, theta)
    rng = np.random.default_rng(0)
    x = rng.random(A.shape[1])
    y = rng.random(A.shape[0])
    rays = list(O.parallel_rays(16, ct, st, off))
    np.testing.assert_allclose(O.matrixfree_apply(16, rays, True, A.shape[0], x, False), A @ x,
                               rtol=1e-13)
    np.testing.assert_allclose(O.matrixfree_apply(16, rays, True, A.shape[0], y, True), A.T @ y,
                               rtol=1e-13)


def test_custom_empty_struct_is_landweber(small):
    A, b, _ = small
    X1, _, _ = O.sirt("landweber", A, b, [10], options={"rho": 100.0})
    X2, _, _ = O.sirt({}, A, b, [10], options={"rho": 100.0})
    np.testing.assert_array_equal(X1, X2)


def test_scaled_custom_is_cimmino(small):
    A, b, _ = small
    m = A.shape[0]
    rn = np.asarray(A.multiply(A).sum(axis=1)).ravel()
    Mc = np.where(rn > 0, 1.0 / np.where(rn > 0, rn, 1), 0.0)
    X1, i1, _ = O.sirt("cimmino", A, b, [15])
    X2, _, _ = O.sirt({"M": Mc}, A, b, [15], options={"rho": i1["rho"] * m})
    np.testing.assert_allclose(X1, X2, rtol=1e-10, atol=1e-12)


def test_constraints_hold(small):
    A, b, _ = small
    X, _, _ = O.sirt("sart", A, b, list(range(1, 11)), options={"lbound": 0.1, "ubound": 0.8})
    assert X.min() >= 0.1 and X.max() <= 0.8
    Xa, _ = O.art("kaczmarz", A, b, [1, 2, 3], options={"lbound": 0.0, "ubound": 0.5})
    assert Xa.min() >= 0.0 and Xa.max() <= 0.5


def test_dp_stop_at_k0_returns_empty(small):
    A, b, _ = small
    X, info, _ = O.sirt("cimmino", A, b, [10], options={"stoprule": {"type": "DP", "taudelta": 1e9}})
    assert X.shape[1] == 0 and info["finaliter"] == 0 and list(info["itersaved"]) == [0]


def test_c_sirt_matches_numpy(small):
    A, b, _ = small
    M, D, _, _ = O.get_mfun_dfun("sart", A)
    X, info, _ = O.sirt("sart", A, b, [12], options={"lbound": 0.0})
    x, k, _ = cbind.sirt_csr(A, b, M, D, info["relaxpar"], 0.0, None, None, 12)
    assert k == 12
    np.testing.assert_allclose(x, X[:, -1], rtol=1e-11, atol=1e-13)


def test_c_kaczmarz_matches_numpy(small):
    A, b, _ = small
    Acsr = A.tocsr()
    nrm = np.asarray(Acsr.multiply(Acsr).sum(axis=1)).ravel()
    rows = np.flatnonzero(nrm > 0)
    Xo, _ = O.art("kaczmarz", A, b, [3], options={"lbound": 0.0, "ubound": 0.9})
    x = cbind.kaczmarz(A, b, nrm, rows, 1.0, 0.0, 0.9, 3)
    np.testing.assert_allclose(x, Xo[:, -1], rtol=1e-11, atol=1e-13)


def test_calczeta_roots():
    z = O.calczeta(np.arange(2, 30))
    k = np.arange(2, 30)
    g = (2 * k - 1) * z ** (k - 1) - np.array([np.sum(zz ** np.arange(kk - 1)) for zz, kk in zip(z, k)])
    assert np.max(np.abs(g)) < 1e-10


def test_unet_oracle_gradient_matches_finite_differences():
    """The NumPy U-Net used as the GPU gradient checker, without BF16 rounding,
    against central differences on random parameters."""
    from oracle import unet_oracle as UO
    base, levels, H, W = 8, 2, 8, 8
    n = sum(co * 9 * ci + co for ci, co in UO.layer_shapes(base, levels)) + base + 1
    rng = np.random.default_rng(4)
    p = rng.standard_normal(n) * 0.3
    x = rng.random((2, H * W))
    t = rng.random((2, H * W))
    UO.EXACT = True
    try:
        _, g, _ = UO.forward_backward(p, x, t, base, levels, H, W)
        for i in rng.choice(n, 25, replace=False):
            e = np.zeros(n)
            e[i] = 1e-6
            lp, _, _ = UO.forward_backward(p + e, x, t, base, levels, H, W)
            lm, _, _ = UO.forward_backward(p - e, x, t, base, levels, H, W)
            fd = (lp - lm) / 2e-6
            assert abs(fd - g[i]) <= 1e-5 * max(1.0, abs(g[i])), (i, fd, g[i])
    finally:
        UO.EXACT = False
