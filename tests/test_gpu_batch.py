"""GPU tests of the batched solvers: every instance of an uneven batch
against the FP64 oracle run on that instance alone (relative iterate error
<= 1e-5, identical DP stopping iteration)."""
import numpy as np
import pytest

import airtoolsii_b200 as airt
from oracle import airt_oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.fixture(scope="module")
def batch():
    rng = np.random.default_rng(17)
    Ns = [16, 16, 24, 32, 32, 48]
    thetas = [np.sort(rng.choice(np.arange(0.0, 180.0, 1.0), size=int(rng.integers(12, 40)),
                                 replace=False)) for _ in Ns]
    B = airt.ParallelBatch(Ns, thetas)
    mats, bs, tds, xs = [], [], [], []
    for k, N in enumerate(Ns):
        A = O.paralleltomo_matrix(N, thetas[k])
        x = airt.random_ellipses(N, 6, seed=30 + k)
        eta = [0.005, 0.01, 0.02, 0.03, 0.01, 0.02][k]
        b, en = airt.add_noise(A @ x, eta, seed=60 + k)
        mats.append(A)
        bs.append(b)
        tds.append(1.02 * en)
        xs.append(x)
    return B, mats, bs, np.array(tds), xs


def test_batch_layout(batch):
    B, mats, *_ = batch
    assert B.K == len(mats)
    assert list(B.inst_nnz()) == [A.nnz for A in mats]
    for k, A in enumerate(mats):
        assert B.row_off[k + 1] - B.row_off[k] == A.shape[0]
        assert B.col_off[k + 1] - B.col_off[k] == A.shape[1]
    assert B.nnz == sum(A.nnz for A in mats)


@pytest.mark.parametrize("method", ["cimmino", "drop"])
def test_batch_rho(batch, method):
    B, mats, bs, _, _ = batch
    rho = B.rho(method)
    for k, A in enumerate(mats):
        _, io, _ = O.sirt(method, A, bs[k], [1])
        assert abs(rho[k] - io["rho"]) <= 1e-4 * io["rho"]


@pytest.mark.parametrize("method", ["cimmino", "drop", "sart"])
def test_batch_sirt_dp_per_instance(batch, method):
    B, mats, bs, tds, _ = batch
    rho = np.ones(B.K) if method == "sart" else B.rho(method)
    xs, info = B.sirt(method, bs, 400, taudelta=tds, rho=rho, lbound=0.0)
    for k, A in enumerate(mats):
        Xo, io, _ = O.sirt(method, A, bs[k], [400], options={
            "stoprule": {"type": "DP", "taudelta": tds[k]}, "rho": float(rho[k]), "lbound": 0.0})
        assert info["finaliter"][k] == io["finaliter"], (k, info["finaliter"][k], io["finaliter"])
        assert info["stoprule"][k] == io["stoprule"]
        assert relerr(xs[k], Xo[:, -1]) <= RTOL


@pytest.mark.parametrize("method", ["cimmino", "drop"])
def test_batch_sirt_me_per_instance(batch, method):
    """The ME rule (check_stoprules.m:74-94) applied per instance."""
    B, mats, bs, tds, _ = batch
    rho = B.rho(method)
    xs, info = B.sirt(method, bs, 400, taudelta=tds, rho=rho, lbound=0.0, stoprule="ME")
    for k, A in enumerate(mats):
        Xo, io, _ = O.sirt(method, A, bs[k], [400], options={
            "stoprule": {"type": "ME", "taudelta": tds[k]}, "rho": float(rho[k]), "lbound": 0.0})
        assert info["finaliter"][k] == io["finaliter"], (k, info["finaliter"][k], io["finaliter"])
        assert info["stoprule"][k] == io["stoprule"]
        assert relerr(xs[k], Xo[:, -1]) <= RTOL


@pytest.mark.parametrize("smooth", [1, 2, 4])
def test_batch_sirt_ncp_per_instance(batch, smooth):
    """The NCP rule (check_stoprules.m:96-151) per instance, each residual
    reshaped to its instance's p x nA projections."""
    B, mats, bs, _, _ = batch
    rho = B.rho("cimmino")
    xs, info = B.sirt("cimmino", bs, 300, rho=rho, stoprule="NCP", ncp_smooth=smooth)
    for k, A in enumerate(mats):
        Xo, io, _ = O.sirt("cimmino", A, bs[k], [300], options={
            "stoprule": {"type": "NCP", "res_dims": [B.ps[k], B.nAs[k]], "ncp_smooth": smooth},
            "rho": float(rho[k])})
        assert info["finaliter"][k] == io["finaliter"], (k, info["finaliter"][k], io["finaliter"])
        assert info["stoprule"][k] == io["stoprule"]
        assert relerr(xs[k], Xo[:, -1]) <= RTOL


def test_batch_sirt_fixed_iterations_box(batch):
    B, mats, bs, _, _ = batch
    rho = B.rho("cimmino")
    xs, info = B.sirt("cimmino", bs, 25, rho=rho, lbound=0.0, ubound=0.7)
    assert np.all(info["finaliter"] == 25)
    for k, A in enumerate(mats):
        Xo, _, _ = O.sirt("cimmino", A, bs[k], [25], options={"rho": float(rho[k]),
                                                               "lbound": 0.0, "ubound": 0.7})
        assert relerr(xs[k], Xo[:, -1]) <= RTOL


def test_batch_kaczmarz(batch):
    B, mats, bs, _, _ = batch
    xs, _ = B.kaczmarz(bs, 3, 1.0, lbound=0.0)
    for k, A in enumerate(mats):
        Xo, _ = O.art("kaczmarz", A, bs[k], [3], options={"lbound": 0.0})
        assert relerr(xs[k], Xo[:, -1]) <= RTOL


@pytest.mark.parametrize("method", ["sart", "cimmino"])
def test_batch_backproject_is_first_sirt_iterate(batch, method):
    """airt_batch_backproject equals a one-iteration batched SIRT call from
    zero with relaxpar 1 bit for bit, and the oracle's first iterate."""
    import torch
    B, mats, bs, _, _ = batch
    b = np.concatenate(bs)
    xs, _ = B.sirt(method, b, 1, relaxpar=1.0)
    db = torch.from_numpy(b).cuda()
    dx = torch.full((B.n,), float("nan"), dtype=torch.float64, device="cuda")
    for _ in range(2):  # the second call reuses the cached weights
        B.backproject_device(method, db.data_ptr(), dx.data_ptr())
        torch.cuda.synchronize()
        got = B.split_cols(dx.cpu().numpy())
        for k, A in enumerate(mats):
            assert np.array_equal(got[k], xs[k])
            Xo, _, _ = O.sirt(method, A, bs[k], [1], options={"relaxpar": 1.0})
            assert relerr(got[k], Xo[:, -1]) <= RTOL


def test_batch_apply_matches_instances(batch):
    import torch
    B, mats, _, _, xs = batch
    x = np.concatenate(xs)
    y = np.concatenate([rng_vec(A.shape[0], k) for k, A in enumerate(mats)])
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    out_f = torch.empty(B.m, dtype=torch.float64, device="cuda")
    out_t = torch.empty(B.n, dtype=torch.float64, device="cuda")
    B.apply_device(dx.data_ptr(), out_f.data_ptr(), False)
    B.apply_device(dy.data_ptr(), out_t.data_ptr(), True)
    f, t = B.split_rows(out_f.cpu().numpy()), B.split_cols(out_t.cpu().numpy())
    for k, A in enumerate(mats):
        assert relerr(f[k], A @ xs[k]) <= 1e-6
        assert relerr(t[k], A.T @ B.split_rows(y)[k]) <= 1e-6


def rng_vec(n, seed):
    return np.random.default_rng(900 + seed).standard_normal(n)


@pytest.mark.parametrize("method,K", [("cimmino", 7), ("sart", 40), ("drop", 300)])
def test_sirt_multi_rhs_vs_oracle(method, K):
    """SIRT on K right-hand sides of one matrix (interleaved iterates, A read
    once per iteration; K = 300 runs as two passes of at most 256) against the
    oracle run per right-hand side: per-instance DP stop and iterate."""
    import torch
    from airtoolsii_b200.batch import sirt_multi_device
    N, theta = 32, np.arange(0.0, 180.0, 6.0)
    A = O.paralleltomo_matrix(N, theta)
    op = airt.afun_matrix(A)
    xs = [airt.random_ellipses(N, 5, seed=700 + k) for k in range(K)]
    bs, tds = [], []
    for k in range(K):
        b, en = airt.add_noise(A @ xs[k], 0.01 + 0.02 * (k % 3), seed=900 + k)
        bs.append(b)
        tds.append(1.02 * en)
    dB = torch.from_numpy(np.stack(bs)).cuda()
    dX = torch.empty((K, A.shape[1]), dtype=torch.float64, device="cuda")
    rho = 1.0 if method == "sart" else O.sirt(method, A, bs[0], [1])[1]["rho"]
    info = sirt_multi_device(op, method, dB.data_ptr(), dX.data_ptr(), K, 500, taudelta=tds,
                             rho=rho, lbound=0.0)
    X = dX.cpu().numpy()
    for k in range(0, K, max(1, K // 12)):
        Xo, io, _ = O.sirt(method, A, bs[k], [500], options={
            "stoprule": {"type": "DP", "taudelta": tds[k]}, "rho": rho, "lbound": 0.0})
        assert info["finaliter"][k] == io["finaliter"], (k, info["finaliter"][k], io["finaliter"])
        assert info["stoprule"][k] == io["stoprule"]
        assert relerr(X[k], Xo[:, -1]) <= RTOL
    # fixed iteration count from a given x0, box [0, 1]
    dX0 = torch.from_numpy(np.stack(xs)).cuda() * 0.5
    info = sirt_multi_device(op, method, dB.data_ptr(), dX.data_ptr(), K, 7, rho=rho,
                             d_X0=dX0.data_ptr(), lbound=0.0, ubound=1.0)
    assert np.all(info["finaliter"] == 7)
    X = dX.cpu().numpy()
    for k in (0, K - 1):
        Xo, _, _ = O.sirt(method, A, bs[k], [7], 0.5 * xs[k], {"rho": rho, "lbound": 0.0,
                                                               "ubound": 1.0})
        assert relerr(X[k], Xo[:, -1]) <= RTOL


def test_sirt_multi_rhs_per_instance_relaxpar_and_saved_iterates():
    """Every instance with its own relaxpar, iterates saved after iterations
    2, 5 and 9, against the oracle per instance."""
    import torch
    from airtoolsii_b200.batch import sirt_multi_device
    N, theta = 24, np.arange(0.0, 180.0, 5.0)
    A = O.paralleltomo_matrix(N, theta)
    op = airt.afun_matrix(A)
    K = 11
    b = A @ O.shepplogan(N)
    lams = np.linspace(0.2, 1.8, K)
    dB = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(b, (K, b.size)))).cuda()
    dX = torch.empty((K, A.shape[1]), dtype=torch.float64, device="cuda")
    save = np.array([2, 5, 9])
    dS = torch.empty((3, K, A.shape[1]), dtype=torch.float64, device="cuda")
    sirt_multi_device(op, "sart", dB.data_ptr(), dX.data_ptr(), K, 9, relaxpar=lams,
                      save=save, d_Xsave=dS.data_ptr())
    S = dS.cpu().numpy()
    for k in range(K):
        Xo, _, _ = O.sirt("sart", A, b, list(save), None, {"relaxpar": float(lams[k])})
        for j in range(3):
            assert relerr(S[j, k], Xo[:, j]) <= RTOL
        assert np.array_equal(S[2, k], dX[k].cpu().numpy())
