"""The MEX gateway (airtoolsii_b200/matlab/airt_mex.c), the reference-side
binding of the C-ABI for MATLAB / GNU Octave host code.

MATLAB is not installed, so the gateway is (1) compiled with gcc against
stub declarations of the documented MEX and mxGPUArray C API
(tests/mex_stub/*.h) with all warnings as errors, with and without the
gpuArray commands, and (2) linked with a minimal stand-in for the MEX
runtime (tests/mex_stub/fake_mex.c) and libairt, and its mexFunction driven
from Python the way MATLAB would call it: command strings, double / int
arrays, option structs, uint64 handles, error identifiers.  The CPU tests
check dispatch and argument errors; the GPU tests run the commands end to
end (matrix upload, generated geometries, sirt / art / cart / fbp, custom
full weights, batches) against the FP64 oracle.
"""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest
import scipy.sparse as sp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STUB = os.path.join(ROOT, "tests", "mex_stub")
GATEWAY = os.path.join(ROOT, "airtoolsii_b200", "matlab", "airt_mex.c")
LIBDIR = os.path.join(ROOT, "airtoolsii_b200")
SO = os.path.join(STUB, "_build", "libfakemex.so")

DOUBLE, SINGLE, INT32, INT64, UINT64, STRUCT = 6, 7, 12, 14, 15, 2


@pytest.mark.parametrize("gpuarray", [False, True])
def test_gateway_compiles_against_the_mex_api(gpuarray):
    cmd = ["gcc", "-fsyntax-only", "-std=c99", "-Wall", "-Wextra", "-Werror", "-I" + STUB,
           "-I" + os.path.join(ROOT, "include"), GATEWAY]
    if gpuarray:
        cmd.insert(1, "-DAIRT_MEX_GPUARRAY")
    out = subprocess.run(cmd, capture_output=True, text=True)
    assert out.returncode == 0, out.stderr


def test_gateway_has_a_command_for_every_part_of_the_c_abi():
    src = open(GATEWAY).read()
    for cmd in ("matrix", "parallel", "fan", "seismic", "spherical", "size", "export", "apply",
                "weights", "rho", "sirt", "art", "cart", "fbp", "destroy", "batch",
                "batch_layout", "batch_rho", "batch_sirt", "batch_kaczmarz", "batch_backproject", "sirt_multi",
                "batch_destroy", "unet", "unet_params", "unet_set_params", "unet_forward",
                "unet_destroy"):
        assert '{"%s", cmd_' % cmd in src, cmd
    for shim in ("sirt.m", "art.m", "cart.m", "paralleltomo.m", "fanlineartomo.m", "fbp.m"):
        assert os.path.exists(os.path.join(ROOT, "airtoolsii_b200", "matlab", shim)), shim


class Mex:
    """mexFunction of the gateway behind the stand-in runtime."""

    def __init__(self):
        srcs = [os.path.join(STUB, "fake_mex.c"), GATEWAY]
        if not os.path.exists(SO) or any(os.path.getmtime(s) > os.path.getmtime(SO) for s in srcs):
            os.makedirs(os.path.dirname(SO), exist_ok=True)
            subprocess.run(["gcc", "-std=c99", "-O1", "-fPIC", "-shared", "-I" + STUB,
                            "-I" + os.path.join(ROOT, "include"), "-o", SO] + srcs +
                           ["-L" + LIBDIR, "-lairt", "-Wl,-rpath," + LIBDIR], check=True)
        L = C.CDLL(SO)
        vp = C.c_void_p
        L.fm_numeric.restype = vp
        L.fm_numeric.argtypes = [C.c_int, C.c_size_t, C.c_size_t, vp]
        L.fm_char.restype = vp
        L.fm_char.argtypes = [C.c_char_p]
        L.fm_sparse.restype = vp
        L.fm_sparse.argtypes = [C.c_size_t, C.c_size_t, C.c_size_t, vp, vp, vp]
        L.fm_struct.restype = vp
        L.fm_struct.argtypes = [C.c_int, C.POINTER(C.c_char_p)]
        L.fm_set_field.argtypes = [vp, C.c_char_p, vp]
        L.fm_get_field.restype = vp
        L.fm_get_field.argtypes = [vp, C.c_char_p]
        for f in ("fm_class", "fm_is_sparse"):
            getattr(L, f).restype = C.c_int
            getattr(L, f).argtypes = [vp]
        for f in ("fm_m", "fm_n"):
            getattr(L, f).restype = C.c_size_t
            getattr(L, f).argtypes = [vp]
        for f in ("fm_data", "fm_jc", "fm_ir"):
            getattr(L, f).restype = vp
            getattr(L, f).argtypes = [vp]
        L.fm_err_id.restype = C.c_char_p
        L.fm_err_msg.restype = C.c_char_p
        L.fm_call.restype = C.c_int
        L.fm_call.argtypes = [C.c_int, C.POINTER(vp), C.c_int, C.POINTER(vp)]
        self.L = L

    # ---- MATLAB values -> mxArray
    def arr(self, v):
        L = self.L
        if isinstance(v, str):
            return L.fm_char(v.encode())
        if isinstance(v, dict):
            names = (C.c_char_p * len(v))(*[k.encode() for k in v])
            s = L.fm_struct(len(v), names)
            for k, x in v.items():
                L.fm_set_field(s, k.encode(), self.arr(x))
            return s
        if sp.issparse(v):
            A = sp.csc_matrix(v, dtype=np.float64)
            A.sort_indices()
            jc = np.ascontiguousarray(A.indptr, np.uint64)
            ir = np.ascontiguousarray(A.indices, np.uint64)
            pr = np.ascontiguousarray(A.data)
            return L.fm_sparse(A.shape[0], A.shape[1], A.nnz, jc.ctypes.data, ir.ctypes.data,
                               pr.ctypes.data)
        a = np.asarray(v)
        cls = {np.dtype(np.float64): DOUBLE, np.dtype(np.float32): SINGLE,
               np.dtype(np.int32): INT32, np.dtype(np.int64): INT64,
               np.dtype(np.uint64): UINT64}.get(a.dtype)
        if cls is None:
            a = a.astype(np.float64)
            cls = DOUBLE
        if a.size == 0:
            return L.fm_numeric(cls, 0, 0, None)
        a2 = a.reshape(a.shape[0], -1) if a.ndim >= 1 else a.reshape(1, 1)
        if a.ndim == 1:
            a2 = a.reshape(-1, 1)
        f = np.asfortranarray(a2)
        return L.fm_numeric(cls, f.shape[0], f.shape[1], f.ctypes.data if f.size else None)

    # ---- mxArray -> Python
    def val(self, p):
        if not p:                        # the command set no output
            return None
        L = self.L
        cls, m, n = L.fm_class(p), L.fm_m(p), L.fm_n(p)
        if L.fm_is_sparse(p):
            jc = np.ctypeslib.as_array(C.cast(L.fm_jc(p), C.POINTER(C.c_uint64)), (n + 1,)).copy()
            nnz = int(jc[-1])
            ir = np.ctypeslib.as_array(C.cast(L.fm_ir(p), C.POINTER(C.c_uint64)), (max(nnz, 1),))
            pr = np.ctypeslib.as_array(C.cast(L.fm_data(p), C.POINTER(C.c_double)), (max(nnz, 1),))
            return sp.csc_matrix((pr[:nnz].copy(), ir[:nnz].astype(np.int64), jc.astype(np.int64)),
                                 shape=(m, n))
        if cls == STRUCT:
            return p
        ct = {DOUBLE: C.c_double, SINGLE: C.c_float, INT32: C.c_int32, INT64: C.c_int64,
              UINT64: C.c_uint64}[cls]
        if m * n == 0:
            return np.zeros((m, n))
        a = np.ctypeslib.as_array(C.cast(L.fm_data(p), C.POINTER(ct)), (m * n,)).copy()
        return a.reshape((m, n), order="F")

    def field(self, s, name):
        return self.val(self.L.fm_get_field(s, name.encode()))

    def __call__(self, cmd, *args, nout=1):
        prhs = (C.c_void_p * (len(args) + 1))(self.arr(cmd), *[self.arr(a) for a in args])
        plhs = (C.c_void_p * max(nout, 1))()
        if self.L.fm_call(nout, plhs, len(args) + 1, prhs):
            raise MexError(self.L.fm_err_id().decode(), self.L.fm_err_msg().decode())
        outs = [self.val(plhs[i]) for i in range(nout)]
        return outs[0] if nout == 1 else outs


class MexError(Exception):
    def __init__(self, ident, msg):
        super().__init__(f"{ident}: {msg}")
        self.ident = ident


@pytest.fixture(scope="module")
def mex():
    return Mex()


def test_gateway_dispatch_and_argument_errors(mex):
    import airtoolsii_b200  # noqa: F401  (the library the gateway links)
    assert mex("version")[0, 0] >= 10000
    with pytest.raises(MexError) as e:
        mex("bogus")
    assert e.value.ident == "AIRT:cmd"
    with pytest.raises(MexError) as e:
        mex("sirt", 1.0)
    assert e.value.ident == "AIRT:usage"
    with pytest.raises(MexError) as e:
        mex("matrix", np.ones((2, 2)))                 # dense, not sparse
    assert e.value.ident == "AIRT:usage"
    with pytest.raises(MexError) as e:
        mex("size", np.array([5.0]))                   # not a uint64 handle
    assert e.value.ident == "AIRT:usage"
    with pytest.raises(MexError) as e:
        mex("size", np.array([0], np.uint64))          # null handle: the library's own error
    assert e.value.ident == "AIRT:arg"


# ------------------------------------------------------------------ GPU
def _relerr(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.gpu
def test_gateway_matrix_sirt_art_cart_fbp_vs_oracle(mex):
    from oracle import airt_oracle as O
    N, theta = 32, np.arange(0.0, 180.0, 4.0)
    A = O.paralleltomo_matrix(N, theta)
    x = O.shepplogan(N)
    b, en = O.add_noise(A @ x, 0.02, seed=3)
    h = mex("matrix", A)
    assert list(mex("size", h).ravel()) == [A.shape[0], A.shape[1]]
    E = mex("export", h)
    assert np.array_equal(E.indptr, A.indptr) and np.array_equal(E.indices, A.indices)
    np.testing.assert_allclose(mex("apply", h, x, 0).ravel(), A @ x, rtol=1e-6)
    # sirt: cimmino, 15 iterations saved at 5 and 15, box [0, 1]
    M, D = mex("weights", h, 1.0, nout=2)
    rho = mex("rho", h, {"method": 1.0})[0, 0]
    Xo, io, _ = O.sirt("cimmino", A, b, [5, 15], None, {"rho": rho, "lbound": 0.0, "ubound": 1.0})
    X, info = mex("sirt", h, {"method": 1.0, "relax_kind": 1.0, "relaxpar": 1.9 / rho,
                              "lbound": 0.0, "ubound": 1.0}, b, np.zeros((0, 0)),
                  np.array([5.0, 15.0]), nout=2)
    assert X.shape == (A.shape[1], 2) and mex.field(info, "finaliter")[0, 0] == 15
    assert _relerr(X[:, 1], Xo[:, 1]) <= 1e-5 and _relerr(X[:, 0], Xo[:, 0]) <= 1e-5
    np.testing.assert_allclose(M.ravel(), O.get_mfun_dfun("cimmino", A)[0], rtol=1e-6)
    # sirt with the DP rule: X trimmed to the saved columns
    X, info = mex("sirt", h, {"method": 4.0, "relaxpar": 1.9, "stoprule": 1.0,
                              "taudelta": 1.02 * en}, b, np.zeros((0, 0)),
                  np.arange(1.0, 301.0), nout=2)
    Xo, io, _ = O.sirt("sart", A, b, list(range(1, 301)), None,
                       {"stoprule": {"type": "DP", "taudelta": 1.02 * en}})
    assert mex.field(info, "finaliter")[0, 0] == io["finaliter"] < 300
    assert X.shape[1] == io["finaliter"] and _relerr(X[:, -1], Xo[:, -1]) <= 1e-5
    # art: symmetric Kaczmarz order (order_kind 1), 3 double sweeps
    X = mex("art", h, {"order_kind": 1.0, "relaxpar": 1.0}, b, np.zeros((0, 0)), np.array([3.0]))
    Xo, _ = O.art("symkaczmarz", A, b, [6])
    assert _relerr(X[:, -1], Xo[:, -1]) <= 1e-5
    # art: caller row order (1-based, as MATLAB passes it)
    order = np.arange(A.shape[0], 0, -1).astype(np.float64)
    X = mex("art", h, {"order_kind": 2.0, "rows": order}, b, np.zeros((0, 0)), np.array([2.0]))
    Xo, _ = O.art((order - 1).astype(np.int64), A, b, [2])
    assert _relerr(X[:, -1], Xo[:, -1]) <= 1e-5
    # cart: columnaction, 4 sweeps
    X = mex("cart", h, {"order_kind": 0.0, "relaxpar": 0.25}, b, np.zeros((0, 0)), np.array([4.0]))
    Xo, _ = O.cart("columnaction", A, b, [4])
    assert _relerr(X[:, -1], Xo[:, -1]) <= 1e-5
    # fbp with the hamming kernel (the handle holds the matrix in FP32)
    from airtoolsii_b200.analytic import fbp_kernel
    xf = mex("fbp", h, b, float(theta.size), fbp_kernel(A.shape[0] // theta.size, "hamming"))
    A32 = A.copy()
    A32.data = A32.data.astype(np.float32).astype(np.float64)
    assert _relerr(xf.ravel(), O.fbp(A32, b, theta, "hamming")) <= 1e-10
    mex("destroy", h)


@pytest.mark.gpu
def test_gateway_geometries_custom_weights_and_batch(mex):
    from oracle import airt_oracle as O
    from airtoolsii_b200 import testprobs as T
    N, theta = 24, np.arange(0.0, 180.0, 6.0)
    th, p, d, ct, st, off = O.parallel_geometry(N, theta)
    h = mex("parallel", float(N), ct, st, off, 0.0)
    E = mex("export", h)
    R = O.paralleltomo_matrix(N, theta)
    assert np.array_equal(E.indices, R.indices) and np.array_equal(E.indptr, R.indptr)
    # the matrix-free handle applies the same operator
    hm = mex("parallel", float(N), ct, st, off, 1.0)
    v = np.random.default_rng(1).random(N * N)
    np.testing.assert_allclose(mex("apply", hm, v, 0).ravel(), mex("apply", h, v, 0).ravel(),
                               rtol=1e-12)
    # fan geometry tables as fanlineartomo.m forms them
    fth, fp, fR, _, _, fct, fst, fcw, fsw = T.fan_tables(N, np.arange(0.0, 360.0, 10.0))
    hf = mex("fan", float(N), fct, fst, fcw, fsw, fR, 0.0)
    Ef = mex("export", hf)
    Rf = O.fanlineartomo_matrix(N, np.arange(0.0, 360.0, 10.0))
    assert np.array_equal(Ef.indices, Rf.indices) and np.array_equal(Ef.indptr, Rf.indptr)
    # custom full M (a non-diagonal SPD matrix) through the options struct
    m = R.shape[0]
    rng = np.random.default_rng(2)
    Q = rng.standard_normal((m, 3))
    Mf = np.diag(rng.uniform(0.5, 1.5, m)) * 1e-3 + 1e-5 * (Q @ Q.T)
    b = R @ O.shepplogan(N)
    rho = mex("rho", h, {"method": 5.0, "M": Mf})[0, 0]
    _, io, _ = O.sirt({"M": Mf}, R, b, [1])
    assert abs(rho - io["rho"]) <= 1e-4 * io["rho"]
    X = mex("sirt", h, {"method": 5.0, "M": Mf, "relaxpar": 1.0 / rho}, b, np.zeros((0, 0)),
            np.array([8.0]))
    Xo, _, _ = O.sirt({"M": Mf}, R, b, [8], None, {"relaxpar": 1.0 / rho})
    assert _relerr(X[:, -1], Xo[:, -1]) <= 1e-5
    # a batch of two instances: layout, cimmino to 12 iterations, Kaczmarz
    Ns = [16, 20]
    ths = [np.arange(0.0, 180.0, 10.0), np.arange(0.0, 180.0, 15.0)]
    tabs = [O.parallel_geometry(n_, t_) for n_, t_ in zip(Ns, ths)]
    bh = mex("batch", np.array(Ns, np.int32), np.array([len(t_) for t_ in ths], np.int32),
             np.array([tb[1] for tb in tabs], np.int32), np.concatenate([tb[3] for tb in tabs]),
             np.concatenate([tb[4] for tb in tabs]), np.concatenate([tb[5] for tb in tabs]))
    ro, co, nz = mex("batch_layout", bh, 2.0, nout=3)
    mats = [O.paralleltomo_matrix(n_, t_) for n_, t_ in zip(Ns, ths)]
    assert int(nz[0, 0]) == sum(M_.nnz for M_ in mats)
    bs = [M_ @ O.shepplogan(n_) for M_, n_ in zip(mats, Ns)]
    rhos = mex("batch_rho", bh, 2.0, 1.0).ravel()
    x, it, sr = mex("batch_sirt", bh, 2.0, {"method": 1.0, "relaxpar": 1.9 / rhos, "kmax": 12.0},
                    np.concatenate(bs), np.zeros((0, 0)), nout=3)
    co = co.ravel().astype(int)
    for k, M_ in enumerate(mats):
        Xo, _, _ = O.sirt("cimmino", M_, bs[k], [12], None, {"rho": rhos[k]})
        assert _relerr(x.ravel()[co[k]:co[k + 1]], Xo[:, -1]) <= 1e-5
    assert list(it.ravel()) == [12, 12]
    xk = mex("batch_kaczmarz", bh, 2.0, np.concatenate(bs), 2.0, 1.0, np.zeros((0, 0)),
             np.zeros((0, 0)))
    for k, M_ in enumerate(mats):
        Xo, _ = O.art("kaczmarz", M_, bs[k], [2])
        assert _relerr(xk.ravel()[co[k]:co[k + 1]], Xo[:, -1]) <= 1e-5
    mex("batch_destroy", bh)
    for hh in (h, hm, hf):
        mex("destroy", hh)
