"""airt_residual_noalloc: the forward residual for callers that cannot
allocate device memory (an application that owns the GPU memory budget
through its own pool, or code that must not call cudaMalloc/cudaFree because
they synchronise the device).  The caller holds the CSR, x, b and r on the
device; the entry point uses its own static scratch.

Checked through the C-ABI, on two calls in a row, against the FP64
residual b - A@x computed by SciPy on the same matrix and against the
existing operator entry point (airt_apply: A*x), within the suite's
relative tolerance of 1e-5.  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import scipy.sparse as sp

import airtoolsii_b200 as airt
from airtoolsii_b200 import _lib
from oracle import airt_oracle as O

pytestmark = pytest.mark.gpu
RTOL = 1e-5


def _relerr(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_residual_noalloc_matches_apply_twice():
    import torch

    A = sp.csr_matrix(O.paralleltomo_matrix(48, np.arange(0.0, 180.0, 2.0)))
    m, n = A.shape
    rng = np.random.default_rng(5)
    x = rng.random(n)
    b = rng.random(m) * 10.0
    r_ref = b - A @ x                              # FP64 SciPy
    op = airt.afun_matrix(A)
    r_apply = b - op(x, "notransp")                # existing entry point airt_apply

    dev = torch.device("cuda")
    rp = torch.from_numpy(A.indptr.astype(np.int64)).to(dev)
    ci = torch.from_numpy(A.indices.astype(np.int32)).to(dev)
    rv = torch.from_numpy(A.data.astype(np.float32)).to(dev)
    dx = torch.from_numpy(x).to(dev)
    db = torch.from_numpy(b).to(dev)
    dr = torch.zeros(m, dtype=torch.float64, device=dev)
    dn = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    L = _lib.lib()
    for _ in range(2):
        dr.fill_(-7.0)
        st = L.airt_residual_noalloc(m, n, C.c_void_p(rp.data_ptr()), C.c_void_p(ci.data_ptr()),
                                     C.c_void_p(rv.data_ptr()), C.c_void_p(dx.data_ptr()),
                                     C.c_void_p(db.data_ptr()), C.c_void_p(dr.data_ptr()),
                                     C.c_void_p(dn.data_ptr()), C.c_void_p(stream))
        assert st == _lib.AIRT_OK, L.airt_last_error()
        torch.cuda.synchronize()
        r = dr.cpu().numpy()
        assert _relerr(r, r_ref) <= RTOL
        assert _relerr(r, r_apply) <= RTOL
        assert abs(float(dn.item()) - np.linalg.norm(r_ref)) <= RTOL * np.linalg.norm(r_ref)


def test_residual_noalloc_flags_a_column_index_out_of_range():
    """A column index outside [0, n) is skipped (no access outside x) and the
    call reports it as a NaN norm; the next call with valid indices is
    clean again, since every call clears the flag."""
    import torch

    A = sp.csr_matrix(O.paralleltomo_matrix(16, np.arange(0.0, 180.0, 10.0)))
    m, n = A.shape
    x = np.ones(n)
    b = np.zeros(m)
    dev = torch.device("cuda")
    ci_ok = A.indices.astype(np.int32)
    ci_bad = ci_ok.copy()
    ci_bad[len(ci_bad) // 2] = n + 5
    rp = torch.from_numpy(A.indptr.astype(np.int64)).to(dev)
    rv = torch.from_numpy(A.data.astype(np.float32)).to(dev)
    dx = torch.from_numpy(x).to(dev)
    db = torch.from_numpy(b).to(dev)
    dr = torch.zeros(m, dtype=torch.float64, device=dev)
    dn = torch.zeros(1, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream().cuda_stream
    L = _lib.lib()
    for ci, expect_nan in ((ci_bad, True), (ci_ok, False)):
        dci = torch.from_numpy(ci).to(dev)
        st = L.airt_residual_noalloc(m, n, C.c_void_p(rp.data_ptr()), C.c_void_p(dci.data_ptr()),
                                     C.c_void_p(rv.data_ptr()), C.c_void_p(dx.data_ptr()),
                                     C.c_void_p(db.data_ptr()), C.c_void_p(dr.data_ptr()),
                                     C.c_void_p(dn.data_ptr()), C.c_void_p(stream))
        assert st == _lib.AIRT_OK, L.airt_last_error()
        torch.cuda.synchronize()
        assert np.isnan(float(dn.item())) == expect_nan
    np.testing.assert_allclose(float(dn.item()), np.linalg.norm(A @ x), rtol=RTOL)


def test_residual_noalloc_rejects_oversize():
    L = _lib.lib()
    st = L.airt_residual_noalloc(10, (1 << 20) + 1, None, None, None, None, None, None, None, None)
    assert st == _lib.AIRT_ERR_ARG
    assert b"no-alloc maximum" in L.airt_last_error()
