"""GPU operator handles: the afun plug-in of AIR Tools II backed by libairt.

An :class:`AirtOperator` owns one ``airt_problem`` (a stored FP32 CSR/CSC
matrix in HBM, or a matrix-free ray geometry) and behaves like the
reference's operator handle ``y = A(v, transp_flag)`` with the flags
``'notransp'``, ``'transp'`` and ``'size'`` (auxil/afun_matrix.m:44-53,
testprobs/paralleltomo.m:146-177).  It also supports ``A @ x``, ``A.T @ y``
and ``A.shape`` so scripts written against a matrix keep working.
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import check, dptr, lib


class AirtOperator:
    """A system matrix (or matrix-free projector) resident on the GPU."""

    def __init__(self, handle: C.c_void_p, kind: str, geometry: dict | None = None):
        self._h = handle
        self.kind = kind                  # 'matrix', 'parallel', 'fan', 'seismic', 'spherical'
        self.geometry = geometry or {}
        m, n, nnz = C.c_int64(), C.c_int64(), C.c_int64()
        check(lib().airt_problem_size(self._h, C.byref(m), C.byref(n), C.byref(nnz)))
        self.m, self.n = int(m.value), int(n.value)
        self.nnz = int(nnz.value)         # -1 for a matrix-free operator
        self._fin = weakref.finalize(self, _destroy, handle)

    # -- construction ------------------------------------------------------
    @classmethod
    def from_matrix(cls, A) -> "AirtOperator":
        """Upload a sparse or dense matrix (kept in FP32 on the device)."""
        if sp.issparse(A):
            Acsc = sp.csc_matrix(A, dtype=np.float64)
        else:
            Acsc = sp.csc_matrix(np.asarray(A, dtype=np.float64))
        Acsc.sum_duplicates()
        Acsc.eliminate_zeros()
        m, n = Acsc.shape
        jc = np.ascontiguousarray(Acsc.indptr, dtype=np.uint64)
        ir = np.ascontiguousarray(Acsc.indices, dtype=np.uint64)
        pr = np.ascontiguousarray(Acsc.data, dtype=np.float64)
        h = C.c_void_p()
        check(lib().airt_problem_from_csc(m, n, _lib.u64ptr(jc),
                                          _lib.u64ptr(ir) if ir.size else None,
                                          dptr(pr) if pr.size else None, C.byref(h)))
        return cls(h, "matrix")

    @property
    def handle(self):
        return self._h

    @property
    def matrix_free(self) -> bool:
        return self.nnz < 0

    @property
    def shape(self):
        return (self.m, self.n)

    # -- the afun protocol ---------------------------------------------------
    def __call__(self, v, transp_flag="notransp"):
        if transp_flag == "size":
            return np.array([self.m, self.n])
        if transp_flag == "notransp":
            return self.apply(v, False)
        if transp_flag == "transp":
            return self.apply(v, True)
        raise ValueError("transp_flag must be 'size', 'notransp' or 'transp'")

    def apply(self, v, transp: bool) -> np.ndarray:
        v = np.ascontiguousarray(np.asarray(v, dtype=np.float64).ravel())
        nin, nout = (self.m, self.n) if transp else (self.n, self.m)
        if v.size != nin:
            raise ValueError("Incorrect length of input vector")
        out = np.empty(nout, dtype=np.float64)
        check(lib().airt_apply(self._h, dptr(v), dptr(out), int(transp)))
        return out

    def __matmul__(self, v):
        v = np.asarray(v, dtype=np.float64)
        if v.ndim == 2:
            return np.stack([self.apply(v[:, k], False) for k in range(v.shape[1])], axis=1)
        return self.apply(v, False)

    @property
    def T(self) -> "_Transposed":
        return _Transposed(self)

    # -- host views ------------------------------------------------------------
    def to_scipy(self) -> sp.csc_matrix:
        """Copy the stored matrix back as a SciPy CSC (FP32 values widened)."""
        if self.matrix_free:
            raise ValueError("a matrix-free operator has no stored matrix")
        jc = np.zeros(self.n + 1, np.uint64)
        ir = np.zeros(max(self.nnz, 1), np.uint64)
        pr = np.zeros(max(self.nnz, 1), np.float64)
        check(lib().airt_problem_export_csc(self._h, _lib.u64ptr(jc), _lib.u64ptr(ir), dptr(pr)))
        return sp.csc_matrix((pr[:self.nnz], ir[:self.nnz].astype(np.int64),
                              jc.astype(np.int64)), shape=(self.m, self.n))

    def weights(self, method: str):
        """Diagonals (M, D) of a built-in SIRT method (get_mfun_dfun.m)."""
        M = np.empty(self.m)
        D = np.empty(self.n)
        check(lib().airt_weights(self._h, _lib.METHODS[method], dptr(M), dptr(D)))
        return M, D

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(lib().airt_problem_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def close(self):
        self._fin()

    def __repr__(self):
        what = "matrix-free" if self.matrix_free else f"nnz={self.nnz}"
        return f"AirtOperator({self.kind}, {self.m}x{self.n}, {what})"


class _Transposed:
    def __init__(self, op: AirtOperator):
        self.op = op

    @property
    def shape(self):
        return (self.op.n, self.op.m)

    def __matmul__(self, v):
        return self.op.apply(v, True)


def _destroy(h):
    try:
        lib().airt_destroy(h)
    except Exception:
        pass


_cache: dict[int, tuple] = {}


def as_operator(A) -> AirtOperator:
    """The GPU operator for A: an AirtOperator as is, a matrix uploaded once
    per matrix object (cached until the object is garbage-collected)."""
    if isinstance(A, AirtOperator):
        return A
    if callable(A) and not sp.issparse(A) and not isinstance(A, np.ndarray):
        raise TypeError("the GPU solvers take a sparse/dense matrix or an AirtOperator "
                        "(paralleltomo/fanlineartomo handles or afun_matrix(A))")
    key = id(A)
    hit = _cache.get(key)
    if hit is not None:
        ref, op, sig = hit
        if ref() is A and sig == _sig(A):
            return op
    op = AirtOperator.from_matrix(A)
    try:
        ref = weakref.ref(A, lambda _r, k=key: _cache.pop(k, None))
        _cache[key] = (ref, op, _sig(A))
    except TypeError:
        pass
    return op


def _sig(A):
    if sp.issparse(A):
        return (A.shape, A.nnz, A.data.ctypes.data if hasattr(A, "data") else 0)
    a = np.asarray(A)
    return (a.shape, a.ctypes.data)


def afun_matrix(A) -> AirtOperator:
    """auxil/afun_matrix.m: the operator handle of an explicit matrix."""
    return AirtOperator.from_matrix(A)
