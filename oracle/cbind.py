"""ctypes binding of the C oracle (oracle/airt_oracle_c.c).

TEST INFRASTRUCTURE ONLY (checker and CPU baseline; never the product).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np
import scipy.sparse as sp

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_p = np.ctypeslib.ndpointer
_D = _p(dtype=np.float64, flags="C_CONTIGUOUS")
_I = _p(dtype=np.int64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the C oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO):
            build()
        L = C.CDLL(_SO)
        L.oracle_trace_count.argtypes = [C.c_int, C.c_int64, _D, _D, _D, _D, C.c_int, _I]
        L.oracle_trace_fill.argtypes = [C.c_int, C.c_int64, _D, _D, _D, _D, C.c_int, _I, _I, _D]
        L.oracle_sirt_csr.argtypes = [C.c_int64, C.c_int64, _I, _I, _D, _I, _I, _D, _D, _D, _D,
                                      C.c_double, C.c_double, C.c_double, C.c_double, C.c_int,
                                      _D, _D]
        L.oracle_sirt_csr.restype = C.c_int
        L.oracle_kaczmarz.argtypes = [C.c_int64, C.c_int64, _I, _I, _D, _D, _D, _I, C.c_int64,
                                      C.c_double, C.c_double, C.c_double, C.c_int, _D]
        L.oracle_num_threads.restype = C.c_int
        _lib = L
    return _lib


def rays_arrays(rays):
    """Collect (row, x0t, y0t, a, b) ray tuples into contiguous arrays."""
    arr = np.array([r[1:] for r in rays], dtype=np.float64).reshape(-1, 4)
    return [np.ascontiguousarray(arr[:, k]) for k in range(4)]


def trace_coo(N, rays, exclude):
    """COO triplets (row-major ray order) from the C restatement."""
    x0t, y0t, a, b = rays_arrays(rays)
    nr = x0t.size
    counts = np.zeros(nr, np.int64)
    lib().oracle_trace_count(N, nr, x0t, y0t, a, b, int(exclude), counts)
    offs = np.zeros(nr + 1, np.int64)
    np.cumsum(counts, out=offs[1:])
    cols = np.zeros(offs[-1], np.int64)
    vals = np.zeros(offs[-1], np.float64)
    lib().oracle_trace_fill(N, nr, x0t, y0t, a, b, int(exclude), offs, cols, vals)
    rows = np.repeat(np.arange(nr, dtype=np.int64), counts)
    return rows, cols, vals


class PreparedSirt:
    """FP64 CSR + CSC arrays of A prepared once, so that timing covers only
    the C iterations (oracle_sirt_csr)."""

    def __init__(self, A, b, M, D):
        A = sp.csr_matrix(A, dtype=np.float64)
        Ac = A.tocsc()
        self.m, self.n = A.shape
        self.rp = A.indptr.astype(np.int64)
        self.ci = A.indices.astype(np.int64)
        self.rv = np.ascontiguousarray(A.data)
        self.cp = Ac.indptr.astype(np.int64)
        self.ri = Ac.indices.astype(np.int64)
        self.cv = np.ascontiguousarray(Ac.data)
        self.b = np.ascontiguousarray(b, np.float64)
        self.M = np.ascontiguousarray(M, np.float64)
        self.D = np.ascontiguousarray(D, np.float64)

    def run(self, lam, lb, ub, kmax, taudelta=None):
        x = np.zeros(self.n)
        resn = np.zeros(kmax + 1)
        k = lib().oracle_sirt_csr(self.m, self.n, self.rp, self.ci, self.rv, self.cp, self.ri,
                                  self.cv, self.b, self.M, self.D, float(lam),
                                  float("nan") if lb is None else float(lb),
                                  float("nan") if ub is None else float(ub),
                                  -1.0 if taudelta is None else float(taudelta), int(kmax), x, resn)
        return x, k, resn[:k + 1]


def sirt_csr(A, b, M, D, lam, lb, ub, taudelta, kmax, x0=None):
    """FP64 SIRT with constant relaxpar (see oracle_sirt_csr).  Returns
    (x, finaliter, resnorms)."""
    A = sp.csr_matrix(A, dtype=np.float64)
    Ac = A.tocsc()
    m, n = A.shape
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    resn = np.zeros(kmax + 1)
    k = lib().oracle_sirt_csr(m, n, A.indptr.astype(np.int64), A.indices.astype(np.int64),
                              np.ascontiguousarray(A.data),
                              Ac.indptr.astype(np.int64), Ac.indices.astype(np.int64),
                              np.ascontiguousarray(Ac.data),
                              np.ascontiguousarray(b, np.float64), np.ascontiguousarray(M, np.float64),
                              np.ascontiguousarray(D, np.float64), float(lam),
                              float("nan") if lb is None else float(lb),
                              float("nan") if ub is None else float(ub),
                              -1.0 if taudelta is None else float(taudelta), int(kmax), x, resn)
    return x, k, resn[:k + 1]


def kaczmarz(A, b, nrm, rows, lam, lb, ub, sweeps, x0=None):
    """FP64 Kaczmarz sweeps in a fixed row order (see oracle_kaczmarz)."""
    A = sp.csr_matrix(A, dtype=np.float64)
    m, n = A.shape
    x = np.zeros(n) if x0 is None else np.array(x0, np.float64)
    rows = np.ascontiguousarray(rows, np.int64)
    lib().oracle_kaczmarz(m, n, A.indptr.astype(np.int64), A.indices.astype(np.int64),
                          np.ascontiguousarray(A.data), np.ascontiguousarray(b, np.float64),
                          np.ascontiguousarray(nrm, np.float64), rows, rows.size, float(lam),
                          float("nan") if lb is None else float(lb),
                          float("nan") if ub is None else float(ub), int(sweeps), x)
    return x


def num_threads() -> int:
    return int(lib().oracle_num_threads())
