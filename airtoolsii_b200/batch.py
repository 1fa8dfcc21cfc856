"""Batched independent reconstructions on one GPU (no reference counterpart:
the reference solves one problem per sirt/art call).

A ParallelBatch holds many paralleltomo instances of uneven size as one
block-diagonal system generated on the GPU.  ``sirt`` runs cimmino/drop/...
on all of them at once with a relaxation parameter and a discrepancy-
principle threshold per instance; every instance stops on its own.
``kaczmarz`` runs one CTA per instance.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib
from ._lib import check, dptr, lib
from .testprobs import parallel_tables

_ip = C.POINTER(C.c_int)


def _batch_signatures():
    L = lib()
    i64p = C.POINTER(C.c_int64)
    sig = {
        "airt_batch_parallel": (C.c_int, [C.c_int, _ip, _ip, _ip, _lib._dp, _lib._dp, _lib._dp,
                                          C.POINTER(C.c_void_p)]),
        "airt_batch_layout": (C.c_int, [C.c_void_p, i64p, i64p, i64p]),
        "airt_batch_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
        "airt_batch_rho": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, _lib._dp]),
        "airt_batch_sirt": (C.c_int, [C.c_void_p, C.c_int, _lib._dp, _lib._dp, _lib._dp, C.c_int64,
                                      C.c_int, C.c_double, C.c_int, C.c_double, _lib._dp, _lib._dp,
                                      i64p, _ip, _lib._dp]),
        "airt_batch_sirt_device": (C.c_int, [C.c_void_p, C.c_int, _lib._dp, C.c_void_p, _lib._dp,
                                             C.c_int64, C.c_int, C.c_double, C.c_int, C.c_double,
                                             C.c_void_p, C.c_void_p, i64p, _ip, _lib._dp]),
        "airt_batch_sirt_rule": (C.c_int, [C.c_void_p, C.c_int, _lib._dp, _lib._dp, C.c_int,
                                           _lib._dp, C.c_int, C.c_int64, C.c_int, C.c_double,
                                           C.c_int, C.c_double, _lib._dp, _lib._dp, i64p, _ip,
                                           _lib._dp]),
        "airt_batch_nnz": (C.c_int, [C.c_void_p, i64p]),
        "airt_batch_apply": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]),
        "airt_batch_backproject": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, _lib._dp]),
        "airt_batch_fbp": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, _lib._dp, C.c_int, _lib._dp,
                                     C.c_void_p, _lib._dp]),
        "airt_batch_kaczmarz": (C.c_int, [C.c_void_p, _lib._dp, C.c_int64, C.c_double, C.c_int,
                                          C.c_double, C.c_int, C.c_double, _lib._dp, _lib._dp]),
        "airt_batch_destroy": (C.c_int, [C.c_void_p]),
    }
    return L, sig


def _bounds(v):
    if v is None:
        return _lib.BOUND_NONE, 0.0
    return _lib.BOUND_SCALAR, float(v)


class ParallelBatch:
    """Instances k = 0..K-1 with image size Ns[k], angles thetas[k] (degrees)
    and ps[k] rays (default round(sqrt(2)*N), offsets linspace(-d/2,d/2,p))."""

    def __init__(self, Ns, thetas, ps=None, ds=None):
        K = len(Ns)
        if K < 1 or len(thetas) != K:
            raise ValueError("one angle list per instance is required")
        ps = [None] * K if ps is None else list(ps)
        ds = [None] * K if ds is None else list(ds)
        Nv, nAv, pv, ct, st, off = [], [], [], [], [], []
        for k in range(K):
            th, p, d, c, s, o = parallel_tables(int(Ns[k]), thetas[k], ps[k], ds[k])
            Nv.append(int(Ns[k]))
            nAv.append(len(th))
            pv.append(p)
            ct.append(c)
            st.append(s)
            off.append(o)
        self.Ns, self.nAs, self.ps = Nv, nAv, pv
        L, sig = _batch_signatures()
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        self._L = L
        arr = lambda v: np.ascontiguousarray(v, dtype=np.int32)  # noqa: E731
        self._keep = [arr(Nv), arr(nAv), arr(pv), np.ascontiguousarray(np.concatenate(ct)),
                      np.ascontiguousarray(np.concatenate(st)),
                      np.ascontiguousarray(np.concatenate(off))]
        h = C.c_void_p()
        a = self._keep
        check(L.airt_batch_parallel(K, a[0].ctypes.data_as(_ip), a[1].ctypes.data_as(_ip),
                                    a[2].ctypes.data_as(_ip), dptr(a[3]), dptr(a[4]), dptr(a[5]),
                                    C.byref(h)))
        self._h = h
        self.K = K
        self.row_off = np.zeros(K + 1, np.int64)
        self.col_off = np.zeros(K + 1, np.int64)
        nnz = C.c_int64()
        check(L.airt_batch_layout(h, _lib.i64ptr(self.row_off), _lib.i64ptr(self.col_off),
                                  C.byref(nnz)))
        self.nnz = int(nnz.value)
        self.m, self.n = int(self.row_off[-1]), int(self.col_off[-1])

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self._L.airt_batch_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def stream_ptr(self) -> int:
        s = C.c_void_p()
        check(self._L.airt_batch_stream(self._h, C.byref(s)))
        return int(s.value or 0)

    def split_rows(self, v):
        return [v[self.row_off[k]:self.row_off[k + 1]] for k in range(self.K)]

    def split_cols(self, v):
        return [v[self.col_off[k]:self.col_off[k + 1]] for k in range(self.K)]

    def rho(self, method: str, tol=1e-7, maxit=200) -> np.ndarray:
        out = np.zeros(self.K)
        check(self._L.airt_batch_rho(self._h, _lib.METHODS[method], tol, maxit, dptr(out)))
        return out

    def sirt(self, method, b, kmax, taudelta=None, relaxpar=None, rho=None, lbound=None,
             ubound=None, x0=None, stoprule=None, ncp_smooth=2):
        """SIRT on every instance; b is the concatenation of the instances'
        right-hand sides (or a list of them).  stoprule: 'DP' (default when
        taudelta is given), 'ME', 'NCP' (each instance's residual as its
        p x nA projections, ncp_smooth values) or 'NONE', applied per
        instance (check_stoprules.m).  Returns (x_list, info) with
        per-instance finaliter, stoprule, rho and relaxpar."""
        b = np.ascontiguousarray(np.concatenate(b) if isinstance(b, (list, tuple)) else b,
                                 dtype=np.float64)
        if b.size != self.m:
            raise ValueError("The size of A and b do not match.")
        if relaxpar is None:
            if method == "sart":
                rho = np.ones(self.K)
            elif rho is None:
                rho = self.rho(method)
            lam = 1.9 / np.asarray(rho, dtype=np.float64)
        else:
            lam = np.broadcast_to(np.asarray(relaxpar, dtype=np.float64), (self.K,)).copy()
        lam = np.ascontiguousarray(lam)
        td = None if taudelta is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(taudelta, dtype=np.float64), (self.K,)))
        x = np.zeros(self.n)
        x0v = None if x0 is None else np.ascontiguousarray(
            np.concatenate(x0) if isinstance(x0, (list, tuple)) else x0, dtype=np.float64)
        fin = np.zeros(self.K, np.int64)
        rule = np.zeros(self.K, np.int32)
        ms = C.c_double()
        lk, lv = _bounds(lbound)
        uk, uv = _bounds(ubound)
        rule_name = (stoprule or ("DP" if td is not None else "NONE")).upper()
        if rule_name not in _lib.STOP:
            raise ValueError("The chosen stopping rule is not valid.")
        if rule_name in ("DP", "ME") and td is None:
            raise ValueError("For stopping rules DP and ME a scalar taudelta must be given in options.")
        check(self._L.airt_batch_sirt_rule(self._h, _lib.METHODS[method], dptr(lam), dptr(b),
                                           _lib.STOP[rule_name], dptr(td), int(ncp_smooth),
                                           int(kmax), lk, lv, uk, uv, dptr(x0v), dptr(x),
                                           _lib.i64ptr(fin), rule.ctypes.data_as(_ip), C.byref(ms)))
        info = {"finaliter": fin, "stoprule": rule, "relaxpar": lam,
                "rho": None if rho is None else np.asarray(rho), "gpu_ms": float(ms.value)}
        return self.split_cols(x), info

    def sirt_device(self, method, d_b, d_x, kmax, taudelta=None, relaxpar=None, rho=None,
                    lbound=None, ubound=None, d_x0=None):
        """sirt on device vectors: d_b (m doubles), d_x (n doubles), optional
        d_x0 (n doubles) given as device addresses.  Returns info as sirt."""
        if relaxpar is None:
            if method == "sart":
                rho = np.ones(self.K)
            elif rho is None:
                rho = self.rho(method)
            lam = 1.9 / np.broadcast_to(np.asarray(rho, dtype=np.float64), (self.K,))
        else:
            lam = np.broadcast_to(np.asarray(relaxpar, dtype=np.float64), (self.K,))
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        td = None if taudelta is None else np.ascontiguousarray(
            np.broadcast_to(np.asarray(taudelta, dtype=np.float64), (self.K,)))
        fin = np.zeros(self.K, np.int64)
        rule = np.zeros(self.K, np.int32)
        ms = C.c_double()
        lk, lv = _bounds(lbound)
        uk, uv = _bounds(ubound)
        check(self._L.airt_batch_sirt_device(self._h, _lib.METHODS[method], dptr(lam),
                                             C.c_void_p(d_b), dptr(td), int(kmax), lk, lv, uk,
                                             uv, C.c_void_p(d_x0 or None), C.c_void_p(d_x),
                                             _lib.i64ptr(fin), rule.ctypes.data_as(_ip),
                                             C.byref(ms)))
        return {"finaliter": fin, "stoprule": rule, "relaxpar": lam, "gpu_ms": float(ms.value)}

    def inst_nnz(self) -> np.ndarray:
        """Nonzeros of every instance's matrix."""
        out = np.zeros(self.K, np.int64)
        check(self._L.airt_batch_nnz(self._h, _lib.i64ptr(out)))
        return out

    def apply_device(self, d_in, d_out, transp=False) -> None:
        """y = A*x (or A'*x) of the whole block-diagonal batch, device vectors."""
        check(self._L.airt_batch_apply(self._h, C.c_void_p(d_in), C.c_void_p(d_out), int(transp)))

    def backproject_device(self, method, d_b, d_x) -> float:
        """x = D .* A'(M .* b) per instance on device vectors (the first SIRT
        iterate from zero with relaxpar 1); returns the device time in ms."""
        ms = C.c_double()
        check(self._L.airt_batch_backproject(self._h, _lib.METHODS[method], C.c_void_p(d_b),
                                             C.c_void_p(d_x), C.byref(ms)))
        return float(ms.value)

    def fbp_device(self, d_b, d_x, filter="ram-lak") -> float:
        """Filtered back projection of every instance (auxil/fbp.m:40-79) on
        device vectors; all instances need the same number of rays.  Returns
        the device time in ms."""
        from .analytic import fbp_kernel
        if len(set(self.ps)) != 1:
            raise ValueError("batch fbp needs the same number of rays in every instance")
        nr = self.ps[0]
        h = fbp_kernel(nr, filter)
        scale = np.concatenate([np.full(na, math.pi / (2.0 * na)) for na in self.nAs])
        ms = C.c_double()
        check(self._L.airt_batch_fbp(self._h, C.c_void_p(d_b), int(nr), dptr(h), int(h.size),
                                     dptr(np.ascontiguousarray(scale)), C.c_void_p(d_x),
                                     C.byref(ms)))
        return float(ms.value)

    def kaczmarz(self, b, sweeps, relaxpar=1.0, lbound=None, ubound=None):
        """Kaczmarz sweeps (row order of art.m:188) on every instance from x0 = 0."""
        b = np.ascontiguousarray(np.concatenate(b) if isinstance(b, (list, tuple)) else b,
                                 dtype=np.float64)
        x = np.zeros(self.n)
        ms = C.c_double()
        lk, lv = _bounds(lbound)
        uk, uv = _bounds(ubound)
        check(self._L.airt_batch_kaczmarz(self._h, dptr(b), int(sweeps), float(relaxpar), lk, lv,
                                          uk, uv, dptr(x), C.byref(ms)))
        return self.split_cols(x), {"gpu_ms": float(ms.value)}


def sirt_multi_device(op, method, d_B, d_X, K, kmax, taudelta=None, relaxpar=None, rho=None,
                      d_X0=None, lbound=None, ubound=None, save=None, d_Xsave=None):
    """SIRT on K right-hand sides of one stored matrix at once
    (airt_sirt_multi_device): d_B (K x m), d_X (K x n) and optional d_X0
    (K x n) are device addresses of instance-major FP64 arrays.  Every
    instance stops on its own by the DP rule when taudelta (K values) is
    given, else runs kmax iterations.  relaxpar: a scalar or K values
    (default 1.9/rho, rho of the method estimated on the device if not
    given; 1 for sart).  save (iteration numbers) with d_Xsave (len(save) x
    K x n) keeps every instance's iterate after those iterations.  Returns
    per-instance finaliter and stoprule and the device time."""
    from .afun import as_operator
    op = as_operator(op)
    L = lib()
    code = _lib.METHODS[method]
    if relaxpar is None:
        if method == "sart":
            rho = 1.0
        elif rho is None:
            r = C.c_double()
            check(L.airt_rho(op.handle, code, None, None, 1e-7, 200, C.byref(r)))
            rho = float(r.value)
        relaxpar = 1.9 / rho
    lamk = None
    if np.ndim(relaxpar) > 0:
        lamk = np.ascontiguousarray(np.broadcast_to(np.asarray(relaxpar, np.float64), (K,)))
        relaxpar = float(lamk[0])
    o = _lib.SirtOpts()
    o.method = code
    o.relax_kind = _lib.RELAX_CONST
    o.relaxpar = float(relaxpar)
    o.stoprule = _lib.STOP["DP" if taudelta is not None else "NONE"]
    o.lb_kind, o.lb = _bounds(lbound)
    o.ub_kind, o.ub = _bounds(ubound)
    o.kmax = int(kmax)
    td = None if taudelta is None else np.ascontiguousarray(
        np.broadcast_to(np.asarray(taudelta, dtype=np.float64), (K,)))
    fin = np.zeros(K, np.int64)
    rule = np.zeros(K, np.int32)
    ms = C.c_double()
    Ks = None if save is None else np.ascontiguousarray(save, np.int64)
    check(L.airt_sirt_multi_device(op.handle, C.byref(o), int(K), C.c_void_p(d_B),
                                   C.c_void_p(d_X0 or None), dptr(td), dptr(lamk),
                                   _lib.i64ptr(Ks), 0 if Ks is None else Ks.size,
                                   C.c_void_p(d_Xsave or None), C.c_void_p(d_X),
                                   _lib.i64ptr(fin), rule.ctypes.data_as(_ip), C.byref(ms)))
    return {"finaliter": fin, "stoprule": rule,
            "relaxpar": float(relaxpar) if lamk is None else lamk, "gpu_ms": float(ms.value)}
