"""sirt / art and their method wrappers, host side.

The host code keeps the reference's argument handling (auxil/check_inputs.m),
relaxation-parameter rules (auxil/calc_relaxpar.m) and output contract
(sirt/sirt.m:270-281, art/art.m:311-330); the iterations themselves run in
libairt on the GPU (airt_sirt / airt_art).  There is no CPU path.

Python conventions: K holds 1-based iteration numbers exactly as in MATLAB;
row indices (custom ART orders) are 0-based; options is a dict mirroring the
MATLAB options struct.
"""
from __future__ import annotations

import ctypes as C
import math
import time
import warnings

import numpy as np
import scipy.sparse as sp

from . import _lib
from ._lib import ArtOpts, CartOpts, Info, SirtOpts, check, dptr, i64ptr, lib
from .afun import AirtOperator, as_operator


class SolverResult(tuple):
    """(X, info) that also carries ``ext_info`` (sirt's third output)."""

    def __new__(cls, X, info, ext_info=None):
        self = super().__new__(cls, (X, info))
        self.X, self.info, self.ext_info = X, info, ext_info
        return self


# ------------------------------------------------------------ check_inputs
def _parse(A, b, K, x0, options, caller):
    """auxil/check_inputs.m:58-259 (host-side contract)."""
    options = dict(options or {})
    op = as_operator(A)
    m, n = op.m, op.n
    b = np.asarray(b, dtype=np.float64)
    if b.ndim > 1 and b.shape[1] != 1 or b.size != m:
        raise ValueError("The size of A and b do not match.")
    b = np.ascontiguousarray(b.ravel())
    if K is None or np.size(K) == 0:
        raise ValueError("Max no. of iterations must ALWAYS be specified.")
    K = np.atleast_1d(np.asarray(K)).astype(np.int64).ravel()
    if not np.all(np.diff(K) > 0):
        raise ValueError("Elements of K must be strictly increasing.")
    if x0 is None or np.size(x0) == 0:
        x0 = None
    else:
        x0 = np.asarray(x0, dtype=np.float64)
        if x0.size != n or (x0.ndim > 1 and x0.shape[1] != 1):
            raise ValueError("The size of x0 does not match the problem.")
        x0 = np.ascontiguousarray(x0.ravel())
    bounds = {}
    for key in ("lbound", "ubound"):
        v = options.get(key)
        if v is None:
            bounds[key] = (_lib.BOUND_NONE, 0.0, None)
            continue
        v = np.atleast_1d(np.asarray(v, dtype=np.float64)).ravel()
        if v.size == 1:
            bounds[key] = (_lib.BOUND_SCALAR, float(v[0]), None)
        elif v.size == n:
            bounds[key] = (_lib.BOUND_VECTOR, 0.0, np.ascontiguousarray(v))
        else:
            which = "lbound (lower bound)" if key == "lbound" else "ubound (upper bound)"
            raise ValueError(f"{which} must either be scalar or same length as vector of unknowns x.")
    sr = options.get("stoprule") or {}
    stype = str(sr.get("type", "NONE")).upper()
    taudelta = float("nan")
    if stype in ("DP", "ME"):
        td = sr.get("taudelta")
        if td is None or np.size(td) != 1 or not np.isscalar(np.asarray(td).item()):
            raise ValueError("For stopping rules DP and ME a scalar taudelta must be given in options.")
        taudelta = float(np.asarray(td).item())
    if stype == "NCP" and "res_dims" not in sr:
        raise ValueError("options.stoprule.res_dims must be specified for NCP stopping rule.")
    if stype not in ("DP", "ME", "NCP", "NONE"):
        raise ValueError("The chosen stopping rule is not valid.")
    if "res_dims" in sr and stype != "NCP":
        warnings.warn("options.stoprule.res_dims given but only used by NCP stopping rule, "
                      "not the one currently specified.")
    if stype == "ME" and caller != "sirt":
        raise ValueError("Stopping rule ME is only available for SIRT methods, not ART and CART.")
    ncp = None
    if stype == "NCP":
        # check_inputs.m:171-209, check_stoprules.m:100-122: a 1D res_dims means the
        # whole residual as one signal; a 2D one a column-major reshape
        rd = np.atleast_1d(np.asarray(sr["res_dims"])).astype(np.int64)
        if rd.size == 1:
            rows, cols = m, 1
        elif rd.size == 2:
            rows, cols = int(rd[0]), int(rd[1])
            if rows * cols != m:
                raise ValueError("To RESHAPE the number of elements must not change.")
        else:
            raise ValueError("NCP stopping rule only implemented for 1D and 2D residuals, the size "
                             "of which should be given using options.stoprule.res_dims.")
        smooth = int(sr.get("ncp_smooth", 2))
        ncp = (rows, cols, smooth)
    elif "ncp_smooth" in sr:
        warnings.warn("options.stoprule.ncp_smooth given but only used by NCP stopping rule, "
                      "not the one currently specified.")
    damp = float(options.get("damp", 0.0))
    if damp < 0:
        raise ValueError("Damping must be positive")
    verbose = int(options.get("verbose", 0) or 0)
    return dict(op=op, m=m, n=n, b=b, K=K, kmax=int(K[-1]), x0=x0, bounds=bounds, stype=stype,
                taudelta=taudelta, damp=damp, verbose=verbose, options=options, ncp=ncp)


def _bound_fields(o, bounds):
    lk, lv, lvec = bounds["lbound"]
    uk, uv, uvec = bounds["ubound"]
    o.lb_kind, o.lb, o.lbv = lk, lv, dptr(lvec)
    o.ub_kind, o.ub, o.ubv = uk, uv, dptr(uvec)


# ------------------------------------------------------------ calc_relaxpar
def calczeta(k):
    """Newton roots of (2k-1)z^(k-1) - (z^(k-2)+...+z+1) = 0 on [0,1]
    (calc_relaxpar.m:179-244: 6 Newton steps from z0 = 1, Horner)."""
    k = np.atleast_1d(np.asarray(k))
    if k.size and k[0] < 2:
        raise ValueError("The polynomial is not defined for k < 2")
    out = np.zeros(k.size)
    for i, kk in enumerate(k):
        coef = [0.0, 2.0 * kk - 1.0] + [-1.0] * int(kk - 1)

        def fung(x):
            f, df = coef[0], 0.0
            for cc in coef[1:]:
                df = df * x + f
                f = f * x + cc
            return f, df
        x = 1.0
        f, df = fung(x)
        h = f / df
        for _ in range(6):
            x -= h
            f, df = fung(x)
            h = f / df
        out[i] = x
    return out


def _relax_sirt(relaxparinput, rho, kmax):
    """SIRT branch of calc_relaxpar.m:105-165 given rho: (kind, value, table)."""
    if relaxparinput is None or (isinstance(relaxparinput, (list, np.ndarray)) and
                                 np.size(relaxparinput) == 0):
        return _lib.RELAX_CONST, 1.9 / rho, None
    if not isinstance(relaxparinput, str):
        lam = float(relaxparinput)
        if lam <= 0 or lam >= 2 / rho:
            warnings.warn("The relaxpar value is outside the interval (0,%f)" % (2 / rho))
        return _lib.RELAX_CONST, lam, None
    s = relaxparinput.lower()
    if s.startswith("line"):
        return _lib.RELAX_LINE, float("nan"), None
    if s.startswith("psi1") or s.startswith("psi2"):
        kk = np.arange(2, kmax)
        z = calczeta(kk) if kk.size else np.zeros(0)
        if s.startswith("psi1"):
            nu = 2.0 if s.startswith("psi1mod") else 1.0
            tail = nu * 2 * (1 - z)
        else:
            nu = 1.5 if s.startswith("psi2mod") else 1.0
            tail = nu * 2 * (1 - z) / ((1 - z ** kk) ** 2)
        table = np.concatenate([[math.sqrt(2), math.sqrt(2)], tail]) / rho
        return _lib.RELAX_TABLE, float("nan"), np.ascontiguousarray(table[:max(kmax, 0)])
    raise ValueError("The chosen relaxation strategy is not valid for this method.")


def _method_code(sirt_method, m, n):
    """get_mfun_dfun.m dispatch: (code, M, D, name, M_full, D_full).  A custom
    struct's M and D become diagonals when they are vectors or diagonal
    matrices (Mflag/Dflag 1, get_mfun_dfun.m:256-271) and stay full
    column-major matrices otherwise (flag 2, applied as dense products on the
    device)."""
    if sirt_method is None:
        sirt_method = "sart"
    if isinstance(sirt_method, str):
        if sirt_method not in _lib.METHODS:
            raise ValueError("SIRT method not defined.")
        return _lib.METHODS[sirt_method], None, None, sirt_method, False, False
    if isinstance(sirt_method, dict):
        out, full = [], []
        for key, size in (("M", m), ("D", n)):
            W = sirt_method.get(key)
            if W is None or np.size(W) == 0:
                out.append(None)
                full.append(False)
                continue
            if sp.issparse(W):
                W = sp.csr_matrix(W, dtype=np.float64)
                if min(W.shape) == 1:
                    W = W.toarray()
                elif (W - sp.diags(W.diagonal(), shape=W.shape)).count_nonzero() == 0:
                    W = np.ascontiguousarray(W.diagonal())
                else:
                    W = W.toarray()
            if not np.issubdtype(np.asarray(W).dtype, np.number):
                raise ValueError(f"{key} must be given as an array, either of dimension 0, 1 or 2.")
            W = np.asarray(W, dtype=np.float64)
            if W.ndim > 2:
                raise ValueError(f"{key} must be given as an array, either of dimension 0, 1 or 2.")
            if W.ndim <= 1 or min(W.shape) == 1:
                v, f = W.ravel(), False
            elif np.count_nonzero(W - np.diag(np.diag(W))) == 0:
                v, f = np.diag(W).copy(), False
            else:
                if W.shape != (size, size):
                    raise ValueError(f"custom {key} has the wrong size")
                v, f = np.asfortranarray(W), True
            if not f and v.size != size:
                raise ValueError(f"custom {key} has the wrong size")
            out.append(v if f else np.ascontiguousarray(v))
            full.append(f)
        return _lib.AIRT_CUSTOM, out[0], out[1], "custom", full[0], full[1]
    raise ValueError("First input must be a string with the SIRT method name or a struct "
                     "with fields M and D characterizing a custom method.")


def _fptr(a):
    """Pointer to a 1-D array or to a Fortran-ordered (column-major) matrix."""
    if a is None:
        return None
    if a.ndim == 2:
        assert a.flags.f_contiguous and a.dtype == np.float64
        return a.ctypes.data_as(_lib._dp)
    return dptr(a)


def _print_verbose(verbose, kmax, resn, lams, total_s, k_final):
    width = max(1, math.ceil(math.log10(kmax))) if kmax > 0 else 1
    per = total_s / max(k_final, 1)
    for k in range(1, k_final + 1):
        if verbose == 1 or (verbose > 1 and (k == 1 or k == k_final or k % verbose == 1)):
            print(f"{k:{width}d}/{kmax}:  resnorm={resn[k]:1.2e}  relaxpar={lams[k - 1]:1.2e}  "
                  f"time(iter/total)={per:1.2e}/{per * k:1.2e} secs.")


# ------------------------------------------------------------------- SIRT
def sirt(sirt_method, A, b, K, x0=None, options=None):
    """[X,info,ext_info] = sirt(sirt_method,A,b,K,x0,options)  (sirt/sirt.m:1).

    Returns a SolverResult that unpacks as (X, info) and carries ext_info.
    """
    t_total = time.perf_counter()
    c = _parse(A, b, K, x0, options, "sirt")
    op: AirtOperator = c["op"]
    m, n, K, kmax = c["m"], c["n"], c["K"], c["kmax"]
    code, Mv, Dv, name, Mfull, Dfull = _method_code(sirt_method, m, n)
    opts = c["options"]
    rho = opts.get("rho", float("nan"))
    rho = float("nan") if rho is None else float(rho)
    if name == "sart":
        rho = 1.0                                   # sirt.m:166-168
    if math.isnan(rho):
        r = C.c_double()
        if Mfull or Dfull:
            check(lib().airt_rho_custom(op.handle, _fptr(Mv), int(Mfull), _fptr(Dv), int(Dfull),
                                        1e-7, 1000, C.byref(r)))
        else:
            check(lib().airt_rho(op.handle, code, dptr(Mv), dptr(Dv), 1e-7, 200, C.byref(r)))
        rho = float(r.value)
    kind, lam, table = _relax_sirt(opts.get("relaxpar"), rho, kmax)

    o = SirtOpts()
    o.method = code
    o.M, o.D = _fptr(Mv), _fptr(Dv)
    o.M_full, o.D_full = int(Mfull), int(Dfull)
    o.relax_kind, o.relaxpar = kind, (lam if kind == _lib.RELAX_CONST else 0.0)
    o.relax_table = dptr(table)
    o.stoprule = _lib.STOP[c["stype"]]
    o.taudelta = c["taudelta"]
    if c["ncp"] is not None:
        o.ncp_rows, o.ncp_cols, o.ncp_smooth = c["ncp"]
    _bound_fields(o, c["bounds"])
    o.kmax = kmax
    X = np.zeros((n, K.size), dtype=np.float64, order="F")
    resn = np.zeros(kmax + 1)
    info = Info()
    check(lib().airt_sirt(op.handle, C.byref(o), dptr(c["b"]), dptr(c["x0"]), i64ptr(K), K.size,
                          X.ctypes.data_as(_lib._dp), dptr(resn), C.byref(info)))
    fin = int(info.finaliter)
    X = X[:, :int(info.nsaved)]
    relaxpar_out = float(info.relaxpar) if fin > 0 else opts.get("relaxpar")
    if fin > 0 and kind == _lib.RELAX_CONST:
        relaxpar_out = lam
    res_info = {
        "stoprule": int(info.stoprule),
        "finaliter": fin,
        "relaxpar": relaxpar_out,
        "rho": rho,
        "itersaved": np.concatenate([K[K < fin], [fin]]),
        "timetaken": time.perf_counter() - t_total,
        "gpu_ms": float(info.gpu_ms),
        "resnorms": resn[:fin + 1],
    }
    if c["verbose"]:
        lams = np.full(fin, lam) if kind == _lib.RELAX_CONST else (
            table[:fin] if kind == _lib.RELAX_TABLE else np.full(fin, float("nan")))
        _print_verbose(c["verbose"], kmax, resn, lams, res_info["timetaken"], fin)
    if code == _lib.AIRT_CUSTOM:
        ext = {"M": np.ones(m) if Mv is None else Mv, "D": np.ones(n) if Dv is None else Dv}
    else:
        Mw, Dw = op.weights(name)
        ext = {"M": Mw, "D": Dw}
    return SolverResult(X, res_info, ext)


def landweber(A, b, K, x0=None, options=None):
    """sirt/landweber.m:119."""
    return sirt("landweber", A, b, K, x0, options)


def cimmino(A, b, K, x0=None, options=None):
    """sirt/cimmino.m:121."""
    return sirt("cimmino", A, b, K, x0, options)


def cav(A, b, K, x0=None, options=None):
    """sirt/cav.m:122."""
    return sirt("cav", A, b, K, x0, options)


def drop(A, b, K, x0=None, options=None):
    """sirt/drop.m:122."""
    return sirt("drop", A, b, K, x0, options)


def sart(A, b, K, x0=None, options=None):
    """sirt/sart.m:129."""
    return sirt("sart", A, b, K, x0, options)


# -------------------------------------------------------------------- ART
def art(art_method, A, b, K, x0=None, options=None):
    """[X,info] = art(art_method,A,b,K,x0,options)  (art/art.m:1).

    art_method: 'kaczmarz', 'symkaczmarz', 'randkaczmarz' or a 0-based row
    order.  randkaczmarz draws its rows from a NumPy generator seeded with
    options['seed'] (default 0): one permutation per sweep and, when the row
    norms are not nearly uniform, one uniform number per step
    (art.m:208-219,241-262).
    """
    t_total = time.perf_counter()
    if art_method is None:
        art_method = "kaczmarz"
    c = _parse(A, b, K, x0, options, "art")
    op: AirtOperator = c["op"]
    m, n, K, kmax = c["m"], c["n"], c["K"], c["kmax"]
    opts = c["options"]
    sym = isinstance(art_method, str) and art_method.lower().startswith("sym")
    Kint = K
    if sym:
        if np.any(K % 2):
            raise ValueError("For symkaczmarz only even iteration numbers can be requested.")
        Kint = K // 2
        kmax = kmax // 2

    relin = opts.get("relaxpar")
    if relin is None:
        lam = 1.0
    elif callable(relin):
        lam = -1000.0
    elif np.isscalar(relin) or np.size(relin) == 1:
        lam = float(np.asarray(relin).item())
        if lam <= 0 or lam >= 2:
            warnings.warn("The relaxpar value is outside the interval (0,2)")
    else:
        raise ValueError("For ART methods the relaxpar must be a scalar or function handle.")

    o = ArtOpts()
    rows = lam_rows = None
    need_norms = callable(relin) or not isinstance(art_method, str) or \
        art_method.lower() == "randkaczmarz"
    normAi = None
    if need_norms:
        Mw, _ = op.weights("drop")               # 1/||a_i||^2, 0 for empty rows
        with np.errstate(divide="ignore"):
            normAi = np.where(Mw > 0, 1.0 / Mw, 0.0)
    if isinstance(art_method, str):
        mth = art_method.lower()
        if mth == "kaczmarz":
            o.order_kind = 0
        elif mth == "symkaczmarz":
            o.order_kind = 1
        elif mth == "randkaczmarz":
            o.order_kind = 2
            if opts.get("row_stream") is not None:
                rows = np.atleast_2d(np.asarray(opts["row_stream"], dtype=np.int64))
                lam_rows = rows
                if rows.shape[0] != kmax:
                    raise ValueError("row_stream must hold one row list per sweep")
            else:
                rows, lam_rows = _randk_stream(normAi, c["damp"], kmax, int(opts.get("seed", 0)))
            o.rows_stride = rows.shape[1]
        else:
            raise ValueError("Unknown ART method specified")
    else:
        o.order_kind = 2
        order = np.asarray(art_method, dtype=np.int64).ravel()
        rows = lam_rows = order[normAi[order] > 0]
        o.rows_stride = 0
    if rows is not None:
        rows = np.ascontiguousarray(rows, dtype=np.int64)
        o.rows = i64ptr(rows)
        o.nrows = rows.shape[-1]
    table = None
    if callable(relin):
        table = _art_lambda_table(relin, art_method, normAi, lam_rows, kmax, m)
        o.relax_table = dptr(table)
    o.relaxpar = lam
    o.damp = c["damp"]
    o.stoprule = _lib.STOP[c["stype"]]
    o.taudelta = c["taudelta"]
    if c["ncp"] is not None:
        o.ncp_rows, o.ncp_cols, o.ncp_smooth = c["ncp"]
    _bound_fields(o, c["bounds"])
    o.kmax = kmax
    X = np.zeros((n, Kint.size), dtype=np.float64, order="F")
    resn = np.zeros(kmax + 1)
    info = Info()
    check(lib().airt_art(op.handle, C.byref(o), dptr(c["b"]), dptr(c["x0"]), i64ptr(Kint),
                         Kint.size, X.ctypes.data_as(_lib._dp), dptr(resn), C.byref(info)))
    fin = int(info.finaliter)
    X = X[:, :int(info.nsaved)]
    Kout = Kint
    if sym:
        fin *= 2
        Kout = 2 * Kint
    res_info = {
        "stoprule": int(info.stoprule),
        "finaliter": fin,
        "relaxpar": float(info.relaxpar) if callable(relin) else (relin if fin == 0 and relin is not None else lam),
        "itersaved": np.concatenate([Kout[Kout < fin], [fin]]),
        "timetaken": time.perf_counter() - t_total,
        "gpu_ms": float(info.gpu_ms),
        "resnorms": resn[:int(info.finaliter) + 1],
    }
    if c["verbose"]:
        _print_verbose(c["verbose"], kmax, resn, np.full(kmax, lam), res_info["timetaken"],
                       int(info.finaliter))
    return SolverResult(X, res_info)


def cart(cart_method, A, b, K, x0=None, options=None):
    """[X,info] = cart(cart_method,A,b,K,x0,options)  (cart/cart.m:1).

    cart_method: 'columnaction' (None means the same) or a 0-based column
    order.  options as for art plus THR (default 1e-4), Kbegin (10) and
    Nunflag (round(kmax/4)); relaxpar is a scalar, default 0.25.  The
    unflagging draws randi(Nunflag) come from a counter-based generator
    seeded with options['seed'] (default 0), keyed by sweep and column.
    """
    t_total = time.perf_counter()
    if cart_method is None:
        cart_method = "columnaction"
    c = _parse(A, b, K, x0, options, "cart")
    op: AirtOperator = c["op"]
    n, K, kmax = c["n"], c["K"], c["kmax"]
    opts = c["options"]
    relin = opts.get("relaxpar")
    if relin is None:
        lam = 0.25
    elif (np.isscalar(relin) or np.size(relin) == 1) and not callable(relin):
        lam = float(np.asarray(relin).item())
        if lam <= 0 or lam >= 2:
            warnings.warn("The relaxpar value is outside the interval (0,2)")
    else:
        raise ValueError("For CART methods the relaxpar must be a scalar.")
    o = CartOpts()
    cols = None
    if isinstance(cart_method, str):
        if cart_method.lower() != "columnaction":
            raise ValueError("Unknown CART method specified")
        o.order_kind = 0
    else:
        o.order_kind = 2
        cols = np.ascontiguousarray(np.asarray(cart_method, dtype=np.int64).ravel())
        o.cols = i64ptr(cols)
        o.ncols = cols.size
    o.relaxpar = lam
    o.damp = c["damp"]
    o.stoprule = _lib.STOP[c["stype"]]
    o.taudelta = c["taudelta"]
    if c["ncp"] is not None:
        o.ncp_rows, o.ncp_cols, o.ncp_smooth = c["ncp"]
    _bound_fields(o, c["bounds"])
    o.kmax = kmax
    o.thr = float(opts.get("THR", 1e-4))
    o.kbegin = int(opts.get("Kbegin", 10))
    o.nunflag = int(opts["Nunflag"]) if "Nunflag" in opts else int(_mround(kmax / 4.0))
    o.seed = int(opts.get("seed", 0)) & 0xFFFFFFFFFFFFFFFF
    X = np.zeros((n, K.size), dtype=np.float64, order="F")
    resn = np.zeros(kmax + 1)
    info = Info()
    check(lib().airt_cart(op.handle, C.byref(o), dptr(c["b"]), dptr(c["x0"]), i64ptr(K), K.size,
                          X.ctypes.data_as(_lib._dp), dptr(resn), C.byref(info)))
    fin = int(info.finaliter)
    X = X[:, :int(info.nsaved)]
    res_info = {
        "stoprule": int(info.stoprule),
        "finaliter": fin,
        "relaxpar": lam,
        "itersaved": np.concatenate([K[K < fin], [fin]]),
        "timetaken": time.perf_counter() - t_total,
        "gpu_ms": float(info.gpu_ms),
        "resnorms": resn[:fin + 1],
    }
    if c["verbose"]:
        _print_verbose(c["verbose"], kmax, resn, np.full(kmax, lam), res_info["timetaken"], fin)
    return SolverResult(X, res_info)


def columnaction(A, b, K, x0=None, options=None):
    """cart/columnaction.m: cart('columnaction', ...)."""
    return cart("columnaction", A, b, K, x0, options)


def _mround(x: float) -> float:
    return math.copysign(math.floor(abs(x) + 0.5), x)


def _randk_stream(normAi, damp, kmax, seed):
    """Row stream of randkaczmarz (art.m:208-219,241-262): the rows executed
    and the rows whose index feeds a relaxpar handle, one (kmax, len(I))
    array each, one row per sweep."""
    m = normAi.size
    I = np.flatnonzero(normAi > 0)
    nd = normAi + damp * np.max(normAi)
    cumul = np.cumsum(nd / np.sum(nd))
    fast = np.max(np.abs(cumul - np.arange(1, m + 1) / m)) < 0.05
    rng = np.random.default_rng(seed)
    out = np.zeros((kmax, I.size), dtype=np.int64)
    lam_rows = np.zeros((kmax, I.size), dtype=np.int64)
    for k in range(kmax):
        I_torun = I[rng.permutation(I.size)]
        lam_rows[k] = I_torun
        if fast:
            out[k] = I_torun
        else:
            u = rng.random(I_torun.size)
            out[k] = np.minimum(np.searchsorted(cumul, u, side="left"), m - 1)
    return out, lam_rows


def _art_lambda_table(relin, art_method, normAi, rows, kmax, m):
    """Values of a relaxpar handle per row step: relaxpar((k-1)*m + i) with
    i the 1-based row index of the step (art.m:273-275)."""
    if isinstance(art_method, str) and art_method.lower() in ("kaczmarz", "symkaczmarz"):
        I = np.flatnonzero(normAi > 0)
        order = I if art_method.lower() == "kaczmarz" else np.concatenate([I, I[::-1]])
        per = [order] * kmax
    elif rows is not None and rows.ndim == 2:
        per = list(rows)
    else:
        per = [rows] * kmax
    tab = [np.array([relin((k * m) + int(i) + 1) for i in per[k]], dtype=np.float64)
           for k in range(kmax)]
    return np.ascontiguousarray(np.concatenate(tab) if tab else np.zeros(0))


def kaczmarz(A, b, K, x0=None, options=None):
    """art/kaczmarz.m:104."""
    return art("kaczmarz", A, b, K, x0, options)


def symkaczmarz(A, b, K, x0=None, options=None):
    """art/symkaczmarz.m:109."""
    return art("symkaczmarz", A, b, K, x0, options)


def randkaczmarz(A, b, K, x0=None, options=None):
    """art/randkaczmarz.m:106."""
    return art("randkaczmarz", A, b, K, x0, options)
