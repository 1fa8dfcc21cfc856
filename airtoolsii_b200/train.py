"""Training of the relaxation parameter and of the DP/ME factor tau
(train/train_relaxpar.m, train/train_dpme.m) on the GPU solvers.

Both are host loops of solves; every solve runs through libairt (sirt, art
and cart/columnaction of solvers.py).  train_dpme's noise matrix comes from the caller (or a
seeded NumPy generator): MATLAB's randn stream cannot be reproduced.
"""
from __future__ import annotations

import math

import numpy as np

from . import solvers

SIRT_METHODS = ("landweber", "cimmino", "cav", "drop", "sart")
ART_METHODS = ("kaczmarz", "symkaczmarz", "randkaczmarz")
CART_METHODS = ("columnaction",)


def _solve(method, A, b, K, x0, options):
    if method in SIRT_METHODS:
        X, info = solvers.sirt(method, A, b, K, x0, options)
    elif method in ART_METHODS or method in CART_METHODS:
        X, info = getattr(solvers, method)(A, b, K, x0, options)
    else:
        raise ValueError(f"Unknown method {method}")
    return np.asarray(X), info


def _colnorm_err(X, x_ex):
    return np.sqrt(np.sum((X - x_ex[:, None]) ** 2, axis=0))


def train_relaxpar(A, b, x_ex, method: str, kmax: int, options=None) -> float:
    """relaxpar = train_relaxpar(A,b,x_ex,method,kmax,options)
    (train/train_relaxpar.m:75-270): the error-minimising iteration count in
    chunks of 10, then a golden-section search for the relaxpar with the
    fastest convergence to within 2% of the minimum error."""
    x_ex = np.asarray(x_ex, np.float64).ravel()
    if options is not None:
        options = dict(options)
        options["stoprule"] = {"type": "none"}
        options.pop("relaxpar", None)
    else:
        options = {}
    fudge = 0.02
    stepk = 10
    K = list(range(1, stepk + 1))
    k = 0
    stop = False
    Er = np.zeros(0)
    x0 = None
    is_sirt = method in SIRT_METHODS
    relaxparmax = 2.0
    while not stop:
        if k + stepk > kmax:
            K = list(range(1, kmax - k + 1))
            k = kmax
        else:
            k = k + stepk
        if k <= stepk:
            if is_sirt:
                Xnew, info = _solve(method, A, b, K, x0, options)
                options["rho"] = info["rho"]
                relaxparmax = 2.0 / info["rho"]
            elif method in ART_METHODS or method in CART_METHODS:  # train_relaxpar.m:90
                options["relaxpar"] = 0.25
                Xnew, _ = _solve(method, A, b, K, x0, options)
                relaxparmax = 2.0
            else:
                raise ValueError(f"Unknown method {method}")
        else:
            Xnew, _ = _solve(method, A, b, K, x0, options)
        Er = np.concatenate([Er, _colnorm_err(Xnew, x_ex)])
        kopt = int(np.argmin(Er)) + 1
        minE = float(Er[kopt - 1])
        if kopt == k and k < kmax:
            x0 = Xnew[:, -1]
        else:
            stop = True
    meub = (1 + fudge) * minE

    def evaluate(p):
        options["relaxpar"] = p
        xnew, _ = _solve(method, A, b, list(range(1, kopt + 1)), None, options)
        ee = _colnorm_err(xnew, x_ex)
        kp = int(np.sum((ee[:-1] > meub) & (np.diff(ee) < 0))) + 1
        return kp, float(ee[kp - 1])

    r = (3 - math.sqrt(5)) / 2
    alpha, beta = 0.0, relaxparmax
    alphap = alpha + r * (beta - alpha)
    betap = alpha + (1 - r) * (beta - alpha)
    k_a, err_a = evaluate(alphap)
    k_b, err_b = evaluate(betap)
    while abs(alphap - betap) > relaxparmax * 0.01:
        # SIRT tests the alpha' error first, ART/CART the beta' error
        # (train_relaxpar.m:151-200 and 202-251)
        if is_sirt:
            move_up = err_a > meub
            move_down = (not move_up) and err_b > meub
        else:
            move_down = err_b > meub
            move_up = (not move_down) and err_a > meub
        if not (move_up or move_down):
            move_up = k_a >= k_b
        if move_up:
            z = alphap + (1 - r) * abs(beta - alphap)
            alpha, alphap, betap = alphap, betap, z
            k_a, err_a = k_b, err_b
            k_b, err_b = evaluate(betap)
        else:
            z = alpha + r * abs(betap - alpha)
            beta, betap, alphap = betap, alphap, z
            k_b, err_b = k_a, err_a
            k_a, err_a = evaluate(alphap)
    return (alphap + betap) / 2


def train_dpme(A, b_exact, x_exact, method: str, type_: str, delta: float, s: int, kmax: int,
               options=None, E=None, seed: int = 0) -> float:
    """tau = train_dpme(A,b_exact,x_exact,method,type,delta,s,kmax,options)
    (train/train_dpme.m:66-136): for s noise realisations of norm delta, the
    error-minimising iterate (chunks of 10 up to kmax) and the tau that the DP
    or ME rule would need to stop there; their mean.  E (m x s) replaces
    randn(m,s); without it a NumPy generator seeded with `seed` draws it.
    As in the reference, the residual is taken at X(:,kopt) of the iterate
    list [x0 = 0, x1, x2, ...], i.e. one iterate before the minimum."""
    options = dict(options or {})
    options["stoprule"] = {"type": "none"}
    b_exact = np.asarray(b_exact, np.float64).ravel()
    x_exact = np.asarray(x_exact, np.float64).ravel()
    m = b_exact.size
    if E is None:
        E = np.random.default_rng(seed).standard_normal((m, s))
    E = np.asarray(E, np.float64).reshape(m, s)
    e = delta * E / np.sqrt(np.sum(E * E, axis=0))[None, :]
    B = b_exact[:, None] + e
    op = A
    kstep = kmax if kmax < 10 else 10
    tauh = np.zeros(s)
    for i in range(s):
        bi = B[:, i]
        X = [np.zeros(x_exact.size)]
        x0 = None
        k = kstep
        K = list(range(1, k + 1))
        Ek = np.zeros(0)
        while True:
            Xny, _ = _solve(method, op, bi, K, x0, options)
            Ek = np.concatenate([Ek, _colnorm_err(Xny, x_exact)])
            X.extend(Xny[:, j] for j in range(Xny.shape[1]))
            I = int(np.argmin(Ek)) + 1
            if I != k or k >= kmax:
                kopt = I
                break
            if k + kstep > kmax:
                K = list(range(1, kmax - k + 1))
                k = kmax
            else:
                k = k + kstep
            x0 = Xny[:, -1]
        rk = bi - _apply(op, X[kopt - 1])
        if type_.upper().startswith("DP"):
            tauk = float(np.linalg.norm(rk)) / delta
        elif type_.upper().startswith("ME"):
            rkm1 = bi - _apply(op, X[kopt - 2])
            tauk = 0.5 * float(rkm1 @ (rkm1 + rk)) / (delta * float(np.linalg.norm(rkm1)))
        else:
            raise ValueError("The chosen type is invalid")
        tauh[i] = tauk
    return float(np.mean(tauh))


def _apply(A, x):
    from .afun import as_operator
    return as_operator(A)(np.ascontiguousarray(x, np.float64), "notransp")
