"""Training of the relaxation parameter and of the DP/ME factor tau
(train/train_relaxpar.m, train/train_dpme.m) on the GPU solvers.

Every solve runs through libairt.  For the SIRT methods on a stored matrix
the independent solves are batched on the multi-right-hand-side engine
(airt_sirt_multi_device: the matrix read once per iteration for all of
them):
  * train_dpme: the s noise replicas run together, every iterate saved, and
    each replica's chunk-of-10 search for the error minimum is replayed on
    the saved errors (the iterates are those of the chunked restarts, which
    continue the same constant-relaxpar iteration);
  * train_relaxpar: the golden-section search evaluates, in one batch, every
    probe its next `depth` steps could ask for (2^(depth+1) - 2 relaxpar
    values, each with its own relaxpar), then walks the steps with the
    results -- the same decisions in depth-times fewer rounds.
ART and CART methods, and matrix-free operators, run the solves one after
another.  train_dpme's noise matrix comes from the caller (or a seeded
NumPy generator): MATLAB's randn stream cannot be reproduced.
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


def train_relaxpar(A, b, x_ex, method: str, kmax: int, options=None, batched: bool = True,
                   depth: int = 3) -> float:
    """relaxpar = train_relaxpar(A,b,x_ex,method,kmax,options)
    (train/train_relaxpar.m:75-270): the error-minimising iteration count in
    chunks of 10, then a golden-section search for the relaxpar with the
    fastest convergence to within 2% of the minimum error.  batched: the
    search's probes run `depth` steps ahead on the multi-right-hand-side
    engine (SIRT methods, stored matrix)."""
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
    if batched and is_sirt and _stored(A):
        return _golden_batched(A, b, x_ex, method, options, kopt, meub, relaxparmax, depth)

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


def _stored(A) -> bool:
    from .afun import as_operator
    return not as_operator(A).matrix_free


def _probe_errors(A, b, x_ex, method, options, lams, kopt):
    """For every relaxpar in lams: the SIRT iterates 1..kopt from zero (the
    options' rule otherwise; stoprule none) on the multi-right-hand-side
    engine, and their errors ||x_k - x_ex|| (a len(lams) x kopt array)."""
    import torch
    from .afun import as_operator
    from .batch import sirt_multi_device
    op = as_operator(A)
    K = len(lams)
    dB = torch.from_numpy(np.ascontiguousarray(np.broadcast_to(b, (K, b.size)))).cuda()
    dX = torch.empty((K, op.n), dtype=torch.float64, device="cuda")
    dS = torch.empty((kopt, K, op.n), dtype=torch.float64, device="cuda")
    lb, ub = options.get("lbound"), options.get("ubound")
    sirt_multi_device(op, method, dB.data_ptr(), dX.data_ptr(), K, kopt, relaxpar=np.asarray(lams),
                      lbound=None if lb is None else float(lb),
                      ubound=None if ub is None else float(ub), save=np.arange(1, kopt + 1),
                      d_Xsave=dS.data_ptr())
    xe = torch.from_numpy(x_ex).cuda()
    return torch.linalg.norm(dS - xe, dim=2).T.cpu().numpy()


def _golden_batched(A, b, x_ex, method, options, kopt, meub, relaxparmax, depth):
    """The golden-section search of train_relaxpar.m:131-200 (SIRT branch),
    with the probes of the next `depth` steps evaluated together."""
    r = (3 - math.sqrt(5)) / 2
    tol = relaxparmax * 0.01

    def kp_err(ee):
        kp = int(np.sum((ee[:-1] > meub) & (np.diff(ee) < 0))) + 1
        return kp, float(ee[kp - 1])

    alpha, beta = 0.0, relaxparmax
    alphap = alpha + r * (beta - alpha)
    betap = alpha + (1 - r) * (beta - alpha)
    E = _probe_errors(A, b, x_ex, method, options, [alphap, betap], kopt)
    (k_a, err_a), (k_b, err_b) = kp_err(E[0]), kp_err(E[1])

    def step(st, up):
        alpha, beta, alphap, betap = st
        if up:
            z = alphap + (1 - r) * abs(beta - alphap)
            return (alphap, beta, betap, z), z
        z = alpha + r * abs(betap - alpha)
        return (alpha, betap, z, alphap), z

    while abs(alphap - betap) > tol:
        # every probe the next `depth` steps can need: one per decision prefix
        probes, frontier = [], [((alpha, beta, alphap, betap), ())]
        for _ in range(depth):
            nxt = []
            for st, path in frontier:
                if abs(st[2] - st[3]) <= tol:
                    continue
                for up in (True, False):
                    st2, z = step(st, up)
                    probes.append((path + (up,), z))
                    nxt.append((st2, path + (up,)))
            frontier = nxt
        E = _probe_errors(A, b, x_ex, method, options, [z for _, z in probes], kopt)
        res = {path: kp_err(E[i]) for i, (path, _) in enumerate(probes)}
        path = ()
        for _ in range(depth):
            if abs(alphap - betap) <= tol:
                break
            move_up = err_a > meub
            move_down = (not move_up) and err_b > meub
            if not (move_up or move_down):
                move_up = k_a >= k_b
            path = path + (move_up,)
            (alpha, beta, alphap, betap), _ = step((alpha, beta, alphap, betap), move_up)
            if move_up:
                k_a, err_a = k_b, err_b
                k_b, err_b = res[path]
            else:
                k_b, err_b = k_a, err_a
                k_a, err_a = res[path]
    return (alphap + betap) / 2


def _dpme_batched(op, B, x_exact, method, type_, delta, kmax, options):
    """train_dpme for a SIRT method on a stored matrix: all replicas (columns
    of B) at once, every iterate 1..kmax saved, then each replica's chunked
    search for the error minimum replayed on its error sequence."""
    import torch
    from .afun import as_operator
    from .batch import sirt_multi_device
    op = as_operator(op)
    m, s = B.shape
    dB = torch.from_numpy(np.ascontiguousarray(B.T)).cuda()
    dX = torch.empty((s, op.n), dtype=torch.float64, device="cuda")
    dS = torch.zeros((kmax + 1, s, op.n), dtype=torch.float64, device="cuda")  # x_0 = 0
    rho = options.get("rho")
    lb, ub = options.get("lbound"), options.get("ubound")
    sirt_multi_device(op, method, dB.data_ptr(), dX.data_ptr(), s, kmax,
                      relaxpar=options.get("relaxpar"), rho=rho,
                      lbound=None if lb is None else float(lb),
                      ubound=None if ub is None else float(ub), save=np.arange(1, kmax + 1),
                      d_Xsave=dS[1:].data_ptr())
    xe = torch.from_numpy(x_exact).cuda()
    Eall = torch.linalg.norm(dS[1:] - xe, dim=2).T.cpu().numpy()   # s x kmax, iterations 1..kmax
    kstep = kmax if kmax < 10 else 10
    tauh = np.zeros(s)
    for i in range(s):
        k = kstep
        while True:
            I = int(np.argmin(Eall[i, :k])) + 1
            if I != k or k >= kmax:
                kopt = I
                break
            k = kmax if k + kstep > kmax else k + kstep
        bi = B[:, i]
        rk = bi - _apply(op, dS[kopt - 1, i].cpu().numpy())
        if type_.upper().startswith("DP"):
            tauh[i] = float(np.linalg.norm(rk)) / delta
        else:
            if kopt < 2:
                raise ValueError("ME needs the error minimum after the first iterate")
            rkm1 = bi - _apply(op, dS[kopt - 2, i].cpu().numpy())
            tauh[i] = 0.5 * float(rkm1 @ (rkm1 + rk)) / (delta * float(np.linalg.norm(rkm1)))
    return float(np.mean(tauh))


def train_dpme(A, b_exact, x_exact, method: str, type_: str, delta: float, s: int, kmax: int,
               options=None, E=None, seed: int = 0, batched: bool = True) -> float:
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
    if not (type_.upper().startswith("DP") or type_.upper().startswith("ME")):
        raise ValueError("The chosen type is invalid")
    if batched and method in SIRT_METHODS and _stored(A) and \
            (options.get("relaxpar") is None or np.isscalar(options.get("relaxpar"))):
        return _dpme_batched(op, B, x_exact, method, type_, delta, kmax, options)
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
            if kopt < 2:
                raise ValueError("ME needs the error minimum after the first iterate")
            rkm1 = bi - _apply(op, X[kopt - 2])
            tauk = 0.5 * float(rkm1 @ (rkm1 + rk)) / (delta * float(np.linalg.norm(rkm1)))
        else:
            raise ValueError("The chosen type is invalid")
        tauh[i] = tauk
    return float(np.mean(tauh))


def _apply(A, x):
    from .afun import as_operator
    return as_operator(A)(np.ascontiguousarray(x, np.float64), "notransp")
