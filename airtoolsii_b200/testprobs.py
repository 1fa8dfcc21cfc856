"""Tomography test problems on the GPU: paralleltomo, fanlineartomo,
fancurvedtomo, seismictomo and sphericaltomo.

The host side prepares the per-angle and per-detector tables in FP64 exactly
as the reference does (cosd/sind of the angles, linspace ray offsets, the
fan's atand detector angles, the seismic source and receiver positions, the
cosines and sines of every circle sample of sphericaltomo);
libairt traces every ray on the device and
either stores A (FP32 CSR + CSC, bit-exact sparsity with the FP64 trace) or
keeps the geometry for matrix-free projection.

Also here: the reference's modified Shepp-Logan and tectonic phantoms and the
random-ellipse phantom family (same rasterisation grid as the Shepp-Logan
image, testprobs/phantomgallery.m:188-214).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check, dptr, lib
from .afun import AirtOperator


def _mround(x: float) -> float:
    return math.copysign(math.floor(abs(x) + 0.5), x)


def _trigd(x: float):
    """(cosd, sind) of one angle in degrees: exact 0/+-1 at multiples of 90,
    otherwise one cos/sin of the angle reduced to [-45, 45] degrees."""
    x = float(x)
    n = _mround(x / 90.0)
    r = x - 90.0 * n
    rad = r * (math.pi / 180.0)
    c, s = math.cos(rad), math.sin(rad)
    q = int(n) % 4
    cd, sd = ((c, s), (-s, c), (-c, -s), (s, -c))[q]
    return cd + 0.0, sd + 0.0


def cosd(x) -> np.ndarray:
    return np.array([_trigd(v)[0] for v in np.atleast_1d(np.asarray(x, float))])


def sind(x) -> np.ndarray:
    return np.array([_trigd(v)[1] for v in np.atleast_1d(np.asarray(x, float))])


def atand(x) -> np.ndarray:
    return np.array([(180.0 / math.pi) * math.atan(v) for v in np.atleast_1d(np.asarray(x, float))])


def _linspace(d1, d2, n):
    n = int(n)
    if n <= 0:
        return np.zeros(0)
    if n == 1:
        return np.array([float(d2)])
    y = d1 + (np.arange(n, dtype=float) * (d2 - d1)) / (n - 1)
    y[0], y[-1] = d1, d2
    return y


# ------------------------------------------------------------------ phantoms
_SHEPP = ((1, .69, .92, 0, 0, 0), (-.8, .6624, .8740, 0, -.0184, 0),
          (-.2, .1100, .3100, .22, 0, -18), (-.2, .1600, .4100, -.22, 0, 18),
          (.1, .2100, .2500, 0, .35, 0), (.1, .0460, .0460, 0, .1, 0),
          (.1, .0460, .0460, 0, -.1, 0), (.1, .0460, .0230, -.08, -.605, 0),
          (.1, .0230, .0230, 0, -.606, 0), (.1, .0230, .0460, .06, -.605, 0))


def ellipse_image(N: int, ellipses, clip_hi=None) -> np.ndarray:
    """Sum of filled ellipses (amplitude, a, b, x0, y0, phi[rad]) on the grid
    of phantomgallery.m:188-190; negatives set to 0, optional upper clip."""
    xn = (np.arange(N) - (N - 1) / 2.0) / ((N - 1) / 2.0)
    Xn = np.tile(xn, (N, 1))
    Yn = np.rot90(Xn)
    X = np.zeros((N, N))
    for A, ea, eb, x0, y0, phi in ellipses:
        x = Xn - x0
        y = Yn - y0
        cph, sph = math.cos(phi), math.sin(phi)
        inside = (((x * cph + y * sph) ** 2) / (ea * ea)
                  + ((y * cph - x * sph)) ** 2 / (eb * eb)) <= 1
        X[inside] += A
    X[X < 0] = 0
    if clip_hi is not None:
        X[X > clip_hi] = clip_hi
    return X


def phantomgallery(name: str, N: int) -> np.ndarray:
    """The 'shepplogan' (testprobs/phantomgallery.m:155-214) or 'tectonic'
    (phantomgallery.m:422-456) image, N x N."""
    if name == "shepplogan":
        return ellipse_image(N, [(a, b, c, d, e, f * math.pi / 180) for a, b, c, d, e, f in _SHEPP])
    if name == "tectonic":
        return tectonic(N)
    raise ValueError("only the 'shepplogan' and 'tectonic' phantoms are provided")


def tectonic(N: int) -> np.ndarray:
    """Two plates meeting at a sloped break (phantomgallery.m:422-456): the
    right plate at 0.75 with a stepped upper edge, the left plate at 1 whose
    rows shift down by one every second column across the break.  Raises
    ValueError for N whose index ranges leave the image (N < 10)."""
    N = int(N)
    n5, n13, n7, n20 = (int(_mround(N / k)) for k in (5, 13, 7, 20))
    X = np.zeros((N, N))

    def put(r0, r1, c0, c1, v):          # MATLAB X(r0:r1, c0:c1) = v, 1-based
        if r0 > r1 or c0 > c1:
            return
        if r0 < 1 or c0 < 1 or r1 > N or c1 > N:
            raise ValueError("tectonic phantom needs N >= 10")
        X[r0 - 1:r1, c0 - 1:c1] = v

    put(n5, n5 + n7, 5 * n13, N, 0.75)
    i = n5
    for j in range(1, n20 + 1, 2):      # the stepped edge of the right plate
        i -= 1
        put(i, i, 5 * n13 + j, N, 0.75)
    put(n5, 2 * n5, 1, 5 * n13, 1.0)
    lo = n5
    for j in range(5 * n13, min(12 * n13, N) + 1):
        if j % 2:
            lo += 1
        put(lo, lo + n5, j, j, 1.0)
    return X


def random_ellipses(N: int, count: int, seed: int, clip=(0.0, 1.0)) -> np.ndarray:
    """Random-ellipse phantom as x(:) (column-major): centres U[-0.6,0.6]^2,
    semi-axes U[0.05,0.4], rotation U[0,pi), intensity U[0.1,1], additive,
    clipped to [0,1]."""
    rng = np.random.default_rng(seed)
    ell = []
    for _ in range(count):
        cx, cy = rng.uniform(-0.6, 0.6, 2)
        a, b = rng.uniform(0.05, 0.4, 2)
        phi = rng.uniform(0.0, math.pi)
        amp = rng.uniform(0.1, 1.0)
        ell.append((amp, a, b, cx, cy, phi))
    X = ellipse_image(N, ell, clip_hi=clip[1])
    return X.ravel(order="F")


def add_noise(b: np.ndarray, eta: float, seed: int):
    """b + e with Gaussian e scaled to ||e|| = eta*||b|| (demo_stoprules.m:43-46).
    Returns (b_noisy, ||e||)."""
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(b.size)
    e = eta * np.linalg.norm(b) * e / np.linalg.norm(e)
    return b + e, float(np.linalg.norm(e))


# ------------------------------------------------------------------ geometries
def parallel_tables(N, theta=None, p=None, d=None):
    """paralleltomo.m:62-89,118,195-200: (theta, p, d, cos_t, sin_t, offsets)."""
    theta = np.arange(180.0) if theta is None else np.asarray(theta, float).ravel()
    if p is None:
        p = int(_mround(math.sqrt(2.0) * N))
    if d is None:
        d = p - 1
    return theta, int(p), float(d), cosd(theta), sind(theta), _linspace(-d / 2.0, d / 2.0, p)


def fan_tables(N, theta=None, p=None, R=None, dw=None, sd=None):
    """fanlineartomo.m:74-114,146-170: (theta, p, R, dw, sd, cos_t, sin_t,
    cos_w, sin_w) with R, dw, sd already multiplied by N."""
    sdv = (3.0 if sd is None else sd) * N
    dwv = (2.5 if dw is None else dw) * N
    Rv = (2.0 if R is None else R) * N
    if p is None:
        p = int(_mround(math.sqrt(2.0) * N))
    theta = np.arange(0.0, 359.0, 2.0) if theta is None else np.asarray(theta, float).ravel()
    if Rv < math.sqrt(2.0) / 2.0 * N:
        raise ValueError("R must be greater than half squareroot 2")
    dew = dwv / p
    if p % 2:
        depos = np.arange(1, (p - 1) // 2 + 1, dtype=float) * dew
        om = 90.0 - atand(sdv / depos)
        omega = np.concatenate([-om[::-1], [0.0], om])
    else:
        depos = (np.arange(1, p // 2 + 1, dtype=float) - 0.5) * dew
        om = 90.0 - atand(sdv / depos)
        omega = np.concatenate([-om[::-1], om])
    return theta, int(p), Rv, dwv, sdv, cosd(theta), sind(theta), cosd(omega), sind(omega)


def fancurved_tables(N, theta=None, p=None, R=None, d=None):
    """fancurvedtomo.m:102-140,161-175: (theta, p, R, d, cos_t, sin_t,
    cos_w, sin_w) with R multiplied by N; the arc detector's rays leave the
    source at omega = linspace(-d/2, d/2, p) degrees about the central ray
    (default d = 2*atand(1/(2R-1)), R = 2)."""
    Rn = 2.0 if R is None else float(R)
    if d is None:
        d = 2.0 * float(atand(1.0 / (2.0 * Rn - 1.0)))
    if p is None:
        p = int(_mround(math.sqrt(2.0) * N))
    theta = np.arange(0.0, 359.0, 2.0) if theta is None else np.asarray(theta, float).ravel()
    if Rn < math.sqrt(2.0) / 2.0:
        raise ValueError("R must be greater than half squareroot 2")
    if d < 0 or d > 180:
        raise ValueError("The angle of the source must be in the interval [0 180]")
    omega = _linspace(-d / 2.0, d / 2.0, int(p))
    return theta, int(p), Rn * N, float(d), cosd(theta), sind(theta), cosd(omega), sind(omega)


def seismic_tables(N, s=None, p=None):
    """seismictomo.m:67-75,98-116: (s, p, src_x, src_y, rcv_x, rcv_y).  s
    sources (default N) on the right edge at y = linspace(-N/2+Ns, N/2-Ns, s);
    p receivers (default 2N): floor(p/2) on the left edge, then ceil(p/2) on
    the top edge, each set at the centres of equal intervals."""
    N = int(N)
    if s is not None and np.size(s) > 1:
        raise ValueError("s must be a scaler")
    s = N if s is None else int(np.asarray(s).ravel()[0])
    p = 2 * N if p is None else int(p)
    h = N / 2.0
    ns = (N / s) / 2.0 if s else math.inf
    p1, p2 = -(-p // 2), p // 2
    np1 = (N / p1) / 2.0 if p1 else math.inf
    np2 = (N / p2) / 2.0 if p2 else math.inf
    src_x = np.full(s, h)
    src_y = _linspace(-h + ns, h - ns, s)
    rcv_x = np.concatenate([np.full(p2, -h), _linspace(-h + np1, h - np1, p1)])
    rcv_y = np.concatenate([_linspace(-h + np2, h - np2, p2), np.full(p1, h)])
    return s, p, src_x, src_y, rcv_x, rcv_y


def seismic_operator(N, src_x, src_y, rcv_x, rcv_y, matrix_free=False) -> AirtOperator:
    sx = np.ascontiguousarray(src_x, np.float64)
    sy = np.ascontiguousarray(src_y, np.float64)
    rx = np.ascontiguousarray(rcv_x, np.float64)
    ry = np.ascontiguousarray(rcv_y, np.float64)
    if sx.size != sy.size or rx.size != ry.size:
        raise ValueError("source and receiver tables need matching x and y lengths")
    h = C.c_void_p()
    check(lib().airt_problem_seismic(int(N), sx.size, dptr(sx), dptr(sy), rx.size, dptr(rx),
                                     dptr(ry), int(bool(matrix_free)), C.byref(h)))
    return AirtOperator(h, "seismic", dict(N=N, s=sx.size, p=rx.size))


def _round_half_away(x):
    a = np.abs(x)
    f = np.floor(a)
    return np.copysign(f + ((a - f) >= 0.5), x)


def sphere_tables(N, angles=None, numCircles=None):
    """sphericaltomo.m:64-75,115-124,203-205: (angles, numCircles, cos_t,
    sin_t, radii, nphi, cos_k, sin_k).  Circle n of radius radii[n] =
    linspace(0,2,numCircles+1)(n+1) is sampled at k = (0:nphi[n])*dPhi,
    nphi = ceil((4*pi/dx)*radii), dPhi = 2*pi/nphi, dx = sqrt(2)/N; cos_k and
    sin_k hold cos(k), sin(k) circle after circle."""
    N = int(N)
    angles = np.arange(0.0, 359.0, 2.0) if angles is None else np.asarray(angles, float).ravel()
    nc = int(_round_half_away(math.sqrt(2.0) * N)) if numCircles is None else int(numCircles)
    radii = _linspace(0.0, 2.0, nc + 1)[1:]
    dx = math.sqrt(2.0) / N
    nphi = np.ceil((4.0 * math.pi / dx) * radii).astype(np.int64)
    dphi = 2.0 * math.pi / nphi
    k = np.concatenate([np.arange(int(q) + 1, dtype=float) * d for q, d in zip(nphi, dphi)]) \
        if nc else np.zeros(0)
    return angles, nc, cosd(angles), sind(angles), radii, nphi, np.cos(k), np.sin(k)


def sphere_operator(N, cos_t, sin_t, radii, nphi, cos_k, sin_k, matrix_free=False) -> AirtOperator:
    ct = np.ascontiguousarray(cos_t, np.float64)
    st = np.ascontiguousarray(sin_t, np.float64)
    rd = np.ascontiguousarray(radii, np.float64)
    nphi = np.ascontiguousarray(nphi, np.int64)
    ck = np.ascontiguousarray(cos_k, np.float64)
    sk = np.ascontiguousarray(sin_k, np.float64)
    if nphi.size != rd.size or ck.size != sk.size or ck.size != int(np.sum(nphi + 1)):
        raise ValueError("circle tables need one nphi per radius and nphi+1 samples per circle")
    h = C.c_void_p()
    check(lib().airt_problem_spherical(int(N), ct.size, dptr(ct), dptr(st), rd.size, dptr(rd),
                                       nphi.ctypes.data_as(C.POINTER(C.c_int64)), dptr(ck), dptr(sk),
                                       int(bool(matrix_free)), C.byref(h)))
    return AirtOperator(h, "spherical", dict(N=N, nA=ct.size, nc=rd.size))


def parallel_operator(N, cos_t, sin_t, offsets, matrix_free=False) -> AirtOperator:
    ct = np.ascontiguousarray(cos_t, np.float64)
    st = np.ascontiguousarray(sin_t, np.float64)
    off = np.ascontiguousarray(offsets, np.float64)
    h = C.c_void_p()
    check(lib().airt_problem_parallel(int(N), ct.size, dptr(ct), dptr(st), off.size, dptr(off),
                                      int(bool(matrix_free)), C.byref(h)))
    return AirtOperator(h, "parallel", dict(N=N, nA=ct.size, p=off.size))


def fan_operator(N, cos_t, sin_t, cos_w, sin_w, R, matrix_free=False) -> AirtOperator:
    ct = np.ascontiguousarray(cos_t, np.float64)
    st = np.ascontiguousarray(sin_t, np.float64)
    cw = np.ascontiguousarray(cos_w, np.float64)
    sw = np.ascontiguousarray(sin_w, np.float64)
    h = C.c_void_p()
    check(lib().airt_problem_fan(int(N), ct.size, dptr(ct), dptr(st), cw.size, dptr(cw), dptr(sw),
                                 float(R), int(bool(matrix_free)), C.byref(h)))
    return AirtOperator(h, "fan", dict(N=N, nA=ct.size, p=cw.size, R=R))


def paralleltomo(N, theta=None, p=None, d=None, isDisp=0, isMatrix=1):
    """[A,b,x,theta,p,d] = paralleltomo(N,theta,p,d,isDisp,isMatrix)
    (testprobs/paralleltomo.m:1).  A is an AirtOperator: the stored system
    matrix (isMatrix=1) or the matrix-free projector (isMatrix=0).  b = A*x for
    the Shepp-Logan phantom x.  isDisp (ray animation) is not supported."""
    theta, p, d, ct, st, off = parallel_tables(N, theta, p, d)
    A = parallel_operator(N, ct, st, off, matrix_free=not isMatrix)
    x = phantomgallery("shepplogan", N).ravel(order="F")
    b = A(x, "notransp")
    return A, b, x, theta, p, d


def fancurvedtomo(N, theta=None, p=None, R=None, d=None, isDisp=0, isMatrix=1):
    """[A,b,x,theta,p,R,d] = fancurvedtomo(N,theta,p,R,d,isDisp,isMatrix)
    (testprobs/fancurvedtomo.m:1): fan beam onto an arc detector; the same
    ray trace as fanlineartomo (no boundary exclusion).  R is returned in
    units of N, d in degrees."""
    theta, p, Rv, d, ct, st, cw, sw = fancurved_tables(N, theta, p, R, d)
    A = fan_operator(N, ct, st, cw, sw, Rv, matrix_free=not isMatrix)
    x = phantomgallery("shepplogan", N).ravel(order="F")
    b = A(x, "notransp")
    return A, b, x, theta, p, Rv / N, d


def seismictomo(N, s=None, p=None, isDisp=0, isMatrix=1):
    """[A,b,x,s,p] = seismictomo(N,s,p,isDisp,isMatrix)
    (testprobs/seismictomo.m:1): straight rays from s sources on the right
    edge to p receivers on the left and top edges (row i*p + j for source i,
    receiver j); x is the 'tectonic' phantom.  isDisp is not supported."""
    s, p, sx, sy, rx, ry = seismic_tables(N, s, p)
    A = seismic_operator(N, sx, sy, rx, ry, matrix_free=not isMatrix)
    x = phantomgallery("tectonic", N).ravel(order="F")
    b = A(x, "notransp")
    return A, b, x, s, p


def sphericaltomo(N, angles=None, numCircles=None, isDisp=0, isMatrix=1):
    """[A,b,x,angles,numCircles] = sphericaltomo(N,angles,numCircles,isDisp,isMatrix)
    (testprobs/sphericaltomo.m:1): spherical-means (circle) integrals about
    centres on the unit circle at the given angles; x is the Shepp-Logan
    phantom.  isDisp is not supported."""
    angles, nc, ct, st, radii, nphi, ck, sk = sphere_tables(N, angles, numCircles)
    A = sphere_operator(N, ct, st, radii, nphi, ck, sk, matrix_free=not isMatrix)
    x = phantomgallery("shepplogan", N).ravel(order="F")
    b = A(x, "notransp")
    return A, b, x, angles, nc


def fanlineartomo(N, theta=None, p=None, R=None, dw=None, sd=None, isDisp=0, isMatrix=1):
    """[A,b,x,theta,p,R,dw,sd] = fanlineartomo(N,theta,p,R,dw,sd,isDisp,isMatrix)
    (testprobs/fanlineartomo.m:1-2).  R, dw, sd are in units of N as in the
    reference; R is returned in units of N."""
    theta, p, Rv, dwv, sdv, ct, st, cw, sw = fan_tables(N, theta, p, R, dw, sd)
    A = fan_operator(N, ct, st, cw, sw, Rv, matrix_free=not isMatrix)
    x = phantomgallery("shepplogan", N).ravel(order="F")
    b = A(x, "notransp")
    return A, b, x, theta, p, Rv / N, dwv, sdv
