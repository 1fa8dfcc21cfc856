"""FP64 NumPy/SciPy restatement of the AIR Tools II hot path (test oracle).

TEST INFRASTRUCTURE ONLY -- the checker for the CUDA path, never the product.
Parity status: unpinned against MATLAB (no MATLAB/Octave here, no golden
vectors in the reference); pinned against the reference demos' invariants and
analytic known answers (see ``oracle/__init__.py``).

Every function cites the reference file:line (paths inside the AIR Tools II
tree) whose behaviour it restates.  Index conventions: rows/columns are
0-based here; iteration numbers K are 1-based counts exactly as in MATLAB.
"""
from __future__ import annotations

import math
import time

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

# ---------------------------------------------------------------------------
# MATLAB numeric helpers
# ---------------------------------------------------------------------------


def mround(x: float) -> float:
    """MATLAB ``round``: half away from zero."""
    return math.copysign(math.floor(abs(x) + 0.5), x)


def _trigd(x: float) -> tuple[float, float]:
    """(cosd(x), sind(x)) for a scalar in degrees.

    Multiples of 90 degrees give exact 0/+-1 as MATLAB's cosd/sind do; other
    arguments are reduced to [-45, 45] degrees by whole quadrants before one
    call of cos/sin on the radian value.  Zeros are returned as +0.
    """
    x = float(x)
    n = mround(x / 90.0)
    r = x - 90.0 * n
    rad = r * (math.pi / 180.0)
    c, s = math.cos(rad), math.sin(rad)
    q = int(n) % 4
    if q == 0:
        cd, sd = c, s
    elif q == 1:
        cd, sd = -s, c
    elif q == 2:
        cd, sd = -c, -s
    else:
        cd, sd = s, -c
    return cd + 0.0, sd + 0.0


def cosd(x):
    """Vectorised degree cosine (see ``_trigd``)."""
    return np.array([_trigd(v)[0] for v in np.atleast_1d(np.asarray(x, float))])


def sind(x):
    """Vectorised degree sine (see ``_trigd``)."""
    return np.array([_trigd(v)[1] for v in np.atleast_1d(np.asarray(x, float))])


def atand(x):
    """Degree arctangent, (180/pi)*atan(x)."""
    return np.array([(180.0 / math.pi) * math.atan(v)
                     for v in np.atleast_1d(np.asarray(x, float))])


def linspace(d1: float, d2: float, n: int) -> np.ndarray:
    """``linspace(d1,d2,n)``: d1 + k*(d2-d1)/(n-1) with exact end points."""
    n = int(n)
    if n <= 0:
        return np.zeros(0)
    if n == 1:
        return np.array([float(d2)])
    k = np.arange(n, dtype=float)
    y = d1 + (k * (d2 - d1)) / (n - 1)
    y[0] = d1
    y[-1] = d2
    return y


# ---------------------------------------------------------------------------
# Ray tracing: testprobs/paralleltomo.m:186-278, testprobs/fanlineartomo.m:
# 230-320.  One ray = one row of A.
# ---------------------------------------------------------------------------


def trace_ray(N: int, x0t: float, y0t: float, a: float, b: float,
              exclude_top_right: bool):
    """Pixel indices (0-based, column-major image) and lengths of one ray.

    Restates paralleltomo.m:207-263 (and fanlineartomo.m:271-318 with
    ``exclude_top_right=False``): intersections with x = const and y = const
    grid lines, a stable ascending sort by the line parameter t (NaN last),
    the box filter, removal of a point whose successor lies within 1e-10 in
    both coordinates, segment lengths sqrt(dx^2+dy^2) and the midpoint cell
    index floor(xm)*N + (N - floor(ym)) (1-based in MATLAB; minus one here).
    """
    g = np.arange(-N / 2.0, N / 2.0 + 0.5, 1.0)  # (-N/2:N/2)'
    with np.errstate(divide="ignore", invalid="ignore"):
        tx = (g - x0t) / a
        yx = b * tx + y0t
        ty = (g - y0t) / b
        xy = a * ty + x0t
    t = np.concatenate([tx, ty])
    xxy = np.concatenate([g, xy])
    yxy = np.concatenate([yx, g])
    order = np.argsort(t, kind="stable")  # MATLAB sort: stable, NaN last
    xxy = xxy[order]
    yxy = yxy[order]
    h = N / 2.0
    keep = (xxy >= -h) & (xxy <= h) & (yxy >= -h) & (yxy <= h)
    xxy = xxy[keep]
    yxy = yxy[keep]
    if xxy.size > 1:
        dup = (np.abs(np.diff(xxy)) <= 1e-10) & (np.abs(np.diff(yxy)) <= 1e-10)
        keep2 = np.ones(xxy.size, dtype=bool)
        keep2[:-1] = ~dup
        xxy = xxy[keep2]
        yxy = yxy[keep2]
    dx = np.diff(xxy)
    dy = np.diff(yxy)
    aval = np.sqrt(dx * dx + dy * dy)
    if aval.size == 0:
        return np.zeros(0, np.int64), np.zeros(0)
    if exclude_top_right and ((b == 0 and abs(y0t - N / 2.0) < 1e-15) or
                              (a == 0 and abs(x0t - N / 2.0) < 1e-15)):
        return np.zeros(0, np.int64), np.zeros(0)
    xm = 0.5 * (xxy[:-1] + xxy[1:]) + N / 2.0
    ym = 0.5 * (yxy[:-1] + yxy[1:]) + N / 2.0
    col1 = np.floor(xm) * N + (N - np.floor(ym))
    return col1.astype(np.int64) - 1, aval


def parallel_geometry(N: int, theta=None, p=None, d=None):
    """Defaults and per-angle tables of paralleltomo.m:62-89, 114-123, 195-200.

    Returns (theta, p, d, cos_t, sin_t, offsets) where offsets is
    linspace(-d/2, d/2, p).
    """
    theta = np.arange(180.0) if theta is None else np.asarray(theta, float).ravel()
    if p is None:
        p = int(mround(math.sqrt(2.0) * N))
    if d is None:
        d = p - 1
    cos_t = cosd(theta)
    sin_t = sind(theta)
    offsets = linspace(-d / 2.0, d / 2.0, p)
    return theta, int(p), float(d), cos_t, sin_t, offsets


def parallel_rays(N, cos_t, sin_t, offsets):
    """Yield (row, x0theta, y0theta, a, b) per ray, paralleltomo.m:186-200."""
    p = len(offsets)
    for i in range(len(cos_t)):
        c, s = float(cos_t[i]), float(sin_t[i])
        a, b = -s, c
        for j in range(p):
            x0 = float(offsets[j])
            x0t = c * x0 - s * 0.0
            y0t = s * x0 + c * 0.0
            yield i * p + j, x0t, y0t, a, b


def fan_geometry(N: int, theta=None, p=None, R=2.0, dw=2.5, sd=3.0):
    """Defaults and tables of fanlineartomo.m:74-114, 146-170.

    Returns (theta, p, Rabs, dwabs, sdabs, cos_t, sin_t, cos_w, sin_w).
    """
    sdv = sd * N
    dwv = dw * N
    Rv = R * N
    if p is None:
        p = int(mround(math.sqrt(2.0) * N))
    theta = (np.arange(0.0, 359.0, 2.0) if theta is None
             else np.asarray(theta, float).ravel())
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
    return (theta, int(p), Rv, dwv, sdv, cosd(theta), sind(theta),
            cosd(omega), sind(omega))


def fancurved_geometry(N: int, theta=None, p=None, R=2.0, d=None):
    """Defaults and tables of fancurvedtomo.m:102-140, 161-175: an arc
    detector, ray angles omega = linspace(-d/2, d/2, p) degrees about the
    central ray.  Returns (theta, p, Rabs, d, cos_t, sin_t, cos_w, sin_w)."""
    if d is None:
        d = 2.0 * float(atand(1.0 / (2.0 * R - 1.0)))
    if p is None:
        p = int(mround(math.sqrt(2.0) * N))
    theta = (np.arange(0.0, 359.0, 2.0) if theta is None
             else np.asarray(theta, float).ravel())
    if R < math.sqrt(2.0) / 2.0:
        raise ValueError("R must be greater than half squareroot 2")
    if d < 0 or d > 180:
        raise ValueError("The angle of the source must be in the interval [0 180]")
    omega = linspace(-d / 2.0, d / 2.0, p)
    return (theta, int(p), R * N, float(d), cosd(theta), sind(theta), cosd(omega), sind(omega))


def fan_rays(N, R, cos_t, sin_t, cos_w, sin_w):
    """Yield (row, x0theta, y0theta, a, b) per ray, fanlineartomo.m:230-257.

    The 2-element matrix products are evaluated as two rounded products and
    one rounded sum (no fused multiply-add).
    """
    p = len(cos_w)
    for i in range(len(cos_t)):
        c, s = float(cos_t[i]), float(sin_t[i])
        x0t = c * 0.0 + (-s) * R
        y0t = s * 0.0 + c * R
        ab1 = (-x0t) / R
        ab2 = (-y0t) / R
        for j in range(p):
            cw, sw = float(cos_w[j]), float(sin_w[j])
            a = cw * ab1 + (-sw) * ab2
            b = sw * ab1 + cw * ab2
            yield i * p + j, x0t, y0t, a, b


def seismic_geometry(N: int, s=None, p=None):
    """Sources and receivers of seismictomo.m:67-75, 98-116: s (default N)
    sources at x0 = N/2, y0 = linspace(-N/2+Ns, N/2-Ns, s), Ns = (N/s)/2;
    p (default 2N) receivers, p2 = floor(p/2) at x = -N/2 with y =
    linspace(-N/2+Np2, N/2-Np2, p2), then p1 = ceil(p/2) at y = N/2 with
    x = linspace(-N/2+Np1, N/2-Np1, p1).  Returns (s, p, x0, y0, xp, yp)."""
    s = N if s is None else int(s)
    p = 2 * N if p is None else int(p)
    N2 = N / 2.0
    Ns = (N / s) / 2.0
    x0 = N2 * np.ones(s)
    y0 = linspace(-N2 + Ns, N2 - Ns, s)
    p1 = int(math.ceil(p / 2.0))
    p2 = int(math.floor(p / 2.0))
    Np1 = (N / p1) / 2.0 if p1 > 0 else math.inf
    Np2 = (N / p2) / 2.0 if p2 > 0 else math.inf
    xp = np.concatenate([-N2 * np.ones(p2), linspace(-N2 + Np1, N2 - Np1, p1)])
    yp = np.concatenate([linspace(-N2 + Np2, N2 - Np2, p2), N2 * np.ones(p1)])
    return s, p, x0, y0, xp, yp


def seismic_rays(x0, y0, xp, yp):
    """Yield (row, x0(i), y0(i), a(j), b(j)) per ray, seismictomo.m:188-200:
    a = xp - x0(i), b = yp - y0(i), row (i-1)*p + j (0-based here)."""
    p = len(xp)
    for i in range(len(x0)):
        a = xp - x0[i]
        b = yp - y0[i]
        for j in range(p):
            yield i * p + j, float(x0[i]), float(y0[i]), float(a[j]), float(b[j])


def seismictomo_matrix(N, s=None, p=None) -> sp.csc_matrix:
    """System matrix of seismictomo.m:96-287 (isMatrix=1)."""
    s, p, x0, y0, xp, yp = seismic_geometry(N, s, p)
    rows, cols, vals = trace_coo(N, seismic_rays(x0, y0, xp, yp), False)
    return coo_to_csc(rows, cols, vals, s * p, N * N)


def mround_array(x) -> np.ndarray:
    """MATLAB ``round`` on an array: nearest integer, halves away from zero
    (x - floor(x) is exact for the magnitudes used here)."""
    x = np.asarray(x, float)
    a = np.abs(x)
    f = np.floor(a)
    r = f + ((a - f) >= 0.5)
    return np.copysign(r, x)


def sphere_geometry(N: int, angles=None, numCircles=None):
    """sphericaltomo.m:64-75, 115-124: angles (default 0:2:358), numCircles
    (default round(sqrt(2)*N)), radii = linspace(0,2,numCircles+1)(2:end),
    centerImg = ceil(N/2), dx = sqrt(2)/N, nPhi = ceil((4*pi/dx)*radii),
    dPhi = 2*pi./nPhi.  Returns (angles, numCircles, radii, nPhi, dPhi,
    centerImg, dx)."""
    angles = np.arange(0.0, 359.0, 2.0) if angles is None else np.asarray(angles, float).ravel()
    nc = int(mround(math.sqrt(2.0) * N)) if numCircles is None else int(numCircles)
    radii = linspace(0.0, 2.0, nc + 1)[1:]
    center = int(math.ceil(N / 2.0))
    dx = math.sqrt(2.0) / N
    nphi = np.ceil((4.0 * math.pi / dx) * radii).astype(np.int64)
    dphi = 2.0 * math.pi / nphi
    return angles, nc, radii, nphi, dphi, center, dx


def sphere_circle_tables(nphi, dphi):
    """cos(k), sin(k) of k = (0:nPhi(n))*dPhi(n), sphericaltomo.m:203-205,
    concatenated circle after circle."""
    ks = [np.arange(int(n) + 1, dtype=float) * d for n, d in zip(nphi, dphi)]
    k = np.concatenate(ks) if ks else np.zeros(0)
    return np.cos(k), np.sin(k)


def sphericaltomo_matrix(N, angles=None, numCircles=None) -> sp.csc_matrix:
    """System matrix of sphericaltomo.m:108-270 (isMatrix=1): per circle the
    samples' pixels, unique(J) and histc counts w, values
    (2*pi*radii(n)/nPhi(n))*w; row (m-1)*numCircles + n."""
    angles, nc, radii, nphi, dphi, center, dx = sphere_geometry(N, angles, numCircles)
    ck, sk = sphere_circle_tables(nphi, dphi)
    off = np.concatenate([[0], np.cumsum(nphi + 1)])
    xi_c, xi_s = cosd(angles), sind(angles)
    R, Cc, V = [], [], []
    for m in range(len(angles)):
        for n in range(nc):
            c, s_ = ck[off[n]:off[n + 1]], sk[off[n]:off[n + 1]]
            xx = (xi_c[m] + radii[n] * c) / dx + center
            yy = (xi_s[m] + radii[n] * s_) / dx + center
            col = mround_array(xx)
            row = mround_array(yy)
            keep = (col > 0) & (col <= N) & (row > 0) & (row <= N)
            J = (N - row[keep] + 1) + (col[keep] - 1) * N
            Ju, w = np.unique(J, return_counts=True)
            if Ju.size:
                R.append(np.full(Ju.size, m * nc + n, np.int64))
                Cc.append(Ju.astype(np.int64) - 1)
                V.append((2.0 * math.pi * radii[n] / nphi[n]) * w.astype(float))
    if not R:
        return sp.csc_matrix((len(angles) * nc, N * N))
    return coo_to_csc(np.concatenate(R), np.concatenate(Cc), np.concatenate(V),
                      len(angles) * nc, N * N)


def trace_coo(N, rays, exclude_top_right):
    """COO triplets of all rays in row order (the rows/cols/vals buffers of
    paralleltomo.m:266-278)."""
    R, C, V = [], [], []
    for row, x0t, y0t, a, b in rays:
        cols, vals = trace_ray(N, x0t, y0t, a, b, exclude_top_right)
        if cols.size:
            R.append(np.full(cols.size, row, np.int64))
            C.append(cols)
            V.append(vals)
    if not R:
        return np.zeros(0, np.int64), np.zeros(0, np.int64), np.zeros(0)
    return np.concatenate(R), np.concatenate(C), np.concatenate(V)


def coo_to_csc(rows, cols, vals, m, n) -> sp.csc_matrix:
    """MATLAB ``sparse(rows,cols,vals,m,n)``: duplicates summed in input
    order, exact zeros dropped (paralleltomo.m:300)."""
    rows = np.asarray(rows, np.int64)
    cols = np.asarray(cols, np.int64)
    vals = np.asarray(vals, float)
    key = cols * m + rows
    order = np.argsort(key, kind="stable")
    key = key[order]
    v = vals[order]
    if key.size:
        starts = np.flatnonzero(np.concatenate([[True], key[1:] != key[:-1]]))
        ends = np.append(starts[1:], key.size)
        summed = v[starts].copy()
        for r in np.flatnonzero(ends - starts > 1):   # duplicates: add in input order
            summed[r] = _seqsum(v[starts[r]:ends[r]])
        ukey = key[starts]
    else:
        summed = v
        ukey = key
    nz = summed != 0
    summed = summed[nz]
    ukey = ukey[nz]
    r = ukey % m
    c = ukey // m
    indptr = np.zeros(n + 1, np.int64)
    np.add.at(indptr, c + 1, 1)
    indptr = np.cumsum(indptr)
    return sp.csc_matrix((summed, r, indptr), shape=(m, n))


def _seqsum(v):
    s = 0.0
    for t in v:
        s = s + float(t)
    return s


def paralleltomo_matrix(N, theta=None, p=None, d=None) -> sp.csc_matrix:
    """System matrix of paralleltomo.m:112-301 (isMatrix=1)."""
    theta, p, d, ct, st, off = parallel_geometry(N, theta, p, d)
    rows, cols, vals = trace_coo(N, parallel_rays(N, ct, st, off), True)
    return coo_to_csc(rows, cols, vals, p * len(theta), N * N)


def fanlineartomo_matrix(N, theta=None, p=None, R=2.0, dw=2.5, sd=3.0):
    """System matrix of fanlineartomo.m:141-358 (isMatrix=1)."""
    theta, p, Rv, _, _, ct, st, cw, sw = fan_geometry(N, theta, p, R, dw, sd)
    rows, cols, vals = trace_coo(N, fan_rays(N, Rv, ct, st, cw, sw), False)
    return coo_to_csc(rows, cols, vals, p * len(theta), N * N)


def matrixfree_apply(N, rays, exclude_top_right, m, u, transp):
    """Matrix-free forward/adjoint of paralleltomo.m:280-288: per ray,
    ``y(row) = aval'*u(col)`` or ``y(col) += u(row)*aval``."""
    u = np.asarray(u, float)
    if not transp:
        y = np.zeros(m)
        for row, x0t, y0t, a, b in rays:
            cols, vals = trace_ray(N, x0t, y0t, a, b, exclude_top_right)
            if cols.size:
                y[row] = float(vals @ u[cols])
        return y
    y = np.zeros(N * N)
    for row, x0t, y0t, a, b in rays:
        cols, vals = trace_ray(N, x0t, y0t, a, b, exclude_top_right)
        if cols.size:
            np.add.at(y, cols, u[row] * vals)
    return y


# ---------------------------------------------------------------------------
# Phantoms: testprobs/phantomgallery.m:155-214 (ellipse rasterisation) plus
# the project's random-ellipse family on the same grid convention.
# ---------------------------------------------------------------------------

_SHEPP = np.array([
    [1, .69, .92, 0, 0, 0],
    [-.8, .6624, .8740, 0, -.0184, 0],
    [-.2, .1100, .3100, .22, 0, -18],
    [-.2, .1600, .4100, -.22, 0, 18],
    [.1, .2100, .2500, 0, .35, 0],
    [.1, .0460, .0460, 0, .1, 0],
    [.1, .0460, .0460, 0, -.1, 0],
    [.1, .0460, .0230, -.08, -.605, 0],
    [.1, .0230, .0230, 0, -.606, 0],
    [.1, .0230, .0460, .06, -.605, 0]])


def ellipse_image(N, ellipses, clip_hi=None):
    """Additive ellipses on the phantomgallery.m:188-214 grid.

    ``ellipses`` rows are (amplitude, semi-axis a, semi-axis b, x0, y0,
    phi in radians).  Returns the N x N image (negative values set to 0 and,
    if ``clip_hi`` is given, values above it clipped).
    """
    xn = (np.arange(N) - (N - 1) / 2.0) / ((N - 1) / 2.0)
    Xn = np.tile(xn, (N, 1))
    Yn = np.rot90(Xn)
    X = np.zeros((N, N))
    for A, ea, eb, x0, y0, phi in ellipses:
        x = Xn - x0
        y = Yn - y0
        inside = (((x * math.cos(phi) + y * math.sin(phi)) ** 2) / (ea * ea)
                  + ((y * math.cos(phi) - x * math.sin(phi))) ** 2 / (eb * eb)) <= 1
        X[inside] += A
    X[X < 0] = 0
    if clip_hi is not None:
        X[X > clip_hi] = clip_hi
    return X


def tectonic(N):
    """phantomgallery.m:422-456, element by element with MATLAB's 1-based
    (row, column) subscripts; returns the N x N image."""
    x = np.zeros((N, N))
    N5 = int(mround(N / 5))
    N13 = int(mround(N / 13))
    N7 = int(mround(N / 7))
    N20 = int(mround(N / 20))

    def setv(r, c, v):
        assert 1 <= r <= N and 1 <= c <= N
        x[r - 1, c - 1] = v

    for r in range(N5, N5 + N7 + 1):               # the right plate
        for c in range(5 * N13, N + 1):
            setv(r, c, 0.75)
    i = N5
    for j in range(1, N20 + 1):                    # its sloped edge
        if j % 2 != 0:
            i = i - 1
            for c in range(5 * N13 + j, N + 1):
                setv(i, c, 0.75)
    for r in range(N5, N5 + N5 + 1):               # the left plate
        for c in range(1, 5 * N13 + 1):
            setv(r, c, 1.0)
    vector = list(range(N5, N5 + N5 + 1))          # the break
    for j in range(5 * N13, min(12 * N13, N) + 1):
        if j % 2 != 0:
            vector = [v + 1 for v in vector]
        for r in vector:
            setv(r, j, 1.0)
    return x


def shepplogan(N):
    """Modified Shepp-Logan head, phantomgallery.m:155-214, as x(:)."""
    e = [(r[0], r[1], r[2], r[3], r[4], r[5] * math.pi / 180) for r in _SHEPP]
    return ellipse_image(N, e).ravel(order="F")


def random_ellipses(N, count, seed):
    """Seeded random-ellipse phantom as x(:), drawn in the same order from the
    same NumPy generator as the product's data generator: centres
    U[-0.6,0.6]^2, semi-axes U[0.05,0.4], rotation U[0,pi), intensity
    U[0.1,1], additive on the phantomgallery.m:188-190 grid, clipped to
    [0,1].  The CPU benchmark arm draws its inputs here so that it loads no
    part of the product."""
    rng = np.random.default_rng(seed)
    ell = []
    for _ in range(count):
        cx, cy = rng.uniform(-0.6, 0.6, 2)
        a, b = rng.uniform(0.05, 0.4, 2)
        phi = rng.uniform(0.0, math.pi)
        amp = rng.uniform(0.1, 1.0)
        ell.append((amp, a, b, cx, cy, phi))
    return ellipse_image(N, ell, clip_hi=1.0).ravel(order="F")


def add_noise(b, eta, seed):
    """b + e, e Gaussian from a seeded NumPy generator scaled to
    ||e|| = eta*||b|| (demos/demo_stoprules.m:43-46); returns (b + e, ||e||)."""
    rng = np.random.default_rng(seed)
    e = rng.standard_normal(b.size)
    e = eta * np.linalg.norm(b) * e / np.linalg.norm(e)
    return b + e, float(np.linalg.norm(e))


# ---------------------------------------------------------------------------
# Solver auxiliaries
# ---------------------------------------------------------------------------


def _inf_to_zero(v):
    v = np.asarray(v, float).copy()
    v[v == np.inf] = 0.0
    return v


def get_mfun_dfun(method, A):
    """Diagonal weights of auxil/get_mfun_dfun.m:43-311 (matrix branch).

    Returns (M, D, Mflag, Dflag).  Vectors for flag 1, matrices for flag 2,
    ``None`` for the identity (flag 0).
    """
    A = sp.csr_matrix(A)
    m, n = A.shape
    if isinstance(method, str):
        absA = abs(A)
        sq = A.multiply(A)
        if method == "landweber":                       # :50-54
            return np.ones(m), np.ones(n), 1, 1
        if method == "cimmino":                         # :56-88
            normAi = np.asarray(sq.sum(axis=1)).ravel()
            with np.errstate(divide="ignore"):
                M = (1.0 / m) * (1.0 / normAi)
            return _inf_to_zero(M), np.ones(n), 1, 1
        if method == "cav":                             # :90-138 (matrix branch)
            s = np.asarray((A != 0).sum(axis=0), float).ravel()
            normAs = np.asarray(sq @ s).ravel()
            with np.errstate(divide="ignore"):
                M = 1.0 / normAs
            return _inf_to_zero(M), np.ones(n), 1, 1
        if method == "drop":                            # :140-198
            normAi = np.asarray(sq.sum(axis=1)).ravel()
            cnt = np.asarray((A != 0).sum(axis=0), float).ravel()
            with np.errstate(divide="ignore"):
                M = 1.0 / normAi
                s = 1.0 / cnt
            return _inf_to_zero(M), _inf_to_zero(s), 1, 1
        if method == "sart":                            # :200-241
            Aip = np.asarray(absA.sum(axis=1)).ravel()
            Apj = np.asarray(absA.sum(axis=0)).ravel()
            with np.errstate(divide="ignore"):
                M = 1.0 / Aip
                D = 1.0 / Apj
            return _inf_to_zero(M), _inf_to_zero(D), 1, 1
        raise ValueError("SIRT method not defined.")
    if isinstance(method, dict):                        # :252-307
        out = []
        for key in ("M", "D"):
            W = method.get(key)
            if W is None or np.size(W) == 0:
                out.append((None, 0))
                continue
            if sp.issparse(W):
                Wc = sp.csr_matrix(W, dtype=float)
                dg = Wc.diagonal()
                if min(Wc.shape) > 1 and (Wc - sp.diags(dg, shape=Wc.shape)).count_nonzero() == 0:
                    out.append((dg, 1))
                    continue
                W = Wc.toarray()
            W = np.asarray(W, float)
            if W.ndim == 1 or min(W.shape) == 1:
                out.append((W.ravel(), 1))
            elif np.count_nonzero(W - np.diag(np.diag(W))) == 0:
                out.append((np.diag(W).copy(), 1))
            else:
                out.append((W, 2))
        (M, mf), (D, df) = out
        return M, D, mf, df
    raise ValueError("First input must be a string with the SIRT method name "
                     "or a struct with fields M and D characterizing a custom method.")


def _apply_w(W, flag, v):
    if flag == 0:
        return v
    if flag == 1:
        return W * v
    return W @ v


def calczeta(k):
    """Newton roots of (2k-1)z^{k-1} - (z^{k-2}+...+1) = 0, calc_relaxpar.m:179-244."""
    k = np.atleast_1d(np.asarray(k))
    if k.size and k[0] < 2:
        raise ValueError("The polynomial is not defined for k < 2")
    z = np.zeros(k.size)
    for i, kk in enumerate(k):
        C = [0.0, 2.0 * kk - 1] + [-1.0] * int(kk - 1)

        def fung(x):
            f = C[0]
            df = 0.0
            for c in C[1:]:
                df = df * x + f
                f = f * x + c
            return f, df
        x = 1.0
        f, df = fung(x)
        h = f / df
        for _ in range(6):
            x = x - h
            f, df = fung(x)
            h = f / df
        z[i] = x
    return z


def estimate_rho(atma, n):
    """Largest eigenvalue of the SIRT iteration operator (calc_relaxpar.m:91-103:
    eigs(atma,n,1,'lm') with tol 1e-4).  ARPACK with a fixed start vector."""
    op = spla.LinearOperator((n, n), matvec=atma, dtype=float)
    vals = spla.eigs(op, k=1, which="LM", tol=1e-4, v0=np.ones(n), return_eigenvectors=False)
    return float(np.real(vals[0]))


def calc_relaxpar_sirt(relaxparinput, rho, kmax, atma, n):
    """SIRT branch of calc_relaxpar.m:89-172.  Returns (relaxpar, casel, rho,
    warning_or_None)."""
    warn = None
    if rho is None or (isinstance(rho, float) and math.isnan(rho)):
        rho = estimate_rho(atma, n)
    if relaxparinput is None:
        return 1.9 / rho, 1, rho, None
    if not isinstance(relaxparinput, str):
        lam = float(relaxparinput)
        if lam <= 0 or lam >= 2 / rho:
            warn = "The relaxpar value is outside the interval (0,%f)" % (2 / rho)
        return lam, 1, rho, warn
    s = relaxparinput.lower()
    if s.startswith("line"):
        return None, 2, rho, None
    if s.startswith("psi1"):
        z = calczeta(np.arange(2, kmax)) if kmax > 2 else np.zeros(0)
        nu = 2.0 if s.startswith("psi1mod") else 1.0
        lam = np.concatenate([[math.sqrt(2), math.sqrt(2)], nu * 2 * (1 - z)]) / rho
        return lam, 3, rho, None
    if s.startswith("psi2"):
        kk = np.arange(2, kmax)
        z = calczeta(kk) if kmax > 2 else np.zeros(0)
        nu = 1.5 if s.startswith("psi2mod") else 1.0
        lam = np.concatenate([[math.sqrt(2), math.sqrt(2)],
                              nu * 2 * (1 - z) / ((1 - z ** kk) ** 2)]) / rho
        return lam, 3, rho, None
    raise ValueError("The chosen relaxation strategy is not valid for this method.")


def check_stoprules(stoprule, rk, relaxpar, taudelta, k, kmax, rkm1, dk, res_dims):
    """auxil/check_stoprules.m:54-164.  Returns (stop, info, rkm1, dk)."""
    info = {}
    st = stoprule.upper()
    stop = False
    if st == "DP":
        nrk = float(np.linalg.norm(rk))
        if nrk <= taudelta or k >= kmax:
            stop = True
            info = {"stoprule": 2 if k != kmax else 0, "finaliter": k, "relaxpar": relaxpar}
    elif st == "ME":
        nrk = float(np.linalg.norm(rkm1))
        dME = float(rkm1 @ (rkm1 + rk)) / 2.0
        with np.errstate(invalid="ignore", divide="ignore"):
            val = dME / nrk
        if val <= taudelta:
            stop = True
            info = {"stoprule": 3, "finaliter": k, "relaxpar": relaxpar}
        elif k >= kmax:
            stop = True
            info = {"stoprule": 0, "finaliter": k, "relaxpar": relaxpar}
        else:
            rkm1 = rk.copy()
    elif st == "NCP":
        dims = list(np.atleast_1d(res_dims))
        if len(dims) == 1:
            mm = rk.size
            q = mm // 2
            pk = np.abs(np.fft.fft(rk)[:q + 1]) ** 2
            c = (np.cumsum(pk[1:]) / np.sum(pk[1:]))[:, None]
        elif len(dims) == 2:
            Rr = rk.reshape(int(dims[0]), int(dims[1]), order="F")
            q = int(dims[0]) // 2
            PK = np.abs(np.fft.fft(Rr, axis=0)[:q + 1, :]) ** 2
            c = np.cumsum(PK[1:, :], axis=0) / np.sum(PK[1:, :], axis=0)
        else:
            raise ValueError("NCP stopping rule only implemented for 1D and 2D residuals")
        c_white = (np.arange(1, q + 1) / q)[:, None]
        ncc = float(np.mean(np.sqrt(np.sum((c - c_white) ** 2, axis=0))))
        if np.max(dk) < np.max(np.concatenate([dk[1:], [ncc]])) or k >= kmax:
            stop = True
            info = {"stoprule": 1 if k != kmax else 0, "finaliter": k, "relaxpar": relaxpar}
        else:
            dk = np.concatenate([dk[1:], [ncc]])
    elif st == "NONE":
        if k >= kmax:
            stop = True
            info = {"stoprule": 0, "finaliter": k, "relaxpar": relaxpar}
    else:
        raise ValueError("Unknown stopping rule given.")
    return stop, info, rkm1, dk


def _parse_common(A, b, K, x0, options, caller):
    """Host-side contract of auxil/check_inputs.m:58-259 for a matrix A."""
    options = options or {}
    A = sp.csr_matrix(A)
    m, n = A.shape
    b = np.asarray(b, float).ravel()
    if b.size != m:
        raise ValueError("The size of A and b do not match.")
    if K is None or np.size(K) == 0:
        raise ValueError("Max no. of iterations must ALWAYS be specified.")
    K = np.atleast_1d(np.asarray(K)).astype(np.int64)
    if not np.all(np.diff(K) > 0):
        raise ValueError("Elements of K must be strictly increasing.")
    x0 = np.zeros(n) if x0 is None or np.size(x0) == 0 else np.asarray(x0, float).ravel().copy()
    if x0.size != n:
        raise ValueError("The size of x0 does not match the problem.")
    lb = options.get("lbound")
    ub = options.get("ubound")
    lb = None if lb is None else np.atleast_1d(np.asarray(lb, float)).ravel()
    ub = None if ub is None else np.atleast_1d(np.asarray(ub, float)).ravel()
    for v, nm in ((lb, "lbound"), (ub, "ubound")):
        if v is not None and v.size not in (1, n):
            raise ValueError(nm + " must either be scalar or same length as vector of unknowns x.")
    sr = options.get("stoprule", {}) or {}
    stype = sr.get("type", "NONE")
    taudelta = float("nan")
    if stype.upper() in ("DP", "ME"):
        td = sr.get("taudelta")
        if td is None or np.size(td) != 1:
            raise ValueError("For stopping rules DP and ME a scalar taudelta must be given in options.")
        taudelta = float(td)
    if stype.upper() == "ME" and caller != "sirt":
        raise ValueError("Stopping rule ME is only available for SIRT methods, not ART and CART.")
    if stype.upper() not in ("DP", "ME", "NCP", "NONE"):
        raise ValueError("The chosen stopping rule is not valid.")
    if stype == "NCP" and "res_dims" not in sr:
        raise ValueError("options.stoprule.res_dims must be specified for NCP stopping rule.")
    res_dims = sr.get("res_dims")
    ncp_smooth = int(sr.get("ncp_smooth", 2))
    rkm1 = np.full(m, np.nan) if stype.upper() == "ME" else None
    dk = np.full(ncp_smooth, np.inf) if stype.upper() == "NCP" else None
    damp = float(options.get("damp", 0.0))
    if damp < 0:
        raise ValueError("Damping must be positive")
    rho = options.get("rho", float("nan"))
    return dict(A=A, m=m, n=n, b=b, K=K, kmax=int(K[-1]), x0=x0, lb=lb, ub=ub,
                stype=stype, taudelta=taudelta, res_dims=res_dims, rkm1=rkm1, dk=dk,
                damp=damp, rho=float(rho), relaxpar=options.get("relaxpar"))


def sirt(method, A, b, K, x0=None, options=None):
    """sirt/sirt.m:134-281 in FP64.  Returns (X, info, ext_info)."""
    t0 = time.perf_counter()
    if method is None:
        method = "sart"
    c = _parse_common(A, b, K, x0, options, "sirt")
    A, m, n, b, K, kmax = c["A"], c["m"], c["n"], c["b"], c["K"], c["kmax"]
    AT = A.T.tocsr()
    M, D, mf, df = get_mfun_dfun(method, A)
    X = np.zeros((n, K.size))
    xk = c["x0"]
    rk = b - A @ xk
    k = 0
    l = 0
    rkm1, dk = c["rkm1"], c["dk"]
    stop, info, rkm1, dk = check_stoprules(c["stype"], rk, c["relaxpar"], c["taudelta"],
                                           k, kmax, rkm1, dk, c["res_dims"])
    rho = c["rho"]
    if isinstance(method, str) and method == "sart":
        rho = 1.0

    def atma(v):
        return _apply_w(D, df, AT @ _apply_w(M, mf, A @ v))
    relaxpar, casel, rho, warn = calc_relaxpar_sirt(c["relaxpar"], rho, kmax, atma, n)
    ext = {"M": np.ones(m) if mf == 0 else _apply_w(M, mf, np.ones(1)) if mf == 1 else M,
           "D": np.ones(n) if df == 0 else _apply_w(D, df, np.ones(1)) if df == 1 else D}
    lb, ub = c["lb"], c["ub"]
    resnorms = []
    lam_used = []
    while not stop:
        k += 1
        Mrk = _apply_w(M, mf, rk)
        ATMrk = AT @ Mrk
        if casel == 1:
            lam = relaxpar
        elif casel == 2:
            lam = float(rk @ Mrk) / float(np.sum(_apply_w(D, df, ATMrk ** 2)))
        else:
            lam = float(relaxpar[k - 1])
        xk = xk + lam * _apply_w(D, df, ATMrk)
        if lb is not None:
            xk = np.maximum(xk, lb)
        if ub is not None:
            xk = np.minimum(xk, ub)
        rk = b - A @ xk
        stop, info, rkm1, dk = check_stoprules(c["stype"], rk, lam, c["taudelta"], k, kmax,
                                               rkm1, dk, c["res_dims"])
        resnorms.append(float(np.linalg.norm(rk)))
        lam_used.append(lam)
        if (l < K.size and k == K[l]) or stop:
            X[:, l] = xk
            l += 1
    X = X[:, :l]
    if not info:
        info = {"stoprule": 0, "finaliter": 0, "relaxpar": relaxpar}
    info["rho"] = rho
    info["itersaved"] = np.concatenate([K[K < info["finaliter"]], [info["finaliter"]]])
    info["timetaken"] = time.perf_counter() - t0
    info["resnorms"] = np.array(resnorms)
    info["relaxpar_used"] = np.array(lam_used)
    info["warning"] = warn
    return X, info, ext


class RandStream:
    """Index stream for randkaczmarz: one permutation per sweep and one
    uniform number per step, drawn from a seeded NumPy generator.  The
    product host code draws the same stream from the same seed."""

    def __init__(self, seed):
        self.rng = np.random.default_rng(seed)

    def randperm(self, n):
        return self.rng.permutation(n)

    def rand(self, count):
        return self.rng.random(count)


def art_row_order(method, normAi, m):
    """Row order of art/art.m:183-203 (0-based); returns (I, is_rand)."""
    if isinstance(method, str):
        I = np.flatnonzero(normAi > 0)
        mth = method.lower()
        if mth == "kaczmarz":
            return I, False
        if mth == "symkaczmarz":
            return np.concatenate([I, I[::-1]]), False
        if mth == "randkaczmarz":
            return I, True
        raise ValueError("Unknown ART method specified")
    I = np.asarray(method, np.int64).ravel()
    return I[normAi[I] > 0], False


def art_sweep_rows(I, normAi_damped, is_rand, stream, m):
    """Rows visited in one sweep (art/art.m:241-262) and the i values that
    index a relaxpar handle.  Returns (ri, i_for_lambda), 0-based."""
    if not is_rand:
        return I, I
    cumul = np.cumsum(normAi_damped / np.sum(normAi_damped))
    fast = np.max(np.abs(cumul - np.arange(1, m + 1) / m)) < 0.05
    I_torun = I[stream.randperm(I.size)]
    if fast:
        return I_torun, I_torun
    u = stream.rand(I_torun.size)
    ri = np.searchsorted(cumul, u, side="left")  # sum(cumul<rand)+1 -> 0-based
    ri = np.minimum(ri, m - 1)
    return ri, I_torun


def art(method, A, b, K, x0=None, options=None, stream=None):
    """art/art.m:109-330 in FP64.  Returns (X, info)."""
    t0 = time.perf_counter()
    if method is None:
        method = "kaczmarz"
    c = _parse_common(A, b, K, x0, options, "art")
    A, m, n, b, K, kmax = c["A"], c["m"], c["n"], c["b"], c["K"], c["kmax"]
    sym = isinstance(method, str) and method.lower().startswith("sym")
    if sym:
        if np.any(K % 2):
            raise ValueError("For symkaczmarz only even iteration numbers can be requested.")
        K = K // 2
        kmax = kmax // 2
    X = np.zeros((n, K.size))
    xk = c["x0"]
    rk = b - A @ xk
    k = 0
    l = 0
    rkm1, dk = c["rkm1"], c["dk"]
    relin = c["relaxpar"]
    stop, info, rkm1, dk = check_stoprules(c["stype"], rk, relin, c["taudelta"], k, kmax,
                                           rkm1, dk, c["res_dims"])
    relaxpar = 1.0 if relin is None else (-1000.0 if callable(relin) else float(relin))
    Acsr = A.tocsr()
    normAi = np.asarray(Acsr.multiply(Acsr).sum(axis=1)).ravel()
    I, is_rand = art_row_order(method, normAi, m)
    normAi = normAi + c["damp"] * np.max(normAi)
    lb, ub = c["lb"], c["ub"]
    ub_active = ub is not None and not np.any(np.isnan(ub))
    indptr, indices, data = Acsr.indptr, Acsr.indices, Acsr.data
    while not stop:
        k += 1
        rows, lam_i = art_sweep_rows(I, normAi, is_rand, stream, m)
        for ri, ii in zip(rows, lam_i):
            s, e = indptr[ri], indptr[ri + 1]
            cols = indices[s:e]
            av = data[s:e]
            if callable(relin):
                relaxpar = float(relin((k - 1) * m + int(ii) + 1))
            xk = xk.copy()
            xk[cols] = xk[cols] + (relaxpar * (b[ri] - float(av @ xk[cols])) / normAi[ri]) * av
            if lb is not None:
                xk = np.maximum(xk, lb)
            if ub_active:
                xk = np.minimum(xk, ub)
        rk = b - A @ xk
        stop, info, rkm1, dk = check_stoprules(c["stype"], rk, relaxpar, c["taudelta"], k, kmax,
                                               rkm1, dk, c["res_dims"])
        if (l < K.size and k == K[l]) or stop:
            X[:, l] = xk
            l += 1
    X = X[:, :l]
    if not info:
        info = {"stoprule": 0, "finaliter": 0, "relaxpar": relaxpar}
    if sym:
        info["finaliter"] = 2 * info["finaliter"]
        K = 2 * K
    info["itersaved"] = np.concatenate([K[K < info["finaliter"]], [info["finaliter"]]])
    info["timetaken"] = time.perf_counter() - t0
    return X, info


_M64 = (1 << 64) - 1


def _splitmix64(z: int) -> int:
    z = (z + 0x9E3779B97F4A7C15) & _M64
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & _M64
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & _M64
    return z ^ (z >> 31)


def cart_randi(seed: int, k: int, j: int, N: int) -> int:
    """The unflagging draw randi(N) of sweep k at 0-based column j: MATLAB's
    randi stream cannot be reproduced, so every draw is a counter-based
    splitmix64 hash of (seed, k, j) mapped to 1 + floor(u*N)."""
    key = ((k << 32) | (j & 0xFFFFFFFF)) & _M64
    z = _splitmix64((seed & _M64) ^ _splitmix64(key))
    u = float(z >> 11) * 2.0 ** -53
    return 1 + min(int(math.floor(u * N)), N - 1)


def cart(method, A, b, K, x0=None, options=None):
    """cart/cart.m:109-320 (columnaction) in FP64, column by column, with
    mm = max(abs(xk)) scanned in full before every column as in the
    reference.  Returns (X, info)."""
    t0 = time.perf_counter()
    options = dict(options or {})
    if method is None:
        method = "columnaction"
    c = _parse_common(A, b, K, x0, options, "cart")
    A, m, n, b, K, kmax = c["A"], c["m"], c["n"], c["b"], c["K"], c["kmax"]
    THR = float(options.get("THR", 1e-4))
    Kbegin = int(options.get("Kbegin", 10))
    Nunflag = int(options["Nunflag"]) if "Nunflag" in options else int(mround(kmax / 4))
    seed = int(options.get("seed", 0))
    X = np.zeros((n, K.size))
    rk = b - A @ c["x0"]
    k = 0
    xk = c["x0"].copy()
    l = 0
    rkm1, dk = c["rkm1"], c["dk"]
    relin = c["relaxpar"]
    stop, info, rkm1, dk = check_stoprules(c["stype"], rk, relin, c["taudelta"], k, kmax,
                                           rkm1, dk, c["res_dims"])
    if relin is not None and (callable(relin) or np.size(relin) != 1):
        raise ValueError("For CART methods the relaxpar must be a scalar.")
    relaxpar = 0.25 if relin is None else float(relin)
    Acsc = sp.csc_matrix(A)
    normAj = np.asarray(Acsc.multiply(Acsc).sum(axis=0)).ravel()
    if isinstance(method, str):
        if method.lower() != "columnaction":
            raise ValueError("Unknown CART method specified")
        J = np.flatnonzero(normAj > 0)
    else:
        J = np.asarray(method, dtype=np.int64).ravel()
        J = J[normAj[J] > 0]
    normAj = normAj + c["damp"] * np.max(normAj)
    F = np.ones(n, dtype=bool)
    Nflag = np.zeros(n, dtype=np.int64)
    lb, ub = c["lb"], c["ub"]
    indptr, indices, data = Acsc.indptr, Acsc.indices, Acsc.data
    while not stop:
        k += 1
        for j in J:
            mm = np.max(np.abs(xk)) if n else 0.0
            if F[j]:
                s_, e_ = indptr[j], indptr[j + 1]
                rows = indices[s_:e_]
                aj = data[s_:e_]
                delta = float(aj @ rk[rows]) / normAj[j]
                od = relaxpar * delta
                xkj = xk[j]
                if lb is not None:
                    lbj = lb[0] if lb.size == 1 else lb[j]
                    if od < lbj - xkj:
                        od = lbj - xkj
                if ub is not None:
                    ubj = ub[0] if ub.size == 1 else ub[j]
                    if od > ubj - xkj:
                        od = ubj - xkj
                xk[j] = xkj + od
                if k >= Kbegin and abs(od) < THR * mm:
                    F[j] = False
                    Nflag[j] = 1
                rk[rows] = rk[rows] - od * aj
            else:
                if Nunflag < 1:
                    raise ValueError("randi: Nunflag must be a positive integer")
                if Nflag[j] < cart_randi(seed, k, int(j), Nunflag):
                    Nflag[j] += 1
                else:
                    F[j] = True
        stop, info, rkm1, dk = check_stoprules(c["stype"], rk, relaxpar, c["taudelta"], k, kmax,
                                               rkm1, dk, c["res_dims"])
        if (l < K.size and k == K[l]) or stop:
            X[:, l] = xk
            l += 1
    X = X[:, :l]
    if not info:
        info = {"stoprule": 0, "finaliter": 0, "relaxpar": relaxpar}
    info["itersaved"] = np.concatenate([K[K < info["finaliter"]], [info["finaliter"]]])
    info["timetaken"] = time.perf_counter() - t0
    return X, info


def _nextpow2(x):
    x = abs(float(x))
    if x == 0:
        return 0
    return int(math.ceil(math.log2(x)))


def fbp(A, b, theta, filter="ram-lak"):
    """auxil/fbp.m:40-79 in FP64: the sinogram reshaped to nr x na, each
    column zero-padded to order = max(64, 2^nextpow2(2*nr)) samples,
    FFT, times the filter, inverse FFT, real part, cropped to nr rows, then
    x = A'*b(:)*pi/(2*na)."""
    filter = filter.lower()
    A = sp.csr_matrix(A)
    if filter == "none":
        return A.T @ np.asarray(b, float)
    m = A.shape[0]
    na = len(np.atleast_1d(theta))
    nr = m // na
    B = np.asarray(b, float).reshape(nr, na, order="F")
    order = max(64, 2 ** _nextpow2(2 * nr))
    n = np.arange(order / 2 + 1)
    f = n / np.max(n)
    f[0] = 0.4 / order
    f[-1] = 1 - f[0]
    w = 2 * math.pi * n / order
    if filter == "ram-lak":
        pass
    elif filter == "shepp-logan":
        f[1:] = f[1:] * (np.sin(w[1:] / 2) / (w[1:] / 2))
    elif filter == "cosine":
        f[1:] = f[1:] * np.cos(w[1:] / 2)
    elif filter == "hamming":
        f[1:] = f[1:] * (0.54 + 0.46 * np.cos(w[1:]))
    elif filter == "hann":
        f[1:] = f[1:] * (1 + np.cos(w[1:])) / 2
    else:
        raise ValueError("Iinvalid filter")
    f = np.concatenate([f, f[-2:0:-1]])
    Bp = np.zeros((order, na))
    Bp[:nr] = B
    Bf = np.fft.fft(Bp, axis=0)
    Bf = Bf * f[:, None]
    Bf = np.real(np.fft.ifft(Bf, axis=0))[:nr]
    return (A.T @ Bf.ravel(order="F")) * math.pi / (2 * na)


# ---------------------------------------------------------------- training
def _run(method, A, b, K, x0, options):
    if method in ("landweber", "cimmino", "cav", "drop", "sart"):
        X, info, _ = sirt(method, A, b, K, x0, options)
    elif method == "columnaction":
        X, info = cart(method, A, b, K, x0, options)
    else:
        X, info = art(method, A, b, K, x0, options)
    return X, info


def train_relaxpar(A, b, x_ex, method, kmax, options=None):
    """train/train_relaxpar.m:75-270, branch for branch."""
    if options is not None:
        options = dict(options)
        options["stoprule"] = {"type": "none"}
        options.pop("relaxpar", None)
    else:
        options = {}
    fudge, stepk = 0.02, 10
    K = list(range(1, stepk + 1))
    k, stop, Er, x0 = 0, False, [], None
    is_sirt = method in ("landweber", "cimmino", "cav", "drop", "sart")
    while not stop:
        if k + stepk > kmax:
            K = list(range(1, kmax - k + 1))
            k = kmax
        else:
            k += stepk
        if k <= stepk:
            if is_sirt:
                Xnew, info = _run(method, A, b, K, x0, options)
                options["rho"] = info["rho"]
                relaxparmax = 2 / info["rho"]
            else:
                options["relaxpar"] = 0.25
                Xnew, _ = _run(method, A, b, K, x0, options)
                relaxparmax = 2
        else:
            Xnew, _ = _run(method, A, b, K, x0, options)
        Er.extend(np.sqrt(np.sum((Xnew - x_ex[:, None]) ** 2, axis=0)))
        kopt = int(np.argmin(Er)) + 1
        minE = Er[kopt - 1]
        if kopt == k and k < kmax:
            x0 = Xnew[:, -1]
        else:
            stop = True
    meub = (1 + fudge) * minE

    def ev(p):
        options["relaxpar"] = p
        xnew, _ = _run(method, A, b, list(range(1, kopt + 1)), None, options)
        ee = np.sqrt(np.sum((xnew - x_ex[:, None]) ** 2, axis=0))
        kk = int(np.sum((ee[:-1] > meub) & (np.diff(ee) < 0))) + 1
        return kk, ee[kk - 1]

    r = (3 - np.sqrt(5)) / 2
    alpha, beta = 0.0, relaxparmax
    alphap, betap = alpha + r * (beta - alpha), alpha + (1 - r) * (beta - alpha)
    k_alphap, err_alphap = ev(alphap)
    k_betap, err_betap = ev(betap)

    def up():
        nonlocal alpha, alphap, betap, k_alphap, err_alphap, k_betap, err_betap
        z = alphap + (1 - r) * abs(beta - alphap)
        alpha, alphap, betap = alphap, betap, z
        k_alphap, err_alphap = k_betap, err_betap
        k_betap, err_betap = ev(betap)

    def down():
        nonlocal beta, alphap, betap, k_alphap, err_alphap, k_betap, err_betap
        z = alpha + r * abs(betap - alpha)
        beta, betap, alphap = betap, alphap, z
        k_betap, err_betap = k_alphap, err_alphap
        k_alphap, err_alphap = ev(alphap)

    while abs(alphap - betap) > relaxparmax * 0.01:
        if is_sirt:
            if err_alphap > meub:
                up()
            elif err_betap > meub:
                down()
            elif k_alphap >= k_betap:
                up()
            else:
                down()
        else:
            if err_betap > meub:
                down()
            elif err_alphap > meub:
                up()
            elif k_alphap >= k_betap:
                up()
            else:
                down()
    return (alphap + betap) / 2


def train_dpme(A, b_exact, x_exact, method, type_, delta, E, kmax, options=None):
    """train/train_dpme.m:66-136 with the noise matrix E (m x s) given."""
    options = dict(options or {})
    options["stoprule"] = {"type": "none"}
    A = sp.csr_matrix(A)
    e = delta * E / np.sqrt(np.sum(E * E, axis=0))[None, :]
    B = b_exact[:, None] + e
    kstep = kmax if kmax < 10 else 10
    taus = []
    for i in range(E.shape[1]):
        bi = B[:, i]
        X = np.zeros((x_exact.size, 1))
        x0 = None
        k = kstep
        K = list(range(1, k + 1))
        Ek = []
        while True:
            Xny, _ = _run(method, A, bi, K, x0, options)
            Ek.extend(np.sqrt(np.sum((Xny - x_exact[:, None]) ** 2, axis=0)))
            X = np.hstack([X, Xny])
            I = int(np.argmin(Ek)) + 1
            if I != k or k >= kmax:
                kopt = I
                break
            if k + kstep > kmax:
                K = list(range(1, kmax - k + 1))
                k = kmax
            else:
                k += kstep
            x0 = Xny[:, -1]
        rk = bi - A @ X[:, kopt - 1]
        if type_.upper().startswith("DP"):
            taus.append(np.linalg.norm(rk) / delta)
        else:
            rkm1 = bi - A @ X[:, kopt - 2]
            taus.append(0.5 * (rkm1 @ (rkm1 + rk)) / (delta * np.linalg.norm(rkm1)))
    return float(np.mean(taus))
