"""Filtered back projection, auxil/fbp.m:40-79, on the GPU.

The host builds fbp.m's frequency-domain filter (ram-lak, shepp-logan,
cosine, hamming or hann on order = max(64, 2^nextpow2(2*nr)) samples) and
turns it into the circular convolution kernel real(ifft(filter)); libairt
convolves every projection with it in FP64, scales by pi/(2*na) and
back-projects with A'.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check, dptr, lib
from .afun import as_operator

FILTERS = ("ram-lak", "shepp-logan", "cosine", "hamming", "hann", "none")


def _nextpow2(x: float) -> int:
    """MATLAB nextpow2: the smallest p with 2^p >= |x|."""
    x = abs(float(x))
    if x == 0:
        return 0
    p = math.frexp(x)[1]
    return p - 1 if x == 2.0 ** (p - 1) else p


def fbp_filter(nr: int, filter: str = "ram-lak") -> np.ndarray:
    """fbp.m:50-73: the filter f of length order (the even extension of
    n/max(n), n = 0..order/2, with f(1) = 0.4/order and f(end) = 1 - f(1),
    times the named window)."""
    filter = filter.lower()
    order = max(64, 2 ** _nextpow2(2 * nr))
    n = np.arange(order // 2 + 1, dtype=float)
    f = n / np.max(n)
    f[0] = 0.4 / order
    f[-1] = 1.0 - f[0]
    w = 2.0 * math.pi * n / order
    if filter == "ram-lak":
        pass
    elif filter == "shepp-logan":
        f[1:] = f[1:] * np.sinc(w[1:] / (2.0 * math.pi))
    elif filter == "cosine":
        f[1:] = f[1:] * np.cos(w[1:] / 2.0)
    elif filter == "hamming":
        f[1:] = f[1:] * (0.54 + 0.46 * np.cos(w[1:]))
    elif filter == "hann":
        f[1:] = f[1:] * (1.0 + np.cos(w[1:])) / 2.0
    else:
        raise ValueError("Iinvalid filter")
    return np.concatenate([f, f[-2:0:-1]])


def fbp_kernel(nr: int, filter: str = "ram-lak") -> np.ndarray:
    """The circular convolution kernel real(ifft(f)) of fbp_filter (order
    entries) that the zero-pad / fft / filter / ifft / crop steps of
    fbp.m:74-78 apply to every projection."""
    return np.ascontiguousarray(np.real(np.fft.ifft(fbp_filter(nr, filter))))


def fbp(A, b, theta, filter: str = "ram-lak") -> np.ndarray:
    """x = fbp(A,b,theta,filter)  (auxil/fbp.m:1): filtered back projection
    of the sinogram b (rays x angles, column-major) for the angles theta."""
    if theta is None:
        raise ValueError("Input A, b, theta must me specified")
    filter = (filter or "ram-lak").lower()
    op = as_operator(A)
    b = np.ascontiguousarray(np.asarray(b, dtype=np.float64).ravel())
    if b.size != op.m:
        raise ValueError("The size of A and b do not match.")
    if filter == "none":
        return op(b, "transp")
    na = int(np.size(theta))
    if na < 1 or op.m % na:
        raise ValueError("the number of angles must divide the number of rows of A")
    h = fbp_kernel(op.m // na, filter)
    x = np.empty(op.n)
    check(lib().airt_fbp(op.handle, dptr(b), na, dptr(h), int(h.size), dptr(x)))
    return x
