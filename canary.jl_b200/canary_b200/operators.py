"""1-D operators of Canary (src/operators.jl, src/GaussQuadrature/quadrature.jl).

Host-side mirror of the reference's setup API: Legendre–Gauss–Lobatto points
and weights by the Golub–Welsch method with the Lobatto end-point
modification, barycentric weights, spectral differentiation and interpolation
matrices.  These run once per mesh on the host and feed the device kernels.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math

import numpy as np

# C99 hypot of the platform libm (CPython's math.hypot uses its own
# algorithm); both are within one ulp of Julia's hypot.
_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
_libm.hypot.restype = ctypes.c_double
_libm.hypot.argtypes = [ctypes.c_double, ctypes.c_double]
_hypot = _libm.hypot

NEITHER, LEFT, RIGHT, BOTH = "N", "L", "R", "B"
_MAXITS = 30  # maxiterations[Float64], quadrature.jl:115


class QuadratureError(RuntimeError):
    pass


def legendre_coefs(n: int):
    """Recurrence coefficients of the monic Legendre polynomials
    (quadrature.jl:140-148)."""
    a = np.zeros(n)
    b = np.zeros(n + 1)
    b[0] = math.sqrt(2.0)
    for k in range(2, n + 2):
        b[k - 1] = (k - 1) / math.sqrt(float((2 * k - 1) * (2 * k - 3)))
    return a, b


def _solve(n, shift, a, b):
    # n-th component of (J_n - shift I)^{-1} e_n (quadrature.jl:216-233)
    t = a[0] - shift
    for i in range(2, n):
        t = (a[i - 1] - shift) - (b[i - 1] * b[i - 1]) / t
    return 1.0 / t


def _eig_first_components(d, e, maxits):
    """Eigenvalues and first eigenvector components of the symmetric
    tridiagonal matrix (diag d, sub-diagonal e[1:]) by the implicit QL method
    (quadrature.jl:235-326, after EISPACK imtql2)."""
    n = len(d)
    z = [0.0] * n
    z[0] = 1.0
    e[n] = 0.0
    if n == 1:
        return z
    eps = np.finfo(np.float64).eps
    for l in range(1, n + 1):
        for j in range(1, maxits + 1):
            m = n
            for i in range(l, n):
                if abs(e[i]) <= eps * (abs(d[i - 1]) + abs(d[i])):
                    m = i
                    break
            p = d[l - 1]
            if m == l:
                continue
            if j == maxits:
                raise QuadratureError(f"No convergence after {j} iterations "
                                      "(try increasing maxits)")
            g = (d[l] - p) / (2.0 * e[l])
            r = _hypot(g, 1.0)
            g = (d[m - 1] - p) + e[l] / (g + math.copysign(r, g))
            s = c = 1.0
            p = 0.0
            for i in range(m - 1, l - 1, -1):
                f = s * e[i]
                bb = c * e[i]
                if abs(f) < abs(g):
                    s = f / g
                    r = _hypot(s, 1.0)
                    e[i + 1] = g * r
                    c = 1.0 / r
                    s *= c
                else:
                    c = g / f
                    r = _hypot(c, 1.0)
                    e[i + 1] = f * r
                    s = 1.0 / r
                    c *= s
                g = d[i] - p
                r = (d[i - 1] - g) * s + (2.0 * c) * bb
                p = s * r
                d[i] = g + p
                g = c * r - bb
                f = z[i]
                z[i] = s * z[i - 1] + c * f
                z[i - 1] = c * z[i - 1] - s * f
            d[l - 1] -= p
            e[l] = g
            e[m] = 0.0
    return z


def custom_gauss_rule(lo, hi, a, b, endpt=NEITHER, maxits=_MAXITS):
    """Gauss rule from monic recurrence coefficients (quadrature.jl:175-214)."""
    a = [float(v) for v in a]
    b = [float(v) for v in b]
    n = len(a)
    if endpt == LEFT:
        a[n - 1] = lo if n == 1 else _solve(n, lo, a, b) * (b[n - 1] * b[n - 1]) + lo
    elif endpt == RIGHT:
        a[n - 1] = hi if n == 1 else _solve(n, hi, a, b) * (b[n - 1] * b[n - 1]) + hi
    elif endpt == BOTH:
        if n == 1:
            raise QuadratureError("Must have at least two points for both ends.")
        g = _solve(n, lo, a, b)
        t1 = (hi - lo) / (g - _solve(n, hi, a, b))
        b[n - 1] = math.sqrt(t1)
        a[n - 1] = lo + g * t1
    z = _eig_first_components(a, b, maxits)
    w = [(b[0] * zi) * (b[0] * zi) for zi in z]
    idx = sorted(range(n), key=lambda i: a[i])  # stable, = sortperm
    if endpt in (LEFT, BOTH):  # `both` pins only the left end (quadrature.jl:208-212)
        a[idx[0]] = lo
    elif endpt == RIGHT:
        a[idx[-1]] = hi
    return np.array([a[i] for i in idx]), np.array([w[i] for i in idx])


def legendre(n: int, endpt: str = NEITHER):
    if n < 1:
        raise ValueError("n >= 1 required")
    a, b = legendre_coefs(n)
    return custom_gauss_rule(-1.0, 1.0, a, b, endpt)


def lglpoints(N: int):
    """N+1 Legendre–Gauss–Lobatto points and weights (operators.jl:10-13)."""
    if N < 1:
        raise ValueError("N >= 1 required")
    return legendre(N + 1, BOTH)


def lgpoints(N: int):
    """N+1 Legendre–Gauss points and weights (operators.jl:21-24)."""
    if N < 1:
        raise ValueError("N >= 1 required")
    return legendre(N + 1, NEITHER)


def baryweights(r):
    """Barycentric weights (operators.jl:36-49)."""
    r = np.asarray(r, dtype=np.float64)
    n = len(r)
    wb = np.ones(n)
    for j in range(n):
        for i in range(n):
            if i != j:
                wb[j] = wb[j] * (r[j] - r[i])
        wb[j] = 1.0 / wb[j]
    return wb


def spectralderivative(r, wb=None):
    """Spectral differentiation matrix D[j, k] = l_k'(r_j) (operators.jl:64-84)."""
    r = np.asarray(r, dtype=np.float64)
    wb = baryweights(r) if wb is None else np.asarray(wb, dtype=np.float64)
    n = len(r)
    D = np.zeros((n, n), order="F")
    for k in range(n):
        for j in range(n):
            if k == j:
                for l in range(n):
                    if l != k:
                        D[j, k] = D[j, k] + 1.0 / (r[k] - r[l])
            else:
                D[j, k] = (wb[k] / wb[j]) / (r[j] - r[k])
    return D


def interpolationmatrix(rsrc, rdst, wbsrc=None):
    """Barycentric interpolation matrix from rsrc to rdst (operators.jl:98-117)."""
    rsrc = np.asarray(rsrc, dtype=np.float64)
    rdst = np.asarray(rdst, dtype=np.float64)
    wb = baryweights(rsrc) if wbsrc is None else np.asarray(wbsrc, dtype=np.float64)
    I = np.zeros((len(rdst), len(rsrc)))
    with np.errstate(divide="ignore", invalid="ignore"):
        for k in range(len(rdst)):
            for j in range(len(rsrc)):
                I[k, j] = wb[j] / (rdst[k] - rsrc[j])
                if not np.isfinite(I[k, j]):
                    I[k, :] = 0.0
                    I[k, j] = 1.0
                    break
            I[k, :] = I[k, :] / I[k, :].sum()
    return I
