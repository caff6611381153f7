"""Grids and metric terms of Canary (src/metric.jl) and the drivers'
computegeometry (examples/3d_kernels/euler3d_set3c.jl:210-248,
examples/2d_kernels/euler2d_set3c.jl:171-208).

Host-side, vectorised over elements and nodes; every reduction over the 1-D
index n is accumulated in the reference's order so that the results are
reproducible bit for bit.  Arrays are Fortran-ordered with the Julia shapes.
"""
from __future__ import annotations

import math

import numpy as np

from .operators import lglpoints, spectralderivative

# vgeo / sgeo field layouts of the set3c drivers
VGEO3D = ("xix", "etax", "zetax", "xiy", "etay", "zetay", "xiz", "etaz", "zetaz", "MJ", "MJI", "x", "y", "z")
SGEO3D = ("nx", "ny", "nz", "sMJ", "vMJI")
VGEO2D = ("xix", "etax", "xiy", "etay", "MJ", "MJI", "x", "y")
SGEO2D = ("nx", "ny", "sMJ", "vMJI")


def creategrid(elemtocoord, r):
    """(Bi/tri)linear blend of element corners onto the LGL grid
    (metric.jl:11-107).  Returns a tuple of d arrays (Nq,...,Nq, nelem)."""
    e2c = np.asarray(elemtocoord, dtype=np.float64)
    d, nvert, nelem = e2c.shape
    r = np.asarray(r, dtype=np.float64)
    Nq = len(r)
    a, b = 1.0 - r, 1.0 + r
    out = []
    if d == 1:
        for n in range(1):
            out.append(np.asfortranarray((a[:, None] * e2c[n, 0][None, :] + b[:, None] * e2c[n, 1][None, :]) / 2.0))
        return tuple(out)
    if d == 2:
        A, B = a[:, None], b[:, None]
        C, Dd = a[None, :], b[None, :]
        w = [A * C, B * C, A * Dd, B * Dd]
        for n in range(2):
            t = w[0][:, :, None] * e2c[n, 0][None, None, :]
            for v in range(1, 4):
                t = t + w[v][:, :, None] * e2c[n, v][None, None, :]
            out.append(np.asfortranarray(t / 4.0))
        return tuple(out)
    ai, bi = a[:, None, None], b[:, None, None]
    cj, dj = a[None, :, None], b[None, :, None]
    gk, hk = a[None, None, :], b[None, None, :]
    w = [ai * cj * gk, bi * cj * gk, ai * dj * gk, bi * dj * gk,
         ai * cj * hk, bi * cj * hk, ai * dj * hk, bi * dj * hk]
    for n in range(3):
        t = w[0][..., None] * e2c[n, 0][None, None, None, :]
        for v in range(1, 8):
            t = t + w[v][..., None] * e2c[n, v][None, None, None, :]
        out.append(np.asfortranarray(t / 8.0))
    return tuple(out)


def _d_ref(D, X, axis):
    """Σ_n D[i, n] X[.., n, ..] along `axis`, accumulated in n order."""
    Nq = D.shape[0]
    out = np.zeros_like(X)
    for n in range(Nq):
        sl = [slice(None)] * X.ndim
        sl[axis] = slice(n, n + 1)
        shape = [1] * X.ndim
        shape[axis] = Nq
        out = out + D[:, n].reshape(shape) * X[tuple(sl)]
    return out


def computemetric2d(x, y, D):
    """2-D metric terms (metric.jl:155-208).  x, y: (Nq, Nq, nelem)."""
    D = np.asarray(D, dtype=np.float64)
    xr, xs = _d_ref(D, x, 0), _d_ref(D, x, 1)
    yr, ys = _d_ref(D, y, 0), _d_ref(D, y, 1)
    J = xr * ys - yr * xs
    xix, etax, xiy, etay = ys / J, -yr / J, -xs / J, xr / J
    Nq, nelem = x.shape[0], x.shape[2]
    nx = np.zeros((Nq, 4, nelem), order="F")
    ny = np.zeros((Nq, 4, nelem), order="F")
    nx[:, 0], ny[:, 0] = -J[0, :] * xix[0, :], -J[0, :] * xiy[0, :]
    nx[:, 1], ny[:, 1] = J[-1, :] * xix[-1, :], J[-1, :] * xiy[-1, :]
    nx[:, 2], ny[:, 2] = -J[:, 0] * etax[:, 0], -J[:, 0] * etay[:, 0]
    nx[:, 3], ny[:, 3] = J[:, -1] * etax[:, -1], J[:, -1] * etay[:, -1]
    sJ = np.hypot(nx, ny)
    nx, ny = nx / sJ, ny / sJ
    f = np.asfortranarray
    return dict(J=f(J), xix=f(xix), etax=f(etax), xiy=f(xiy), etay=f(etay),
                sJ=f(sJ), nx=f(nx), ny=f(ny))


def _hypot3(a, b, c):
    # Julia's n-argument hypot: maxabs * sqrt(sum((v / maxabs)^2))
    m = np.maximum(np.maximum(np.abs(a), np.abs(b)), np.abs(c))
    with np.errstate(invalid="ignore", divide="ignore"):
        p, q, s = a / m, b / m, c / m
        h = m * np.sqrt((p * p + q * q) + s * s)
    return np.where((m == 0) | np.isinf(m), m, h)


def computemetric3d(x, y, z, D):
    """3-D metric terms in the curl-invariant form (metric.jl:230-400).
    x, y, z: (Nq, Nq, Nq, nelem).  Face arrays are (Nq^2, 6, nelem)."""
    D = np.asarray(D, dtype=np.float64)
    Nq, nelem = x.shape[0], x.shape[3]
    xr, xs, xt = _d_ref(D, x, 0), _d_ref(D, x, 1), _d_ref(D, x, 2)
    yr, ys, yt = _d_ref(D, y, 0), _d_ref(D, y, 1), _d_ref(D, y, 2)
    zr, zs, zt = _d_ref(D, z, 0), _d_ref(D, z, 1), _d_ref(D, z, 2)
    J = (xr * (ys * zt - zs * yt) + yr * (zs * xt - xs * zt)) + zr * (xs * yt - ys * xt)
    JI2 = 1.0 / (2.0 * J)
    yzr, yzs, yzt = y * zr - z * yr, y * zs - z * ys, y * zt - z * yt
    zxr, zxs, zxt = z * xr - x * zr, z * xs - x * zs, z * xt - x * zt
    xyr, xys, xyt = x * yr - y * xr, x * ys - y * xs, x * yt - y * xt
    del xr, xs, xt, yr, ys, yt, zr, zs, zt

    def curl(pos_arr, pos_ax, neg_arr, neg_ax):
        out = np.zeros_like(x)
        for n in range(Nq):
            for arr, ax, sgn in ((pos_arr, pos_ax, 1), (neg_arr, neg_ax, -1)):
                sl = [slice(None)] * 4
                sl[ax] = slice(n, n + 1)
                shape = [1, 1, 1, 1]
                shape[ax] = Nq
                term = D[:, n].reshape(shape) * arr[tuple(sl)]
                out = out + term if sgn > 0 else out - term
        return out * JI2

    m = dict(
        xix=curl(yzt, 1, yzs, 2), etax=curl(yzr, 2, yzt, 0), zetax=curl(yzs, 0, yzr, 1),
        xiy=curl(zxt, 1, zxs, 2), etay=curl(zxr, 2, zxt, 0), zetay=curl(zxs, 0, zxr, 1),
        xiz=curl(xyt, 1, xys, 2), etaz=curl(xyr, 2, xyt, 0), zetaz=curl(xys, 0, xyr, 1))
    N1 = Nq - 1

    def face(arr, f):
        # face node (i, j) of face f -> volume trace, linear index i + Nq j
        if f == 0:
            v = arr[0]
        elif f == 1:
            v = arr[N1]
        elif f == 2:
            v = arr[:, 0]
        elif f == 3:
            v = arr[:, N1]
        elif f == 4:
            v = arr[:, :, 0]
        else:
            v = arr[:, :, N1]
        return v.reshape(Nq * Nq, nelem, order="F")

    dirs = ("xi", "xi", "eta", "eta", "zeta", "zeta")
    nx = np.zeros((Nq * Nq, 6, nelem), order="F")
    ny = np.zeros_like(nx)
    nz = np.zeros_like(nx)
    for f in range(6):
        sgn = -1.0 if f % 2 == 0 else 1.0
        Jf = face(J, f)
        for comp, out in (("x", nx), ("y", ny), ("z", nz)):
            t = Jf * face(m[dirs[f] + comp], f)
            out[:, f] = -t if sgn < 0 else t
    sJ = _hypot3(nx, ny, nz)
    f_ = np.asfortranarray
    res = {k: f_(v) for k, v in m.items()}
    res.update(J=f_(J), sJ=f_(sJ), nx=f_(nx / sJ), ny=f_(ny / sJ), nz=f_(nz / sJ))
    return res


def _sin_libm(a):
    # libm sin on the distinct values (bitwise identical to C's sin)
    u, inv = np.unique(a, return_inverse=True)
    s = np.array([math.sin(v) for v in u])
    return s[inv].reshape(a.shape)


def warp_sinusoidal(X, amp=0.05):
    """x_i += amp * sin(x) sin(y) [sin(z)] applied to every coordinate."""
    s = _sin_libm(X[0])
    for c in X[1:]:
        s = s * _sin_libm(c)
    dx = amp * s
    return tuple(np.asfortranarray(c + dx) for c in X)


def computegeometry(dim, N, elemtocoord, vmapM, meshwarp=None):
    """vgeo (Np, nvgeo, nelem) and sgeo (nsgeo, Nfp, nface, nelem) of the set3c
    drivers.  meshwarp maps the coordinate tuple to the warped tuple."""
    r, w = lglpoints(N)
    D = spectralderivative(r)
    Nq = N + 1
    X = creategrid(elemtocoord, r)
    if meshwarp is not None:
        X = meshwarp(X)
    nelem = X[0].shape[-1]
    Np, Nfp, nface = Nq ** dim, Nq ** (dim - 1), 2 * dim
    if dim == 3:
        m = computemetric3d(*X, D)
        M = (w[None, None, :] * w[None, :, None]) * w[:, None, None]  # kron(1, ω, ω, ω)
        names, snames = VGEO3D, SGEO3D
        sM = np.array([w[n // Nq] * w[n % Nq] for n in range(Nfp)])  # kron(1, ω, ω)
    else:
        m = computemetric2d(*X, D)
        M = w[None, :] * w[:, None]  # kron(1, ω, ω): M[p, q] = ω[q] ω[p]
        names, snames = VGEO2D, SGEO2D
        sM = w.copy()
    vgeo = np.zeros((Np, len(names), nelem), order="F")
    nmet = dim * dim
    for f in range(nmet):
        vgeo[:, f, :] = m[names[f]].reshape(Np, nelem, order="F")
    MJ = M.reshape(Np, order="F")[:, None] * m["J"].reshape(Np, nelem, order="F")
    vgeo[:, nmet, :] = MJ
    vgeo[:, nmet + 1, :] = 1.0 / MJ
    for c in range(dim):
        vgeo[:, nmet + 2 + c, :] = X[c].reshape(Np, nelem, order="F")
    sgeo = np.zeros((len(snames), Nfp, nface, nelem), order="F")
    for c, key in enumerate(("nx", "ny", "nz")[:dim]):
        sgeo[c] = m[key]
    sgeo[dim] = sM[:, None, None] * m["sJ"]
    MJI = vgeo[:, nmet + 1, :].ravel(order="F")
    sgeo[dim + 1] = MJI[np.asarray(vmapM) - 1]
    return vgeo, sgeo, r, w, D
