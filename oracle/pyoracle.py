"""ctypes front end of the C oracle (oracle/canary_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and by
the CPU-baseline / reference arm of bench.py, always as the checker or the
timed CPU restatement, never as part of the product.

Arrays follow the reference's Julia layouts and are returned as Fortran-ordered
numpy arrays with the Julia shapes, e.g. Q is (Np, nstate, nelem), vgeo is
(Np, nvgeo, nelem), sgeo is (nsgeo, Nfp, nface, nelem) and vmapM/vmapP are
(Nfp, nface, nelem) int64 holding 1-based node ids.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

# reference constants (examples/3d_kernels/euler3d_set3c.jl:113-118,
# examples/2d_kernels/nse2d.jl:127-128)
REFERENCE_PHYS = dict(gamma=1.4, R_gas=287.17, c_p=1004.67, c_v=717.5,
                      gravity=10.0, Pr=7.1, **{"lambda": -2.0 / 3.0}, visc=0.0)


def build(force: bool = False) -> str:
    """Compile liboracle.so with the Makefile next to this file."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE, "liboracle.so"], check=True)
    return _LIB_PATH


class Phys(C.Structure):
    _fields_ = [(n, C.c_double) for n in
                ("gamma", "R_gas", "c_p", "c_v", "gravity", "Pr", "lambda_", "visc")]


def make_phys(**kw) -> Phys:
    d = dict(REFERENCE_PHYS)
    d.update(kw)
    return Phys(d["gamma"], d["R_gas"], d["c_p"], d["c_v"], d["gravity"],
                d["Pr"], d["lambda"], d["visc"])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _lib.or_brickmesh.restype = C.c_int64
        _lib.or_L2energysquared.restype = C.c_double
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data)


def _f64(shape):
    return np.zeros(shape, dtype=np.float64, order="F")


def _i64(shape):
    return np.zeros(shape, dtype=np.int64, order="F")


class OracleError(RuntimeError):
    pass


# ---------------------------------------------------------------- quadrature
def legendre_coefs(n):
    a, b = _f64(n), _f64(n + 1)
    lib().or_legendre_coefs(n, _p(a), _p(b))
    return a, b


def custom_gauss_rule(lo, hi, a, b, endpt, maxits=30):
    a = np.array(a, dtype=np.float64)
    b = np.array(b, dtype=np.float64)
    n = len(a)
    x, w = _f64(n), _f64(n)
    it = C.c_int(0)
    rc = lib().or_custom_gauss_rule(C.c_double(lo), C.c_double(hi), n, _p(a), _p(b),
                                    C.c_char(endpt.encode()), maxits, _p(x), _p(w),
                                    C.byref(it))
    if rc == 1:
        raise OracleError("Must have at least two points for both ends.")
    if rc == 2:
        raise OracleError(f"No convergence after {it.value} iterations "
                          "(try increasing maxits)")
    return x, w


def legendre(n, endpt="N"):
    a, b = legendre_coefs(n)
    return custom_gauss_rule(-1.0, 1.0, a, b, endpt)


def lglpoints(N):
    return legendre(N + 1, "B")


def lgpoints(N):
    return legendre(N + 1, "N")


def baryweights(r):
    r = np.ascontiguousarray(r, dtype=np.float64)
    wb = _f64(len(r))
    lib().or_baryweights(len(r), _p(r), _p(wb))
    return wb


def spectralderivative(r):
    r = np.ascontiguousarray(r, dtype=np.float64)
    D = _f64((len(r), len(r)))
    lib().or_spectralderivative(len(r), _p(r), _p(D))
    return D


def interpolationmatrix(rsrc, rdst):
    rsrc = np.ascontiguousarray(rsrc, dtype=np.float64)
    rdst = np.ascontiguousarray(rdst, dtype=np.float64)
    I = _f64((len(rdst), len(rsrc)))
    lib().or_interpolationmatrix(len(rsrc), _p(rsrc), len(rdst), _p(rdst), _p(I))
    return I


# ---------------------------------------------------------------------- mesh
def hilbertcode(Y, bits=64):
    Y = np.ascontiguousarray(Y, dtype=np.uint64)
    H = np.zeros(len(Y), dtype=np.uint64)
    lib().or_hilbertcode(len(Y), _p(Y), bits, _p(H))
    return H


def centroidtocode(elemtocoord):
    etc = np.asfortranarray(elemtocoord, dtype=np.float64)
    d, nvert, nelem = etc.shape
    code = np.zeros((d, nelem), dtype=np.uint64, order="F")
    lib().or_centroidtocode(d, nvert, C.c_int64(nelem), _p(etc), _p(code))
    return code


def vertsortandorder(*v):
    vin = np.array(v, dtype=np.int64)
    out = np.zeros(len(v), dtype=np.int64)
    o = C.c_int(0)
    flips = (C.c_int * 5)()
    rc = lib().or_vertsortandorder(len(v), _p(vin), _p(out), C.byref(o), flips)
    if rc:
        raise OracleError("Problem finding vertex ordering "
                          f"{tuple(int(t) for t in out)} with flips "
                          f"{tuple(bool(flips[i]) for i in range(len(v) if len(v) < 4 else 5))}")
    return tuple(int(t) for t in out), o.value


def brickmesh(x, periodic, part=1, numparts=1, boundary=None):
    d = len(x)
    if boundary is None:
        boundary = np.ones((2, d), dtype=np.int64)
    bnd = np.asfortranarray(np.array(boundary, dtype=np.int64).reshape(2, d, order="F"))
    xs = np.concatenate([np.asarray(xi, dtype=np.float64) for xi in x])
    nx = np.array([len(xi) for xi in x], dtype=np.int64)
    per = np.array([1 if p else 0 for p in periodic], dtype=np.int32)
    total = int(np.prod(nx - 1))
    maxloc = total // numparts + 2
    nvert, nface, nfv = 2 ** d, 2 * d, 2 ** (d - 1)
    etv = _i64((nvert, maxloc))
    etc = _f64((d, nvert, maxloc))
    etb = _i64((nface, maxloc))
    fc = np.zeros((maxloc * d + 1, 2 + nfv), dtype=np.int64)  # row-major rows
    nfc = C.c_int64(0)
    nloc = lib().or_brickmesh(d, _p(xs), _p(nx), _p(per), C.c_int64(part),
                              C.c_int64(numparts), _p(bnd), _p(etv), _p(etc),
                              _p(etb), _p(fc), C.byref(nfc))
    if nloc < 0:
        raise OracleError("bad brickmesh arguments")
    return (np.asfortranarray(etv[:, :nloc]), np.asfortranarray(etc[:, :, :nloc]),
            np.asfortranarray(etb[:, :nloc]), [list(r) for r in fc[:nfc.value]])


def partition(etv, etc, etb, fc):
    etv = np.array(etv, dtype=np.int64, order="F")
    etc = np.array(etc, dtype=np.float64, order="F")
    etb = np.array(etb, dtype=np.int64, order="F")
    d, nvert, nelem = etc.shape
    nfv = 2 ** (d - 1)
    fca = np.zeros((max(len(fc), 1) + d * nelem, 2 + nfv), dtype=np.int64)
    for i, row in enumerate(fc):
        fca[i] = row
    nfc = C.c_int64(len(fc))
    lib().or_partition(d, C.c_int64(nelem), _p(etv), _p(etc), _p(etb), _p(fca),
                       C.byref(nfc))
    return etv, etc, etb, [list(r) for r in fca[:nfc.value]]


def connectmesh(etv, etc, etb, fc):
    etv = np.asfortranarray(etv, dtype=np.int64)
    etb_in = np.asfortranarray(etb, dtype=np.int64)
    d, nvert, nelem = np.shape(etc)
    nface, nfv = 2 * d, 2 ** (d - 1)
    fca = np.zeros((max(len(fc), 1), 2 + nfv), dtype=np.int64)
    for i, row in enumerate(fc):
        fca[i] = row
    e2e, e2f, e2o, e2b = (_i64((nface, nelem)) for _ in range(4))
    rc = lib().or_connectmesh(d, C.c_int64(nelem), _p(etv), _p(etb_in), _p(fca),
                              C.c_int64(len(fc)), _p(e2e), _p(e2f), _p(e2o), _p(e2b))
    if rc == 1:
        raise OracleError("Problem finding vertex ordering")
    if rc == 2:
        raise OracleError("TODO add support for other orientations")
    return dict(elemtocoord=np.asfortranarray(etc), elemtoelem=e2e, elemtoface=e2f,
                elemtoordr=e2o, elemtobndy=e2b, elems=range(1, nelem + 1),
                realelems=range(1, nelem + 1))


def mappings(N, elemtoelem, elemtoface, elemtoordr):
    e2e = np.asfortranarray(elemtoelem, dtype=np.int64)
    e2f = np.asfortranarray(elemtoface, dtype=np.int64)
    e2o = np.asfortranarray(elemtoordr, dtype=np.int64)
    nface, nelem = e2e.shape
    d = nface // 2
    Nfp = (N + 1) ** (d - 1)
    vmapM, vmapP = _i64((Nfp, nface, nelem)), _i64((Nfp, nface, nelem))
    rc = lib().or_mappings(d, N, C.c_int64(nelem), _p(e2e), _p(e2f), _p(e2o),
                           _p(vmapM), _p(vmapP))
    if rc:
        raise OracleError("unsupported face orientation")
    return vmapM, vmapP


# -------------------------------------------------------------------- metric
def creategrid(elemtocoord, r):
    e2c = np.asfortranarray(elemtocoord, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    d, _, nelem = e2c.shape
    Nq = len(r)
    shape = (Nq,) * d + (nelem,)
    X = [_f64(shape) for _ in range(3)]
    lib().or_creategrid(d, Nq, C.c_int64(nelem), _p(e2c), _p(r), _p(X[0]), _p(X[1]), _p(X[2]))
    return tuple(X[:d])


def computemetric(D, *X):
    D = np.asfortranarray(D, dtype=np.float64)
    Nq = D.shape[0]
    d = len(X)
    X = [np.asfortranarray(x, dtype=np.float64) for x in X]
    nelem = X[0].shape[-1]
    vshape = X[0].shape
    if d == 1:
        J, xix = _f64(vshape), _f64(vshape)
        sJ, nx = _f64((1, 2, nelem)), _f64((1, 2, nelem))
        lib().or_computemetric1d(Nq, C.c_int64(nelem), _p(X[0]), _p(J), _p(xix), _p(sJ), _p(nx), _p(D))
        return dict(J=J, xix=xix, sJ=sJ, nx=nx)
    if d == 2:
        A = [_f64(vshape) for _ in range(5)]
        S = [_f64((Nq, 4, nelem)) for _ in range(3)]
        lib().or_computemetric2d(Nq, C.c_int64(nelem), _p(X[0]), _p(X[1]), *[_p(a) for a in A],
                                 *[_p(s) for s in S], _p(D))
        return dict(J=A[0], xix=A[1], etax=A[2], xiy=A[3], etay=A[4], sJ=S[0], nx=S[1], ny=S[2])
    A = [_f64(vshape) for _ in range(10)]
    S = [_f64((Nq * Nq, 6, nelem)) for _ in range(4)]
    lib().or_computemetric3d(Nq, C.c_int64(nelem), _p(X[0]), _p(X[1]), _p(X[2]),
                             *[_p(a) for a in A], *[_p(s) for s in S], _p(D))
    names = ["J", "xix", "etax", "zetax", "xiy", "etay", "zetay", "xiz", "etaz", "zetaz"]
    out = {n: a for n, a in zip(names, A)}
    out.update(sJ=S[0], nx=S[1], ny=S[2], nz=S[3])
    return out


def computegeometry(dim, N, elemtocoord, vmapM, warp=0, warp_amp=0.05):
    e2c = np.asfortranarray(elemtocoord, dtype=np.float64)
    vmapM = np.asfortranarray(vmapM, dtype=np.int64)
    nelem = e2c.shape[2]
    Nq = N + 1
    Np, Nfp, nface = Nq ** dim, Nq ** (dim - 1), 2 * dim
    nvgeo, nsgeo = (14, 5) if dim == 3 else (8, 4)
    vgeo = _f64((Np, nvgeo, nelem))
    sgeo = _f64((nsgeo, Nfp, nface, nelem))
    rc = lib().or_computegeometry(dim, N, C.c_int64(nelem), _p(e2c), _p(vmapM), warp,
                                  C.c_double(warp_amp), _p(vgeo), _p(sgeo))
    if rc:
        raise OracleError(f"computegeometry failed ({rc})")
    return vgeo, sgeo


# ----------------------------------------------------------- full mesh setup
@dataclass
class Setup:
    dim: int
    N: int
    nelem: int
    r: np.ndarray
    w: np.ndarray
    D: np.ndarray
    vgeo: np.ndarray
    sgeo: np.ndarray
    vmapM: np.ndarray
    vmapP: np.ndarray
    elemtobndy: np.ndarray
    elemtocoord: np.ndarray
    elemtoelem: np.ndarray
    elemtoface: np.ndarray


def setup(dim, N, x, periodic, warp=0, warp_amp=0.05, boundary=None):
    """brickmesh -> partition -> connectmesh -> mappings -> lglpoints ->
    spectralderivative -> computegeometry, as euler() does
    (euler3d_set3c.jl:1689-1708)."""
    mesh = partition(*brickmesh(x, periodic, boundary=boundary))
    cm = connectmesh(*mesh)
    vmapM, vmapP = mappings(N, cm["elemtoelem"], cm["elemtoface"], cm["elemtoordr"])
    r, w = lglpoints(N)
    D = spectralderivative(r)
    vgeo, sgeo = computegeometry(dim, N, cm["elemtocoord"], vmapM, warp, warp_amp)
    return Setup(dim, N, vgeo.shape[2], r, w, D, vgeo, sgeo, vmapM, vmapP,
                 cm["elemtobndy"], cm["elemtocoord"], cm["elemtoelem"], cm["elemtoface"])


# ---------------------------------------------------------------- RHS kernels
def _nthreads(n):
    if n is None:
        return os.cpu_count() or 1
    return n


def volumerhs(dim, N, rhs, Q, vgeo, D, phys=None, nthreads=None):
    phys = phys or make_phys()
    nelem = Q.shape[-1]
    lib().or_volumerhs(dim, N, _p(rhs), _p(Q), _p(vgeo), _p(D), C.c_int64(nelem),
                       C.byref(phys), _nthreads(nthreads))


def fluxrhs(dim, N, rhs, Q, sgeo, vgeo, vmapM, vmapP, elemtobndy, phys=None, nthreads=None):
    phys = phys or make_phys()
    nelem = Q.shape[-1]
    rc = lib().or_fluxrhs(dim, N, _p(rhs), _p(Q), _p(sgeo), _p(vgeo), C.c_int64(nelem),
                          _p(vmapM), _p(vmapP), _p(elemtobndy), C.byref(phys),
                          _nthreads(nthreads))
    if rc:
        raise OracleError("Invalid boundary conditions")


def updatesolution(dim, N, rhs, Q, vgeo, rka, rkb, dt, rhs_gradQ=None, visc=0.0, nthreads=None):
    nelem = Q.shape[-1]
    lib().or_updatesolution(dim, N, _p(rhs), _p(rhs_gradQ) if rhs_gradQ is not None else None,
                            _p(Q), _p(vgeo), C.c_int64(nelem), C.c_double(rka),
                            C.c_double(rkb), C.c_double(dt), C.c_double(visc),
                            _nthreads(nthreads))


def volume_grad(dim, N, rhs, Q, vgeo, D, phys=None, nthreads=None):
    phys = phys or make_phys()
    lib().or_volume_grad(dim, N, _p(rhs), _p(Q), _p(vgeo), _p(D), C.c_int64(Q.shape[-1]),
                         C.byref(phys), _nthreads(nthreads))


def flux_grad(dim, N, rhs, Q, sgeo, vgeo, vmapM, vmapP, elemtobndy, phys=None, nthreads=None):
    phys = phys or make_phys()
    rc = lib().or_flux_grad(dim, N, _p(rhs), _p(Q), _p(sgeo), _p(vgeo), C.c_int64(Q.shape[-1]),
                            _p(vmapM), _p(vmapP), _p(elemtobndy), C.byref(phys),
                            _nthreads(nthreads))
    if rc:
        raise OracleError("Invalid boundary conditions")


def update_gradQ(dim, N, gradQ, rhs, vgeo, nthreads=None):
    lib().or_update_gradQ(dim, N, _p(gradQ), _p(rhs), _p(vgeo), C.c_int64(gradQ.shape[-1]),
                          _nthreads(nthreads))


def volume_div(dim, N, rhs, gradQ, Q, vgeo, D, phys=None, nthreads=None):
    phys = phys or make_phys()
    lib().or_volume_div(dim, N, _p(rhs), _p(gradQ), _p(Q), _p(vgeo), _p(D),
                        C.c_int64(Q.shape[-1]), C.byref(phys), _nthreads(nthreads))


def flux_div(dim, N, rhs, gradQ, Q, sgeo, vmapM, vmapP, elemtobndy, phys=None, nthreads=None):
    phys = phys or make_phys()
    rc = lib().or_flux_div(dim, N, _p(rhs), _p(gradQ), _p(Q), _p(sgeo), C.c_int64(Q.shape[-1]),
                           _p(vmapM), _p(vmapP), _p(elemtobndy), C.byref(phys),
                           _nthreads(nthreads))
    if rc:
        raise OracleError("Invalid boundary conditions")


def lowstorageRK(dim, N, vgeo, sgeo, Q, rhs, D, dt, nsteps, vmapM, vmapP, elemtobndy,
                 phys=None, nthreads=None):
    """Advance Q (and the residual carry rhs) in place by nsteps LSRK(5,4) steps."""
    phys = phys or make_phys()
    for a in (vgeo, sgeo, Q, rhs, D, vmapM, vmapP, elemtobndy):
        assert a.flags.f_contiguous or a.flags.c_contiguous and a.ndim == 1
    rc = lib().or_lowstorageRK(dim, N, C.c_int64(Q.shape[-1]), _p(vgeo), _p(sgeo), _p(Q),
                               _p(rhs), _p(D), C.c_double(dt), C.c_int64(nsteps), _p(vmapM),
                               _p(vmapP), _p(elemtobndy), C.byref(phys), _nthreads(nthreads))
    if rc:
        raise OracleError("Invalid boundary conditions")


def L2energysquared(dim, N, Q, vgeo):
    nstate = Q.shape[1]
    return lib().or_L2energysquared(dim, N, nstate, _p(Q), _p(vgeo), C.c_int64(Q.shape[-1]))
