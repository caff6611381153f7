"""Python mirror of the reference's GPU-method API for the DG hot path.

The reference dispatches `volumerhs!`, `fluxrhs!`, `updatesolution!` and the
LDG passes on the array type (`rhs::CuArray`, examples/2d_kernels/
euler2d_set3c.jl:975-996); here the same calls take CUDA torch tensors and
run the sm_100a kernels of libcanary_b200.so through its C-ABI.  Tensors hold
the reference's column-major data as flat buffers (a Julia (Np, nstate,
nelem) array is a C-order (nelem, nstate, Np) tensor), so the memory of a
`CuArray` and of these tensors is byte-for-byte the same.

Calls are asynchronous on the current torch stream (or `stream=`) and raise
`CanaryError` on any failure; nothing falls back to a CPU path.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import CanaryError, cb_phys, check
from .mesh import brickmesh, connectmesh, mappings, partition
from .metric import computegeometry

# Physical constants of the reference drivers (euler3d_set3c.jl:113-118,
# nse2d.jl:127-128): P = (R_gas/c_v)(E - |U|²/2ρ - ρ g z).
REFERENCE_PHYS = dict(gamma=1.4, R_gas=287.17, c_p=1004.67, c_v=717.5, gravity=10.0,
                      Pr=7.1, lam=-2.0 / 3.0, visc=0.0)
# The benchmark workloads: p = (γ-1)(E - ρ|u|²/2) with γ = 1.4, no gravity,
# nondimensional R = 1 (so R/c_v = γ-1 = 0.4), Pr = 0.72.
WORKLOAD_PHYS = dict(gamma=1.4, R_gas=1.0, c_p=3.5, c_v=2.5, gravity=0.0, Pr=0.72,
                     lam=-2.0 / 3.0, visc=0.0)


def make_phys(**kw) -> cb_phys:
    d = dict(WORKLOAD_PHYS)
    d.update(kw)
    return cb_phys(d["gamma"], d["R_gas"], d["c_p"], d["c_v"], d["gravity"], d["Pr"],
                   d["lam"], d["visc"])


def nstate(dim: int) -> int:
    return 5 if dim == 3 else 4


def viscous_fused(dim: int, N: int) -> bool:
    """Whether the viscous solver of (dim, N) runs the two fused passes per
    stage (element groups of at most two nodes per thread of a 256-thread
    block: every 2-D order, 3-D up to N = 7) and so takes state offsets; other
    orders run the reference's unfused pass sequence."""
    return dim == 2 or (N + 1) ** 3 <= 512


def _torch():
    import torch
    return torch


def _ptr(t, dtype, numel=None, name="array"):
    torch = _torch()
    if t is None:
        return None
    if not isinstance(t, torch.Tensor) or not t.is_cuda:
        raise TypeError(f"{name} must be a CUDA torch tensor")
    if t.dtype != dtype:
        raise TypeError(f"{name} must have dtype {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if numel is not None and t.numel() < numel:
        raise ValueError(f"{name} has {t.numel()} entries, needs {numel}")
    return C.c_void_p(t.data_ptr())


def _stream(stream):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _nelem(elems) -> int:
    return len(elems) if hasattr(elems, "__len__") else int(elems)


def _real(Q):
    torch = _torch()
    if Q.dtype == torch.float64:
        return torch.float64, ""
    if Q.dtype == torch.float32:
        return torch.float32, "_f32"
    raise TypeError("state must be float64 or float32")


def _sizes(dim, N, nelem):
    Nq = N + 1
    return Nq ** dim, Nq ** (dim - 1), 2 * dim


# ---------------------------------------------------------- per-kernel API
def volumerhs(dim, N, rhs, Q, vgeo, D, elems, phys=None, stream=None):
    """rhs += volume integral (volumerhs!, euler3d_set3c.jl:253-339)."""
    torch = _torch()
    real, suf = _real(Q)
    n = _nelem(elems)
    Np, _, _ = _sizes(dim, N, n)
    ns = nstate(dim)
    L = _lib.lib()
    check(getattr(L, "cb_volumerhs" + suf)(
        dim, N, _ptr(rhs, real, Np * ns * n, "rhs"), _ptr(Q, real, Np * ns * n, "Q"),
        _ptr(vgeo, real, Np * (14 if dim == 3 else 8) * n, "vgeo"),
        _ptr(D, real, (N + 1) ** 2, "D"), n, C.byref(phys or make_phys()), _stream(stream)))


def fluxrhs(dim, N, rhs, Q, sgeo, vgeo, elems, vmapM, vmapP, elemtobndy, phys=None, stream=None):
    """rhs -= sMJ · Rusanov flux (fluxrhs!, euler3d_set3c.jl:342-458)."""
    torch = _torch()
    real, suf = _real(Q)
    n = _nelem(elems)
    Np, Nfp, nf = _sizes(dim, N, n)
    ns = nstate(dim)
    L = _lib.lib()
    check(getattr(L, "cb_fluxrhs" + suf)(
        dim, N, _ptr(rhs, real, Np * ns * n, "rhs"), _ptr(Q, real, Np * ns * n, "Q"),
        _ptr(sgeo, real, (dim + 2) * Nfp * nf * n, "sgeo"),
        _ptr(vgeo, real, Np * (14 if dim == 3 else 8) * n, "vgeo"), n,
        _ptr(vmapM, torch.int64, Nfp * nf * n, "vmapM"), _ptr(vmapP, torch.int64, Nfp * nf * n, "vmapP"),
        _ptr(elemtobndy, torch.int64, nf * n, "elemtobndy"), C.byref(phys or make_phys()),
        _stream(stream)))


def updatesolution(dim, N, rhs, rhs_gradQ, Q, vgeo, elems, rka, rkb, dt, visc=0.0, stream=None):
    """rhs += visc rhs_gradQ[:,:,1,:]; Q += rkb dt rhs MJI; rhs *= rka
    (updatesolution!, euler3d_set3c.jl:862-872)."""
    real, suf = _real(Q)
    n = _nelem(elems)
    Np, _, _ = _sizes(dim, N, n)
    ns = nstate(dim)
    L = _lib.lib()
    check(getattr(L, "cb_updatesolution" + suf)(
        dim, N, _ptr(rhs, real, Np * ns * n, "rhs"),
        _ptr(rhs_gradQ, real, Np * ns * dim * n, "rhs_gradQ") if rhs_gradQ is not None else None,
        _ptr(Q, real, Np * ns * n, "Q"), _ptr(vgeo, real, None, "vgeo"), n, float(rka), float(rkb),
        float(dt), float(visc), _stream(stream)))


def volume_grad(dim, N, rhs, Q, vgeo, D, elems, phys=None, stream=None):
    torch = _torch()
    n = _nelem(elems)
    check(_lib.lib().cb_volume_grad(dim, N, _ptr(rhs, torch.float64), _ptr(Q, torch.float64),
                                    _ptr(vgeo, torch.float64), _ptr(D, torch.float64), n,
                                    C.byref(phys or make_phys()), _stream(stream)))


def flux_grad(dim, N, rhs, Q, sgeo, vgeo, elems, vmapM, vmapP, elemtobndy, phys=None, stream=None):
    torch = _torch()
    n = _nelem(elems)
    check(_lib.lib().cb_flux_grad(dim, N, _ptr(rhs, torch.float64), _ptr(Q, torch.float64),
                                  _ptr(sgeo, torch.float64), _ptr(vgeo, torch.float64), n,
                                  _ptr(vmapM, torch.int64), _ptr(vmapP, torch.int64),
                                  _ptr(elemtobndy, torch.int64), C.byref(phys or make_phys()),
                                  _stream(stream)))


def update_gradQ(dim, N, gradQ, rhs, vgeo, elems, stream=None):
    torch = _torch()
    n = _nelem(elems)
    check(_lib.lib().cb_update_gradQ(dim, N, _ptr(gradQ, torch.float64), _ptr(rhs, torch.float64),
                                     _ptr(vgeo, torch.float64), n, _stream(stream)))


def volume_div(dim, N, rhs, gradQ, Q, vgeo, D, elems, phys=None, stream=None):
    torch = _torch()
    n = _nelem(elems)
    check(_lib.lib().cb_volume_div(dim, N, _ptr(rhs, torch.float64), _ptr(gradQ, torch.float64),
                                   _ptr(Q, torch.float64), _ptr(vgeo, torch.float64),
                                   _ptr(D, torch.float64), n, C.byref(phys or make_phys()),
                                   _stream(stream)))


def flux_div(dim, N, rhs, gradQ, Q, sgeo, elems, vmapM, vmapP, elemtobndy, phys=None, stream=None):
    torch = _torch()
    n = _nelem(elems)
    check(_lib.lib().cb_flux_div(dim, N, _ptr(rhs, torch.float64), _ptr(gradQ, torch.float64),
                                 _ptr(Q, torch.float64), _ptr(sgeo, torch.float64), n,
                                 _ptr(vmapM, torch.int64), _ptr(vmapP, torch.int64),
                                 _ptr(elemtobndy, torch.int64), C.byref(phys or make_phys()),
                                 _stream(stream)))


NOALLOC_SCRATCH_BYTES = 32 * 1024 * 1024  # CB_NOALLOC_SCRATCH_BYTES


def lsrk_stage_noalloc(dim, N, Q, rhs, vgeo, sgeo, vmapM, vmapP, elemtobndy, D, elems, rka,
                       rkb, dt, phys=None, status=None, stream=None):
    """One fused FP64 LSRK stage without any device allocation (for hosts
    that own every device allocation): same result as volumerhs, fluxrhs and
    updatesolution in sequence.  Its scratch is a fixed static device array
    shared by all calls, so calls must not overlap on the GPU.  `status`, if
    given, is a CUDA int32 tensor that receives the kernel status bits;
    otherwise they go to a sticky word that `noalloc_status` reads."""
    torch = _torch()
    n = _nelem(elems)
    Np, Nfp, nf = _sizes(dim, N, n)
    ns = nstate(dim)
    check(_lib.lib().cb_lsrk_stage_noalloc(
        dim, N, _ptr(Q, torch.float64, Np * ns * n, "Q"), _ptr(rhs, torch.float64, Np * ns * n, "rhs"),
        _ptr(vgeo, torch.float64), _ptr(sgeo, torch.float64), _ptr(vmapM, torch.int64),
        _ptr(vmapP, torch.int64), _ptr(elemtobndy, torch.int64), _ptr(D, torch.float64), n,
        C.byref(phys or make_phys()), float(rka), float(rkb), float(dt),
        _ptr(status, torch.int32) if status is not None else None, _stream(stream)))


def noalloc_status(stream=None) -> int:
    """Synchronise, read and clear the sticky status word of the
    allocation-free stage (calls made with status=None); raises CanaryError
    for a set bit, else returns 0."""
    bits = C.c_uint(0)
    check(_lib.lib().cb_noalloc_status(_stream(stream), C.byref(bits)))
    return bits.value


def device_status(stream=None) -> None:
    """Synchronise and raise if a kernel met an invalid boundary code or a
    non-finite state since the last check."""
    check(_lib.lib().cb_device_status(_stream(stream)))


# ------------------------------------------------------------------ mesh
@dataclass
class Mesh:
    """Host-side mesh data of one DG instance, reference layouts (numpy)."""
    dim: int
    N: int
    nelem: int
    vgeo: np.ndarray
    sgeo: np.ndarray
    vmapM: np.ndarray
    vmapP: np.ndarray
    elemtobndy: np.ndarray
    D: np.ndarray
    r: np.ndarray
    w: np.ndarray
    elemtocoord: np.ndarray

    @property
    def Np(self):
        return (self.N + 1) ** self.dim

    def coords(self):
        nm = self.dim * self.dim
        return tuple(self.vgeo[:, nm + 2 + c, :] for c in range(self.dim))


def build_mesh(dim, N, x, periodic, boundary=None, meshwarp=None) -> Mesh:
    """brickmesh -> partition -> connectmesh -> mappings -> computegeometry,
    the setup sequence of euler() (euler3d_set3c.jl:1689-1708)."""
    cm = connectmesh(*partition(*brickmesh(x, periodic, boundary=boundary)))
    vmapM, vmapP = mappings(N, cm["elemtoelem"], cm["elemtoface"], cm["elemtoordr"])
    vgeo, sgeo, r, w, D = computegeometry(dim, N, cm["elemtocoord"], vmapM, meshwarp)
    return Mesh(dim, N, vgeo.shape[2], vgeo, sgeo, vmapM, vmapP, cm["elemtobndy"], D, r, w,
                cm["elemtocoord"])


def to_device(a: np.ndarray, dtype=None, device="cuda"):
    """Column-major numpy array -> flat CUDA tensor with the same memory order.
    The copy goes through pinned memory and is ordered on the current stream
    without waiting for it (a copy from pageable memory would first wait for
    all earlier work of the stream)."""
    torch = _torch()
    flat = np.asarray(a).ravel(order="F")
    t = torch.from_numpy(np.ascontiguousarray(flat))
    if dtype is not None:
        t = t.to(dtype)
    if torch.device(device).type == "cuda":
        return t.pin_memory().to(device, non_blocking=True)
    return t.to(device)


def dev_i64(a, device="cuda"):
    return to_device(a, _torch().int64, device)


def from_device(t, shape) -> np.ndarray:
    """Flat tensor -> Fortran-ordered numpy array of the Julia shape."""
    return np.asarray(t.detach().cpu().numpy()).reshape(shape, order="F")


@dataclass
class DeviceMesh:
    """Device copies of one mesh (FP64 geometry, int64 maps)."""
    mesh: Mesh
    vgeo: object
    sgeo: object
    vmapM: object
    vmapP: object
    elemtobndy: object
    D: object

    @classmethod
    def build(cls, dim, N, x, periodic, warp_amp=0.0, device="cuda", boundary=None, stream=None,
              connect="device"):
        """Brick mesh, connectivity (brickmesh -> partition -> connectmesh ->
        mappings, euler3d_set3c.jl:1689-1708) and geometry in FP64, with the
        optional warp x_c += warp_amp * prod_d sin(x_d).  The connectivity is
        built on the device (cb_brickmesh) or, with connect="host", by the
        host mirror; the grid and geometry on the device (cb_computegeometry).
        The returned mesh keeps no host copies of vgeo / sgeo (and, with the
        device connectivity, none of the maps)."""
        torch = _torch()
        from .operators import lglpoints, spectralderivative
        r, w = lglpoints(N)
        D = spectralderivative(r)
        Nq = N + 1
        Np, Nfp = Nq ** dim, Nq ** (dim - 1)
        nvg, nsg = (14, 5) if dim == 3 else (8, 4)
        dev = lambda a: to_device(a, torch.float64, device)
        keep = []
        if connect == "device":
            n = [len(xi) - 1 for xi in x]
            nelem = int(np.prod(n))
            dx = [dev(np.asarray(xi, dtype=np.float64)) for xi in x]
            keep.extend(dx)
            de2c = torch.empty(dim * 2 ** dim * nelem, dtype=torch.float64, device=device)
            detb = torch.empty(2 * dim * nelem, dtype=torch.int64, device=device)
            dvM = torch.empty(Nfp * 2 * dim * nelem, dtype=torch.int64, device=device)
            dvP = torch.empty_like(dvM)
            bnd = None
            if boundary is not None:
                b = np.asarray(boundary, dtype=np.int64).reshape(2, dim, order="F")
                bnd = (C.c_int64 * (2 * dim))(*[int(v) for v in b.ravel(order="F")])
            check(_lib.lib().cb_brickmesh(
                dim, N, (C.c_int64 * dim)(*n), (C.c_void_p * dim)(*[t.data_ptr() for t in dx]),
                (C.c_int * dim)(*[1 if p else 0 for p in periodic]), bnd, _ptr(de2c, torch.float64),
                _ptr(detb, torch.int64), _ptr(dvM, torch.int64), _ptr(dvP, torch.int64), _stream(stream)))
            vmapM = vmapP = etb = e2c = None
        else:
            cm = connectmesh(*partition(*brickmesh(x, periodic, boundary=boundary)))
            vmapM, vmapP = mappings(N, cm["elemtoelem"], cm["elemtoface"], cm["elemtoordr"])
            e2c = np.asarray(cm["elemtocoord"], dtype=np.float64)
            etb = cm["elemtobndy"]
            nelem = e2c.shape[2]
            de2c = dev(e2c)
            dvM, dvP, detb = dev_i64(vmapM, device), dev_i64(vmapP, device), dev_i64(etb, device)
        dr, dw, dD = dev(np.asarray(r)), dev(np.asarray(w)), dev(D)
        keep.extend([dr, dw])
        vgeo = torch.empty(Np * nvg * nelem, dtype=torch.float64, device=device)
        sgeo = torch.empty(nsg * Nfp * 2 * dim * nelem, dtype=torch.float64, device=device)
        check(_lib.lib().cb_computegeometry(dim, N, nelem, _ptr(de2c, torch.float64), float(warp_amp),
                                            _ptr(dr, torch.float64), _ptr(dw, torch.float64),
                                            _ptr(dD, torch.float64), _ptr(vgeo, torch.float64),
                                            _ptr(sgeo, torch.float64), _stream(stream)))
        mesh = Mesh(dim, N, nelem, None, None, vmapM, vmapP, etb, D, np.asarray(r), np.asarray(w), e2c)
        out = cls(mesh, vgeo, sgeo, dvM, dvP, detb, dD)
        out.elemtocoord = de2c  # device (dim, 2^dim, nelem); with the inputs of the set-up kernels
        out._keep = keep
        return out

    def coords(self):
        """Node coordinates as device tensors (nelem, Np), one per dimension."""
        m = self.mesh
        nvg = 14 if m.dim == 3 else 8
        v = self.vgeo.view(m.nelem, nvg, m.Np)
        return tuple(v[:, m.dim * m.dim + 2 + c, :] for c in range(m.dim))

    @classmethod
    def upload(cls, mesh: Mesh, device="cuda"):
        torch = _torch()
        return cls(mesh, to_device(mesh.vgeo, torch.float64, device), to_device(mesh.sgeo, torch.float64, device),
                   to_device(mesh.vmapM, torch.int64, device), to_device(mesh.vmapP, torch.int64, device),
                   to_device(mesh.elemtobndy, torch.int64, device), to_device(mesh.D, torch.float64, device))


# ---------------------------------------------------------------- solver
class LSRK:
    """Fused, graph-captured LSRK(5,4) driver bound to one state (the
    lowstorageRK of euler3d_set3c.jl:1361-1523 / nse2d.jl:1728-1890).

    Q and rhs are CUDA tensors owned by the caller (float64 for precision 64,
    float32 for precision 32); they are advanced in place."""

    def __init__(self, dmesh: DeviceMesh, Q, rhs, precision=64, phys=None, stream=None):
        torch = _torch()
        m = dmesh.mesh
        real = torch.float64 if precision == 64 else torch.float32
        n = m.nelem * m.Np * nstate(m.dim)
        self.dmesh, self.Q, self.rhs, self.precision = dmesh, Q, rhs, precision
        self.phys = phys or make_phys()
        self._h = C.c_void_p()
        self._stream = stream
        check(_lib.lib().cb_solver_create(
            C.byref(self._h), m.dim, m.N, precision, m.nelem, _ptr(Q, real, n, "Q"),
            _ptr(rhs, real, n, "rhs"), _ptr(dmesh.vgeo, torch.float64), _ptr(dmesh.sgeo, torch.float64),
            _ptr(dmesh.vmapM, torch.int64), _ptr(dmesh.vmapP, torch.int64),
            _ptr(dmesh.elemtobndy, torch.int64), _ptr(dmesh.D, torch.float64),
            C.byref(self.phys), _stream(stream)))

    @classmethod
    def for_state(cls, dmesh: DeviceMesh, Q: np.ndarray, precision=64, phys=None, stream=None,
                  offset=None):
        """Solver for a host state Q (Np, nstate, nelem).  For precision 32 the
        device state holds Q - qref with qref = per-field mean of Q (unless
        `offset` is given), which keeps the FP32 update's rounding relative to
        the deviation; `state()` returns the full FP64 state."""
        torch = _torch()
        Q = np.asarray(Q, dtype=np.float64)
        ns = Q.shape[1]
        if offset is None:
            offset = Q.mean(axis=(0, 2)) if precision == 32 else np.zeros(ns)
        offset = np.asarray(offset, dtype=np.float64)
        real = torch.float64 if precision == 64 else torch.float32
        dev = dmesh.vgeo.device
        dQ = to_device(Q - offset[None, :, None], real, dev)
        drhs = torch.zeros_like(dQ)
        s = cls(dmesh, dQ, drhs, precision, phys, stream)
        s.set_offset(offset)
        return s

    def set_offset(self, qref) -> None:
        ns = nstate(self.dmesh.mesh.dim)
        arr = (C.c_double * 5)(*([float(v) for v in qref] + [0.0] * (5 - ns)))
        check(_lib.lib().cb_solver_set_offset(self._h, arr))
        self.offset = np.array(list(qref)[:ns], dtype=np.float64)

    def state(self) -> np.ndarray:
        """Full FP64 state (Np, nstate, nelem) on the host."""
        m = self.dmesh.mesh
        shape = (m.Np, nstate(m.dim), m.nelem)
        off = getattr(self, "offset", np.zeros(shape[1]))
        return from_device(self.Q.double(), shape) + off[None, :, None]

    def run(self, nsteps: int, dt: float) -> None:
        check(_lib.lib().cb_lsrk_run(self._h, int(nsteps), float(dt)))

    def status_async(self, host) -> None:
        """Enqueue a copy of the status bits into `host` (a pinned int32
        tensor) on the solver's stream."""
        check(_lib.lib().cb_solver_status_async(self._h, C.c_void_p(host.data_ptr())))

    def set_kernel(self, kernel: int) -> None:
        """Stage kernel: 0 = the shape's default, 1 = the CUDA-core stages,
        2 = the tensor-core (DMMA) stage of the inviscid 3-D N=7 form, 3 = the
        unpipelined grouped stages (for the fused viscous form: the grouped
        passes instead of the pipelined ones), 4 = the lean pipelined stage
        of the inviscid form (only the state staged in shared memory)."""
        check(_lib.lib().cb_solver_set_kernel(self._h, int(kernel)))

    @property
    def kernel(self) -> int:
        """The stage kernel the solver runs: 1 CUDA-core, 2 tensor-core, 3
        grouped, 4 lean."""
        v = C.c_int(0)
        check(_lib.lib().cb_solver_get_kernel(self._h, C.byref(v)))
        return v.value

    def reset_status(self) -> None:
        """Clear the solver's sticky status bits (stream-ordered)."""
        check(_lib.lib().cb_solver_reset_status(self._h))

    def test_timeout(self) -> None:
        """Test hook of the bounded device waits: enqueue one stage whose
        first state copy per block is withheld, so that every block's wait
        gives up; the stage stores nothing and raises the timeout status
        (CB_ERR_TIMEOUT from `sums`)."""
        check(_lib.lib().cb_solver_test_timeout(self._h))

    def sums(self) -> np.ndarray:
        """Compensated FP64 (Σ MJ Q_s, Σ MJ Q_s²) per field, shape (2, nstate)."""
        ns = nstate(self.dmesh.mesh.dim)
        out = (C.c_double * (2 * ns))()
        check(_lib.lib().cb_solver_sums(self._h, out))
        return np.array(out[:]).reshape(2, ns)

    def close(self) -> None:
        if self._h:
            _lib.lib().cb_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def lowstorageRK(dim, N, dmesh: DeviceMesh, Q, rhs, dt, nsteps, precision=64, phys=None, stream=None):
    """Advance Q (and the residual carry rhs) by nsteps LSRK(5,4) steps."""
    s = LSRK(dmesh, Q, rhs, precision, phys, stream)
    try:
        s.run(nsteps, dt)
    finally:
        s.close()
