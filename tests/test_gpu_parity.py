"""GPU parity: the sm_100a kernels, called through the C-ABI, against the CPU
oracle on the same seeded inputs.

Tolerances (relative L2 per state field):
  * single kernel call, FP64 ............................ 1e-13
  * full LSRK(5,4) runs, FP64 (incl. 500-step vortex) ... 1e-12
  * FP32 precision form vs the FP64 oracle .............. 1e-5
"""
import math
import os

import numpy as np
import pytest

from conftest import cuda_available
from oracle import pyoracle as O
from canary_b200 import dg, ic

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

NT = os.cpu_count() or 1


def oracle_phys(d):
    d = dict(d)
    d["lambda"] = d.pop("lam")
    return O.make_phys(**d)


def relerr(a, b, axis_state=1):
    a = np.asarray(a)
    b = np.asarray(b)
    out = []
    for s in range(a.shape[axis_state]):
        x = np.take(a, s, axis=axis_state)
        y = np.take(b, s, axis=axis_state)
        den = np.linalg.norm(y)
        out.append(np.linalg.norm(x - y) / (den if den > 0 else 1.0))
    return max(out)


def make_mesh(dim, N, n=3, periodic=True, warp=True, L=1.0):
    x = (np.linspace(0.0, L, n + 1),) * dim
    per = (True,) * dim if periodic else (True,) * (dim - 1) + (False,)
    from canary_b200.metric import warp_sinusoidal
    return dg.build_mesh(dim, N, x, per, meshwarp=(lambda X: warp_sinusoidal(X, 0.05)) if warp else None)


def random_state(mesh, seed=0, big=False):
    rng = np.random.default_rng(seed)
    dim, Np, ne = mesh.dim, mesh.Np, mesh.nelem
    ns = dg.nstate(dim)
    scale = 100.0 if big else 1.0
    rho = 1.0 + 0.2 * rng.random((Np, ne))
    vel = [0.3 * (rng.random((Np, ne)) - 0.5) for _ in range(dim)]
    p = scale * (1.0 + 0.2 * rng.random((Np, ne)))
    Q = np.zeros((Np, ns, ne), order="F")
    for c in range(dim):
        Q[:, c] = rho * vel[c]
    ir, ie = (3, 4) if dim == 3 else (2, 3)
    Q[:, ir] = rho
    Q[:, ie] = p / 0.4 + 0.5 * rho * sum(v * v for v in vel)
    return Q


def dev(a, dtype=None):
    import torch
    return dg.to_device(a, dtype)


PHYS_SETS = {"workload": dg.WORKLOAD_PHYS, "reference": dg.REFERENCE_PHYS}


@pytest.mark.parametrize("dim,N", [(2, 1), (2, 4), (2, 8), (3, 1), (3, 3), (3, 4), (3, 7), (3, 10)])
@pytest.mark.parametrize("physname", ["workload", "reference"])
def test_volumerhs_parity(dim, N, physname):
    import torch
    m = make_mesh(dim, N, n=2 if N >= 7 else 3)
    ph = PHYS_SETS[physname]
    Q = random_state(m, 1, big=physname == "reference")
    rhs0 = np.asfortranarray(np.random.default_rng(2).standard_normal(Q.shape))
    ref = rhs0.copy(order="F")
    O.volumerhs(dim, N, ref, Q, m.vgeo, m.D, oracle_phys(ph), NT)
    dm = dg.DeviceMesh.upload(m)
    dQ, drhs = dev(Q), dev(rhs0)
    dg.volumerhs(dim, N, drhs, dQ, dm.vgeo, dm.D, m.nelem, dg.make_phys(**ph))
    out = dg.from_device(drhs, Q.shape)
    assert relerr(out, ref) < 1e-13


@pytest.mark.parametrize("dim,N", [(2, 1), (2, 4), (2, 7), (3, 1), (3, 4), (3, 7), (3, 10)])
@pytest.mark.parametrize("walls", [False, True])
def test_fluxrhs_parity(dim, N, walls):
    m = make_mesh(dim, N, n=2 if N >= 7 else 3, periodic=not walls)
    if walls:
        assert (m.elemtobndy == 1).any()
    ph = dg.REFERENCE_PHYS if walls else dg.WORKLOAD_PHYS
    Q = random_state(m, 3, big=walls)
    rhs0 = np.asfortranarray(np.random.default_rng(4).standard_normal(Q.shape))
    ref = rhs0.copy(order="F")
    O.fluxrhs(dim, N, ref, Q, m.sgeo, m.vgeo, m.vmapM, m.vmapP, m.elemtobndy, oracle_phys(ph), NT)
    dm = dg.DeviceMesh.upload(m)
    dQ, drhs = dev(Q), dev(rhs0)
    dg.fluxrhs(dim, N, drhs, dQ, dm.sgeo, dm.vgeo, m.nelem, dm.vmapM, dm.vmapP, dm.elemtobndy,
               dg.make_phys(**ph))
    dg.device_status()
    out = dg.from_device(drhs, Q.shape)
    assert relerr(out, ref) < 1e-13


@pytest.mark.parametrize("dim,N", [(2, 4), (3, 7)])
def test_updatesolution_parity(dim, N):
    m = make_mesh(dim, N, n=2)
    Q = random_state(m, 5)
    rhs0 = np.asfortranarray(np.random.default_rng(6).standard_normal(Q.shape))
    rq, rr = Q.copy(order="F"), rhs0.copy(order="F")
    O.updatesolution(dim, N, rr, rq, m.vgeo, -0.4, 0.3, 1e-3)
    dm = dg.DeviceMesh.upload(m)
    dQ, drhs = dev(Q), dev(rhs0)
    dg.updatesolution(dim, N, drhs, None, dQ, dm.vgeo, m.nelem, -0.4, 0.3, 1e-3)
    assert relerr(dg.from_device(dQ, Q.shape), rq) < 1e-14
    assert relerr(dg.from_device(drhs, Q.shape), rr) < 1e-14


def vortex_setup():
    m = dg.build_mesh(2, 4, (np.linspace(0, 10, 11),) * 2, (True, True))
    x, y = m.coords()
    U, V, rho, E = ic.isentropic_vortex(x, y)
    Q = np.zeros((m.Np, 4, m.nelem), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3] = U, V, rho, E
    return m, Q


def test_fused_lsrk_vortex_500_steps():
    """The 2-D isentropic-vortex workload (10x10 quads, N=4, dt=0.002, 500
    steps) through the fused, graph-captured driver vs the oracle."""
    m, Q = vortex_setup()
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(2, 4, m.vgeo, m.sgeo, ref, rref, m.D, 0.002, 500, m.vmapM, m.vmapP,
                   m.elemtobndy, oracle_phys(dg.WORKLOAD_PHYS), NT)
    dm = dg.DeviceMesh.upload(m)
    dQ, drhs = dev(Q), dev(np.zeros_like(Q))
    s = dg.LSRK(dm, dQ, drhs, 64, dg.make_phys())
    s.run(500, 0.002)
    out = dg.from_device(dQ, Q.shape)
    assert relerr(out, ref) < 1e-12
    assert relerr(dg.from_device(drhs, Q.shape), rref) < 1e-9  # residual carry (small values)
    sums = s.sums()
    mj = m.vgeo[:, 4, :]
    assert np.allclose(sums[0], [(mj * ref[:, q]).sum() for q in range(4)], rtol=1e-12)
    s.close()


@pytest.mark.parametrize("N,n,nsteps", [(7, 4, 1), (7, 4, 7), (7, 8, 4), (4, 8, 2), (3, 6, 2), (10, 2, 2)])
def test_fused_lsrk_3d_warped(N, n, nsteps):
    """Fused driver on warped periodic cubes; n=8 at N=7 gives more elements
    than SMs so every block runs several pipelined iterations; N=4 and N=3
    stage through per-thread async copies (slab sizes not 16-byte multiples)
    and N=10 uses the non-pipelined stage kernel."""
    m = make_mesh(3, N, n=n, L=2 * math.pi)
    x, y, z = m.coords()
    U, V, W, rho, E = ic.fourier_state(x, y, z, seed=0)
    Q = np.zeros((m.Np, 5, m.nelem), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3], Q[:, 4] = U, V, W, rho, E
    dt = ic.fourier_dt(Q, N, h=2 * math.pi / n)
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(3, N, m.vgeo, m.sgeo, ref, rref, m.D, dt, nsteps, m.vmapM, m.vmapP,
                   m.elemtobndy, oracle_phys(dg.WORKLOAD_PHYS), NT)
    dm = dg.DeviceMesh.upload(m)
    dQ, drhs = dev(Q), dev(np.zeros_like(Q))
    s = dg.LSRK(dm, dQ, drhs, 64)
    s.run(nsteps, dt)
    assert relerr(dg.from_device(dQ, Q.shape), ref) < 1e-12
    s.close()


@pytest.mark.parametrize("n_side,N", [(40, 4), (24, 3), (16, 7)])
def test_fused_lsrk_2d_many_blocks(n_side, N):
    """2-D vortex on finer meshes: more element groups than SMs, so the
    pipelined stage kernel iterates."""
    m = dg.build_mesh(2, N, (np.linspace(0, 10, n_side + 1),) * 2, (True, True))
    x, y = m.coords()
    U, V, rho, E = ic.isentropic_vortex(x, y)
    Q = np.zeros((m.Np, 4, m.nelem), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3] = U, V, rho, E
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(2, N, m.vgeo, m.sgeo, ref, rref, m.D, 0.001, 60, m.vmapM, m.vmapP,
                   m.elemtobndy, oracle_phys(dg.WORKLOAD_PHYS), NT)
    s = dg.LSRK(dg.DeviceMesh.upload(m), dev(Q), dev(np.zeros_like(Q)), 64)
    s.run(60, 0.001)
    assert relerr(dg.from_device(s.Q, Q.shape), ref) < 1e-12
    s.close()


def test_fp32_precision_form_vortex():
    m, Q = vortex_setup()
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(2, 4, m.vgeo, m.sgeo, ref, rref, m.D, 0.002, 500, m.vmapM, m.vmapP,
                   m.elemtobndy, oracle_phys(dg.WORKLOAD_PHYS), NT)
    dm = dg.DeviceMesh.upload(m)
    s = dg.LSRK.for_state(dm, Q, 32)
    s.run(500, 0.002)
    out = s.state()
    errs = [np.linalg.norm(out[:, q] - ref[:, q]) / np.linalg.norm(ref[:, q]) for q in range(4)]
    print("fp32 rel L2 per field (U, V, rho, E):", errs)
    assert max(errs) < 1e-5
    sums = s.sums()
    mj = m.vgeo[:, 4, :]
    assert np.allclose(sums[0], [(mj * out[:, q]).sum() for q in range(4)], rtol=1e-6)
    s.close()


def test_fp32_precision_form_3d_fourier():
    N = 7
    m = make_mesh(3, N, n=4, L=2 * math.pi)
    x, y, z = m.coords()
    U, V, W, rho, E = ic.fourier_state(x, y, z, seed=0)
    Q = np.zeros((m.Np, 5, m.nelem), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3], Q[:, 4] = U, V, W, rho, E
    dt = ic.fourier_dt(Q, N, h=2 * math.pi / 4)
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(3, N, m.vgeo, m.sgeo, ref, rref, m.D, dt, 40, m.vmapM, m.vmapP,
                   m.elemtobndy, oracle_phys(dg.WORKLOAD_PHYS), NT)
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, 32)
    s.run(40, dt)
    out = s.state()
    errs = [np.linalg.norm(out[:, q] - ref[:, q]) / np.linalg.norm(ref[:, q]) for q in range(5)]
    print("fp32 3-D rel L2 per field:", errs)
    assert max(errs) < 1e-5
    s.close()


@pytest.mark.parametrize("dim,N", [(2, 3), (2, 5), (3, 3), (3, 5)])
@pytest.mark.parametrize("walls", [False, True])
def test_viscous_passes_parity(dim, N, walls):
    import torch
    m = make_mesh(dim, N, n=2, periodic=not walls)
    ph = dict(dg.WORKLOAD_PHYS, visc=1e-3)
    op = oracle_phys(ph)
    Q = random_state(m, 7)
    sh = (m.Np, dg.nstate(dim), dim, m.nelem)
    dm = dg.DeviceMesh.upload(m)
    dQ = dev(Q)
    # gradient pass
    r = np.zeros(sh, order="F")
    O.volume_grad(dim, N, r, Q, m.vgeo, m.D, op, NT)
    O.flux_grad(dim, N, r, Q, m.sgeo, m.vgeo, m.vmapM, m.vmapP, m.elemtobndy, op, NT)
    g = np.zeros(sh, order="F")
    O.update_gradQ(dim, N, g, r, m.vgeo, NT)
    dr = torch.zeros(int(np.prod(sh)), dtype=torch.float64, device="cuda")
    dg.volume_grad(dim, N, dr, dQ, dm.vgeo, dm.D, m.nelem, dg.make_phys(**ph))
    dg.flux_grad(dim, N, dr, dQ, dm.sgeo, dm.vgeo, m.nelem, dm.vmapM, dm.vmapP, dm.elemtobndy,
                 dg.make_phys(**ph))
    dgq = torch.zeros_like(dr)
    dg.update_gradQ(dim, N, dgq, dr, dm.vgeo, m.nelem)
    gout = dg.from_device(dgq, sh)
    assert relerr(gout.reshape(m.Np, -1, m.nelem, order="F"), g.reshape(m.Np, -1, m.nelem, order="F")) < 1e-12
    # divergence pass on the oracle's gradient
    rd = np.zeros(sh, order="F")
    O.volume_div(dim, N, rd, g, Q, m.vgeo, m.D, op, NT)
    O.flux_div(dim, N, rd, g, Q, m.sgeo, m.vmapM, m.vmapP, m.elemtobndy, op, NT)
    ddiv = torch.zeros_like(dr)
    dgg = dev(g)
    dg.volume_div(dim, N, ddiv, dgg, dQ, dm.vgeo, dm.D, m.nelem, dg.make_phys(**ph))
    dg.flux_div(dim, N, ddiv, dgg, dQ, dm.sgeo, m.nelem, dm.vmapM, dm.vmapP, dm.elemtobndy,
                dg.make_phys(**ph))
    dg.device_status()
    dout = dg.from_device(ddiv, sh)
    assert relerr(dout[:, :, 0, :], rd[:, :, 0, :]) < 1e-12
    assert np.all(dout[:, :, 1:, :] == 0)


def test_viscous_solver_vortex():
    m, Q = vortex_setup()
    ph = dict(dg.WORKLOAD_PHYS, visc=1e-3)
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(2, 4, m.vgeo, m.sgeo, ref, rref, m.D, 0.002, 50, m.vmapM, m.vmapP,
                   m.elemtobndy, oracle_phys(ph), NT)
    dm = dg.DeviceMesh.upload(m)
    dQ, drhs = dev(Q), dev(np.zeros_like(Q))
    s = dg.LSRK(dm, dQ, drhs, 64, dg.make_phys(**ph))
    s.run(50, 0.002)
    assert relerr(dg.from_device(dQ, Q.shape), ref) < 1e-12
    s.close()


@pytest.mark.parametrize("N,walls", [(3, True), (5, False), (8, True)])
def test_viscous_solver_3d(N, walls):
    """cb_lsrk_run with visc > 0: orders 3 and 5 run the two fused passes per
    stage, order 8 (groups of more than two nodes per thread) the unfused
    reference sequence; both against the oracle, and the fused form with
    state offsets (Q stored as Q - qref) to the same tolerance."""
    m = make_mesh(3, N, n=2, periodic=not walls)
    ph = dict(dg.WORKLOAD_PHYS, visc=0.02)
    Q = random_state(m, 11)
    dt, k = 2e-4, 3
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(3, N, m.vgeo, m.sgeo, ref, rref, m.D, dt, k, m.vmapM, m.vmapP, m.elemtobndy,
                   oracle_phys(ph), NT)
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, 64, phys=dg.make_phys(**ph))
    s.run(k, dt)
    assert relerr(s.state(), ref) < 1e-12
    s.close()
    if N < 8:
        off = Q.mean(axis=(0, 2))
        s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, 64, phys=dg.make_phys(**ph), offset=off)
        s.run(k, dt)
        assert relerr(s.state(), ref) < 1e-12
        s.close()


@pytest.mark.parametrize("dim,N,walls", [(3, 3, True), (3, 4, False), (3, 5, True), (3, 7, False), (2, 4, True),
                                         (2, 7, False)])
def test_pipelined_viscous_passes(dim, N, walls):
    """The fused viscous form with the pipelined passes (k_ns_grad_pipe and
    k_ns_stage_pipe: bulk-copied state (and gradient) slabs, the default) and
    with the grouped ones (kernel 3): both against the oracle at 1e-12
    relative L2 per field, and each other to round-off (1e-13); 3-D even
    orders take the ragged 16-byte-rounded slab copies."""
    m = make_mesh(dim, N, n=3 if dim == 3 else 5, periodic=not walls)
    ph = dict(dg.WORKLOAD_PHYS, visc=0.02)
    Q = random_state(m, 21 + N)
    dt, k = 2e-4, 3
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(dim, N, m.vgeo, m.sgeo, ref, rref, m.D, dt, k, m.vmapM, m.vmapP, m.elemtobndy,
                   oracle_phys(ph), NT)
    dm = dg.DeviceMesh.upload(m)
    out = {}
    for kernel in (0, 3):
        s = dg.LSRK.for_state(dm, Q, 64, phys=dg.make_phys(**ph))
        s.set_kernel(kernel)
        s.run(k, dt)
        out[kernel] = s.state()
        s.close()
        assert relerr(out[kernel], ref) < 1e-12, kernel
    assert relerr(out[0], out[3]) < 1e-13


def test_invalid_boundary_code_is_reported():
    import torch
    from canary_b200._lib import CanaryError, CB_ERR_BC
    m = make_mesh(3, 3, n=2, periodic=False)
    bnd = m.elemtobndy.copy(order="F")
    bnd[bnd == 1] = 7
    dm = dg.DeviceMesh.upload(m)
    dbnd = dev(bnd, torch.int64)
    Q = random_state(m, 8)
    dQ, drhs = dev(Q), dev(np.zeros_like(Q))
    dg.fluxrhs(3, 3, drhs, dQ, dm.sgeo, dm.vgeo, m.nelem, dm.vmapM, dm.vmapP, dbnd)
    with pytest.raises(CanaryError) as ei:
        dg.device_status()
    assert ei.value.code == CB_ERR_BC
    dg.device_status()  # cleared
    dm.elemtobndy = dbnd
    with pytest.raises(CanaryError) as ei:
        dg.LSRK(dm, dQ, drhs, 64)
    assert ei.value.code == CB_ERR_BC


def test_nonconforming_vmap_is_rejected():
    import torch
    from canary_b200._lib import CanaryError, CB_ERR_MESH
    m = make_mesh(2, 3, n=3)
    vp = m.vmapP.copy(order="F")
    vp[0, 0, 0], vp[1, 0, 0] = vp[1, 0, 0], vp[0, 0, 0]  # flipped orientation
    dm = dg.DeviceMesh.upload(m)
    dm.vmapP = dev(vp, torch.int64)
    Q = random_state(m, 9)
    with pytest.raises(CanaryError) as ei:
        dg.LSRK(dm, dev(Q), dev(np.zeros_like(Q)), 64)
    assert ei.value.code == CB_ERR_MESH


def test_zero_elements_is_a_noop():
    import torch
    t = torch.zeros(64, dtype=torch.float64, device="cuda")
    dg.volumerhs(3, 3, t, t, t, t, 0)
    dg.updatesolution(3, 3, t, None, t, t, 0, 0.1, 0.2, 0.3)
    assert torch.all(t == 0)
