"""Compensated conservation sums and L2energysquared on the GPU.

cb_solver_sums returns, per state field, Σ MJ·Q and Σ MJ·Q² accumulated with
Neumaier's compensated summation in FP64 on the device (per-thread pairs,
merged across the warp, the block and the blocks).  Checked against
  * the oracle's L2energysquared (euler3d_set3c.jl:1252-1264: Σ over fields
    and nodes of MJ·Q²) and Σ MJ·Q after LSRK steps run by both;
  * the exactly rounded sum (math.fsum) on an ill-conditioned field, where a
    plain sequential FP64 sum — the reference's loop — loses about ten
    digits, so that the compensation is shown to matter.
Also free-stream preservation of the fused stage on a warped mesh.
"""
import math
import os

import numpy as np
import pytest

from conftest import cuda_available
from oracle import pyoracle as O
from canary_b200 import dg, ic
from canary_b200.metric import warp_sinusoidal

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

NT = os.cpu_count() or 1


def _phys():
    d = dict(dg.WORKLOAD_PHYS)
    d["lambda"] = d.pop("lam")
    return O.make_phys(**d)


def _warped(dim, N, n):
    return dg.build_mesh(dim, N, (np.linspace(0.0, 2 * math.pi, n + 1),) * dim, (True,) * dim,
                         meshwarp=lambda X: warp_sinusoidal(X, 0.05))


@pytest.mark.parametrize("precision", [64, 32])
def test_sums_match_the_oracle_l2energysquared(precision):
    N, n, k = 7, 4, 6
    m = _warped(3, N, n)
    Q = np.asfortranarray(np.stack(ic.fourier_state(*m.coords(), seed=4), axis=1))
    dt = ic.fourier_dt(Q, N, h=2 * math.pi / n)
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, precision)
    s.run(k, dt)
    sums = s.sums()
    s.close()
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(3, N, m.vgeo, m.sgeo, ref, rref, m.D, dt, k, m.vmapM, m.vmapP, m.elemtobndy,
                   _phys(), NT)
    e2 = O.L2energysquared(3, N, ref, m.vgeo)
    mj = m.vgeo[:, 9, :]
    mass = np.array([math.fsum((mj * ref[:, q]).ravel()) for q in range(5)])
    absm = np.array([math.fsum(np.abs(mj * ref[:, q]).ravel()) for q in range(5)])
    tol = 1e-12 if precision == 64 else 2e-6
    assert abs(sums[1].sum() - e2) <= tol * e2
    assert np.all(np.abs(sums[0] - mass) <= tol * absm)


def test_compensated_sum_on_an_ill_conditioned_field():
    import torch
    m = dg.build_mesh(2, 7, (np.linspace(0.0, 10.0, 65),) * 2, (True, True))
    Np, ne = m.Np, m.nelem
    rng = np.random.default_rng(0)
    # field 0 alternates ±1e10 node by node with an O(1) positive part:
    # Σ|MJ·Q| / |Σ MJ·Q| ≈ 2e10
    sign = np.where(np.arange(Np * ne).reshape(ne, Np).T % 2 == 0, 1.0, -1.0)
    Q = np.zeros((Np, 4, ne), order="F")
    Q[:, 0] = 1e10 * sign + rng.random((Np, ne))
    Q[:, 2] = 1.0
    Q[:, 3] = 2.5
    mj = m.vgeo[:, 4, :]
    x = (mj * Q[:, 0]).ravel(order="F")
    exact = math.fsum(x.tolist())
    naive = float(np.cumsum(x)[-1])  # left-to-right, as the reference's loop
    dQ = dg.to_device(Q)
    s = dg.LSRK(dg.DeviceMesh.upload(m), dQ, torch.zeros_like(dQ), 64)
    got = s.sums()[0][0]
    s.close()
    assert abs(naive - exact) > 1e-11 * abs(exact)  # the plain sum loses digits here
    assert abs(got - exact) <= 1e-14 * abs(exact), (got, exact, naive)


@pytest.mark.parametrize("dim,N,n,precision", [(3, 7, 3, 64), (3, 4, 4, 64), (2, 5, 6, 64), (3, 7, 3, 32)])
def test_fused_stage_preserves_the_free_stream(dim, N, n, precision):
    m = _warped(dim, N, n)
    ns = dg.nstate(dim)
    vel = [0.3, -0.2, 0.1][:dim]
    Q = np.zeros((m.Np, ns, m.nelem), order="F")
    for c in range(dim):
        Q[:, c] = vel[c]
    Q[:, dim] = 1.0
    Q[:, dim + 1] = 1.0 / 0.4 + 0.5 * sum(v * v for v in vel)
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, precision, offset=np.zeros(ns))
    s.run(3, 0.01)
    out = s.state()
    s.close()
    tol = 1e-13 if precision == 64 else 1e-6
    for q in range(ns):
        assert np.abs(out[:, q] - Q[:, q]).max() <= tol * max(1.0, np.abs(Q[:, q]).max())
