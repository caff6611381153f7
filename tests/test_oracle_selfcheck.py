"""Self-checks of the oracle's restatement of the RHS and LSRK path.

The reference's own tests never execute volumerhs!/fluxrhs!/lowstorageRK and
no reference-produced vectors exist for them, so the oracle's physics is
pinned here by properties the reference's discretisation must have:

  * free-stream preservation: a constant state on a warped (curvilinear)
    periodic mesh has volume and face terms that cancel to round-off, because
    the curl-invariant metric (src/metric.jl:230-400) satisfies the discrete
    metric identities and the LGL derivative matrix is summation-by-parts;
  * conservation: Σ MJ·Q of every conserved field is constant to round-off on
    a periodic mesh (the weak form's volume terms sum to zero and the
    Rusanov face fluxes cancel pairwise, euler3d_set3c.jl:394-446);
  * accuracy: the 2-D isentropic vortex converges to the exact translated
    vortex under h-refinement at about the order N+1 and under N-refinement;
  * L2energysquared (euler3d_set3c.jl:1252-1264) is Σ MJ·Q² over all fields.
"""
import math
import os

import numpy as np
import pytest

from oracle import pyoracle as O
from canary_b200 import dg, ic
from canary_b200.metric import warp_sinusoidal

NT = os.cpu_count() or 1


def _phys():
    d = dict(dg.WORKLOAD_PHYS)
    d["lambda"] = d.pop("lam")
    return O.make_phys(**d)


def _warped(dim, N, n):
    return dg.build_mesh(dim, N, (np.linspace(0.0, 2 * math.pi, n + 1),) * dim, (True,) * dim,
                         meshwarp=lambda X: warp_sinusoidal(X, 0.05))


@pytest.mark.parametrize("dim,N,n", [(3, 4, 3), (3, 7, 2), (2, 5, 4), (2, 8, 3)])
def test_free_stream_is_preserved_on_warped_meshes(dim, N, n):
    m = _warped(dim, N, n)
    ns = dg.nstate(dim)
    vel = [0.3, -0.2, 0.1][:dim]
    Q = np.zeros((m.Np, ns, m.nelem), order="F")
    for c in range(dim):
        Q[:, c] = vel[c]
    Q[:, dim] = 1.0
    Q[:, dim + 1] = 1.0 / 0.4 + 0.5 * sum(v * v for v in vel)
    vol = np.zeros_like(Q, order="F")
    O.volumerhs(dim, N, vol, Q, m.vgeo, m.D, _phys(), NT)
    tot = vol.copy(order="F")
    O.fluxrhs(dim, N, tot, Q, m.sgeo, m.vgeo, m.vmapM, m.vmapP, m.elemtobndy, _phys(), NT)
    assert np.abs(vol).max() > 0.1  # the terms themselves are O(1) on the warped mesh
    assert np.abs(tot).max() <= 1e-13 * np.abs(vol).max()


def _vortex(N, n):
    m = dg.build_mesh(2, N, (np.linspace(0.0, 10.0, n + 1),) * 2, (True, True))
    x, y = m.coords()
    return m, np.asfortranarray(np.stack(ic.isentropic_vortex(x, y), axis=1))


def _run(m, Q, dt, steps):
    r = np.zeros_like(Q, order="F")
    O.lowstorageRK(m.dim, m.N, m.vgeo, m.sgeo, Q, r, m.D, dt, steps, m.vmapM, m.vmapP,
                   m.elemtobndy, _phys(), NT)


def test_conservation_on_periodic_meshes():
    # 2-D vortex
    m, Q = _vortex(4, 10)
    mj = m.vgeo[:, 4, :]
    s0 = np.array([(mj * Q[:, q]).sum() for q in range(4)])
    a0 = np.array([(mj * np.abs(Q[:, q])).sum() for q in range(4)])
    _run(m, Q, 0.002, 100)
    s1 = np.array([(mj * Q[:, q]).sum() for q in range(4)])
    assert np.all(np.abs(s1 - s0) <= 1e-13 * a0), (s1 - s0) / a0
    # 3-D warped cube, a smooth periodic state (p = 1)
    m = _warped(3, 4, 3)
    x, y, z = m.coords()
    rho = 1.0 + 0.1 * np.sin(x) * np.cos(y)
    u, v, w = 0.1 * np.sin(z), 0.1 * np.cos(x), 0.05 * np.sin(y + z)
    Q = np.asfortranarray(np.stack([rho * u, rho * v, rho * w, rho,
                                    1.0 / 0.4 + 0.5 * rho * (u * u + v * v + w * w)], axis=1))
    mj = m.vgeo[:, 9, :]
    s0 = np.array([(mj * Q[:, q]).sum() for q in range(5)])
    a0 = np.array([(mj * np.abs(Q[:, q])).sum() for q in range(5)])
    _run(m, Q, ic.fourier_dt(Q, 4, h=2 * math.pi / 3), 20)
    assert np.all(np.isfinite(Q))
    s1 = np.array([(mj * Q[:, q]).sum() for q in range(5)])
    assert np.all(np.abs(s1 - s0) <= 1e-13 * a0), (s1 - s0) / a0


def _vortex_error(N, n, T=0.5, dt=0.001):
    """Relative MJ-weighted L2 error of ρ against the exact vortex advected
    by the free stream for time T."""
    m, Q = _vortex(N, n)
    _run(m, Q, dt, int(round(T / dt)))
    x, y = m.coords()
    ex = ic.isentropic_vortex(x, y, t=T)[2]
    mj = m.vgeo[:, 4, :]
    return math.sqrt((mj * (Q[:, 2] - ex) ** 2).sum() / (mj * ex ** 2).sum())


def test_vortex_converges_under_h_refinement():
    e = [_vortex_error(3, n) for n in (8, 16, 32)]
    rates = [math.log2(e[i] / e[i + 1]) for i in range(2)]
    assert e[-1] < 5e-5, e
    assert min(rates) > 2.8, (e, rates)  # order N+1 = 4 asymptotically


def test_vortex_converges_under_N_refinement():
    e = [_vortex_error(N, 10) for N in (2, 3, 4, 5)]
    assert all(e[i + 1] < e[i] / 3 for i in range(3)), e
    assert e[-1] < 1e-4, e


def test_l2energysquared_is_the_weighted_sum_of_squares():
    m = _warped(3, 3, 2)
    Q = np.asfortranarray(np.stack(ic.fourier_state(*m.coords(), seed=5), axis=1))
    mj = m.vgeo[:, 9, :]
    expect = math.fsum(float(v) for q in range(5) for v in (mj * Q[:, q] ** 2).ravel())
    got = O.L2energysquared(3, 3, Q, m.vgeo)
    assert abs(got - expect) <= 1e-13 * expect
