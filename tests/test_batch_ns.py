"""Viscous batches (cb_batch_create with visc > 0): the LDG Navier–Stokes
stage of the reference's nse drivers (nse2d.jl:396-778, nse3d.jl:475-955,
the viscous branch of lowstorageRK nse2d.jl:1826-1849) fused into a gradient
pass and a stage pass per RK stage, over many instances at once.

Tolerances: FP64 batch vs the FP64 oracle 1e-12 relative L2 per field (the
viscous terms are summed with the inviscid ones rather than in a separate
residual: the same terms rounded in another order); vs the single-mesh
viscous solver (cb_lsrk_run, the six unfused passes) 1e-12; FP32 batch vs the
oracle 1e-4 (the viscous form of the precision tests); alone vs in the mix
bit-identical.
"""
import math

import numpy as np
import pytest

from conftest import cuda_available
from dg_cases import oracle_run, relerr_fields
from canary_b200 import batch as B
from canary_b200 import CanaryError, dg, ic
from canary_b200.metric import warp_sinusoidal

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

MU = 0.02  # large enough that the viscous terms move the result well above round-off


def vortex(N, n, walls=False, beta=4.0):
    per = (True, not walls)
    m = dg.build_mesh(2, N, (np.linspace(0, 10, n + 1),) * 2, per)
    x, y = m.coords()
    Q = np.zeros((m.Np, 4, m.nelem), order="F")
    for c, v in enumerate(ic.isentropic_vortex(x, y, beta, 5.0, 5.0)):
        Q[:, c] = v
    return m, Q, 0.002


def fourier(N, n, walls=False, seed=0):
    per = (True, True, not walls)
    m = dg.build_mesh(3, N, (np.linspace(0, 2 * math.pi, n + 1),) * 3, per,
                      meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    x, y, z = m.coords()
    Q = np.zeros((m.Np, 5, m.nelem), order="F")
    for c, v in enumerate(ic.fourier_state(x, y, z, seed=seed)):
        Q[:, c] = v
    if walls:  # no normal momentum through the walls z = 0, 2π at the start
        Q[:, 2] *= np.sin(z / 2.0) ** 2
        rho = Q[:, 3]
        Q[:, 4] = 1.0 / 0.4 + 0.5 * (Q[:, 0] ** 2 + Q[:, 1] ** 2 + Q[:, 2] ** 2) / rho
    return m, Q, 0.25 * ic.fourier_dt(Q, N, h=2 * math.pi / n)


def _cases():
    out = []
    for (N, n, walls) in [(3, 4, False), (5, 3, True), (8, 2, False), (1, 6, True)]:
        m, Q, dt = vortex(N, n, walls)
        out.append((m, Q, dt, 4 + N % 3))
    for (N, n, walls) in [(3, 3, False), (5, 2, True), (7, 2, False), (2, 3, True)]:
        m, Q, dt = fourier(N, n, walls, seed=N)
        out.append((m, Q, dt, 3 + N % 2))
    return out


@pytest.fixture(scope="module")
def cases():
    return _cases()


@pytest.fixture(scope="module")
def oracle_results(cases):
    ph = dict(dg.WORKLOAD_PHYS, visc=MU)
    return [oracle_run(m, Q, dt, k, phys=ph) for (m, Q, dt, k) in cases]


def _run(cases, precision, idx=None, chunks=(1, 2, 100)):
    idx = range(len(cases)) if idx is None else idx
    b = B.Batch(precision, max_instances=16, phys=dg.make_phys(visc=MU))
    meshes, slots = [], []
    for i in idx:
        m, Q, dt, k = cases[i]
        bm = B.BatchMesh(dg.DeviceMesh.upload(m), precision)
        meshes.append(bm)
        slots.append(b.add_state(bm, Q, dt, k))
    for c in chunks:
        b.run(c)
    assert not b.status().any()
    out = [b.result(s) for s in slots]
    b.close()
    return out


def test_ns_batch_fp64_matches_oracle(cases, oracle_results):
    out = _run(cases, 64)
    for (m, Q, dt, k), got, ref in zip(cases, out, oracle_results):
        assert max(relerr_fields(got, ref)) < 1e-12, (m.dim, m.N)


def test_viscous_terms_matter(cases, oracle_results):
    """The inviscid result differs from the viscous one far above the
    tolerance, so the parity above checks the viscous terms."""
    for (m, Q, dt, k), ref in list(zip(cases, oracle_results))[:2]:
        inv = oracle_run(m, Q, dt, k)
        assert max(relerr_fields(inv, ref)) > 1e-8


def test_ns_batch_fp32_matches_oracle(cases, oracle_results):
    out = _run(cases, 32)
    for (m, Q, dt, k), got, ref in zip(cases, out, oracle_results):
        assert max(relerr_fields(got, ref)) < 1e-4, (m.dim, m.N)


def test_ns_batch_matches_single_mesh_solver(cases):
    m, Q, dt, k = cases[5]  # 3-D N=5 with walls
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, 64, phys=dg.make_phys(visc=MU))
    s.run(k, dt)
    single = s.state()
    s.close()
    got = _run(cases, 64, idx=[5], chunks=(100,))[0]
    assert max(relerr_fields(got, single)) < 1e-12


def test_ns_batch_same_alone_and_in_mix(cases):
    alone = [_run(cases, 32, idx=[i], chunks=(100,))[0] for i in (1, 6)]
    mixed = _run(cases, 32, chunks=(2, 1, 100))
    for a, i in zip(alone, (1, 6)):
        assert np.array_equal(a, mixed[i])


def test_viscous_batch_runs_variant_1_only():
    b = B.Batch(64, 2, phys=dg.make_phys(visc=MU))
    assert b.variant(3, 5) == 1
    b.set_variant(3, 5, 1)
    with pytest.raises(CanaryError):
        b.set_variant(2, 4, 0)
    b.close()
