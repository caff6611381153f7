"""The fused paths (single-mesh pipelined solver and the batch) with the
reference drivers' physics: the reference's gas constants and gravity
(P = (R/c_v)(E - |U|^2/2ρ - ρ g z), euler3d_set3c.jl:113-118, buoyancy source
euler3d_set3c.jl:323) and reflective walls on the non-periodic direction
(elemtobndy = 1, euler3d_set3c.jl:382-389), against the oracle.

Tolerance: 1e-12 relative L2 per state field after a few LSRK steps (FP64).
"""
import numpy as np
import pytest

from conftest import cuda_available
from dg_cases import oracle_run, relerr_fields
from canary_b200 import batch as B
from canary_b200 import dg
from canary_b200.metric import warp_sinusoidal

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def walled_case(dim, N, n, seed=0):
    """Box [0,1]^dim, periodic except the last (vertical) direction, which has
    walls; warped; a perturbed hydrostatic-like state under the reference's
    constants (ρ ~ 1, E large enough that the pressure stays positive)."""
    x = (np.linspace(0.0, 1.0, n + 1),) * dim
    per = (True,) * (dim - 1) + (False,)
    m = dg.build_mesh(dim, N, x, per, meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    rng = np.random.default_rng(seed)
    ns = dg.nstate(dim)
    z = m.coords()[dim - 1]
    rho = 1.0 + 0.1 * rng.random((m.Np, m.nelem))
    vel = [0.5 * (rng.random((m.Np, m.nelem)) - 0.5) for _ in range(dim)]
    Q = np.zeros((m.Np, ns, m.nelem), order="F")
    for c in range(dim):
        Q[:, c] = rho * vel[c]
    Q[:, dim] = rho
    # E = P c_v / R + |U|^2 / 2ρ + ρ g z with P ~ 1e5 (an air-like state)
    Q[:, dim + 1] = 1e5 * 717.5 / 287.17 + 0.5 * rho * sum(v * v for v in vel) + rho * 10.0 * z
    assert np.any(m.elemtobndy == 1)
    return m, Q


@pytest.mark.parametrize("dim,N,n", [(3, 3, 3), (3, 5, 2), (3, 7, 2), (2, 4, 4), (2, 7, 3)])
def test_fused_solver_reference_physics_with_walls(dim, N, n):
    m, Q = walled_case(dim, N, n)
    dt, k = 2e-6, 6
    ref = oracle_run(m, Q, dt, k, phys=dg.REFERENCE_PHYS)
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, 64, phys=dg.make_phys(**dg.REFERENCE_PHYS))
    s.run(k, dt)
    assert max(relerr_fields(s.state(), ref)) < 1e-12
    s.close()


def test_batch_reference_physics_with_walls():
    cases = [walled_case(3, 3, 3, 1), walled_case(2, 5, 4, 2), walled_case(3, 5, 2, 3)]
    refs = [oracle_run(m, Q, 2e-6, 5 + i, phys=dg.REFERENCE_PHYS) for i, (m, Q) in enumerate(cases)]
    b = B.Batch(64, 8, phys=dg.make_phys(**dg.REFERENCE_PHYS))
    meshes, slots = [], []
    for i, (m, Q) in enumerate(cases):
        bm = B.BatchMesh(dg.DeviceMesh.upload(m), 64)
        meshes.append(bm)
        slots.append(b.add_state(bm, Q, 2e-6, 5 + i))
    b.run(10)
    assert not b.status().any()
    for s, ref in zip(slots, refs):
        assert max(relerr_fields(b.result(s), ref)) < 1e-12
    b.close()
