"""Affine-element stage of the batch (cb_mesh_affine, cb_batch_set_affine):
uniform brick meshes are detected as affine and warped ones are not; the
affine stage (one geometry record per element, MJ / MJI / sMJ formed from the
LGL weights as computegeometry does, euler3d_set3c.jl:222-246) matches the
FP64 oracle to 1e-12 relative L2 per field and the per-node-geometry stage to
1e-13 (FP64) / 1e-5 (FP32, against the oracle).  With gravity on the batch
keeps the per-node geometry (the buoyancy term needs the coordinates).
"""
import math

import numpy as np
import pytest

from conftest import cuda_available
from dg_cases import fourier_case, oracle_run, relerr_fields, vortex_case
from canary_b200 import batch as B
from canary_b200 import dg, ic

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def brick_3d(N, n, seed=0):
    """3-D Fourier state on the unwarped periodic cube [0,2π]^3."""
    m = dg.build_mesh(3, N, (np.linspace(0, 2 * math.pi, n + 1),) * 3, (True,) * 3)
    x, y, z = m.coords()
    Q = np.zeros((m.Np, 5, m.nelem), order="F")
    for c, v in enumerate(ic.fourier_state(x, y, z, seed=seed)):
        Q[:, c] = v
    return m, Q, ic.fourier_dt(Q, N, h=2 * math.pi / n)


def walled_vortex(N, n):
    """2-D vortex on [0,10]^2 with walls at y = 0 and y = 10 (unwarped)."""
    m = dg.build_mesh(2, N, (np.linspace(0, 10, n + 1),) * 2, (True, False))
    x, y = m.coords()
    Q = np.zeros((m.Np, 4, m.nelem), order="F")
    for c, v in enumerate(ic.isentropic_vortex(x, y, 3.0, 5.0, 5.0)):
        Q[:, c] = v
    return m, Q


def _cases():
    out = []
    for N, n, beta, steps in [(3, 4, 5.0, 6), (8, 2, 3.0, 4), (5, 3, 2.0, 5), (1, 6, 4.0, 5)]:
        m, Q = vortex_case(N, n, beta)
        out.append((m, Q, 0.002, steps))
    m, Q = walled_vortex(4, 4)
    out.append((m, Q, 0.002, 5))
    for N, n, steps in [(3, 4, 4), (5, 2, 3), (7, 2, 3)]:
        m, Q, dt = brick_3d(N, n)
        out.append((m, Q, dt, steps))
    return out


@pytest.fixture(scope="module")
def cases():
    return _cases()


@pytest.fixture(scope="module")
def oracle_results(cases):
    return [oracle_run(m, Q, dt, k) for (m, Q, dt, k) in cases]


def _run(cases, precision, affine=True, phys=None):
    b = B.Batch(precision, max_instances=16, phys=phys)
    b.set_affine(affine)
    meshes, slots, used = [], [], []
    for m, Q, dt, k in cases:
        bm = B.BatchMesh(dg.DeviceMesh.upload(m), precision)
        meshes.append(bm)
        s = b.add_state(bm, Q, dt, k)
        slots.append(s)
        used.append(b.slot_variant(s))
    b.run(2)
    b.run(100)
    assert not b.status().any()
    out = [b.result(s) for s in slots]
    b.close()
    return out, used


def test_affine_detection(cases):
    for m, Q, dt, k in cases:
        assert B.BatchMesh(dg.DeviceMesh.upload(m), 64).affine
    m, Q, dt = fourier_case(3, 2)  # warped
    assert not B.BatchMesh(dg.DeviceMesh.upload(m), 64).affine


def test_affine_stage_matches_oracle(cases, oracle_results):
    out, used = _run(cases, 64)
    assert all(v == B.VAR_AFFINE for v in used)
    for (m, Q, dt, k), got, ref in zip(cases, out, oracle_results):
        assert max(relerr_fields(got, ref)) < 1e-12, (m.dim, m.N)


def test_affine_stage_matches_per_node_geometry(cases):
    on, used_on = _run(cases, 64, True)
    off, used_off = _run(cases, 64, False)
    assert all(v != B.VAR_AFFINE for v in used_off)
    for a, b in zip(on, off):
        assert max(relerr_fields(a, b)) < 1e-13


def test_affine_stage_fp32_matches_oracle(cases, oracle_results):
    out, used = _run(cases, 32)
    assert all(v == B.VAR_AFFINE for v in used)
    for (m, Q, dt, k), got, ref in zip(cases, out, oracle_results):
        assert max(relerr_fields(got, ref)) < 1e-5, (m.dim, m.N)


def test_gravity_keeps_per_node_geometry():
    m, Q = walled_vortex(4, 4)
    # a hydrostatic-like energy so that the pressure stays positive under g = 10
    Q[:, 3] += 10.0 * Q[:, 2] * m.coords()[1]
    phys = dict(dg.WORKLOAD_PHYS, gravity=10.0)
    ref = oracle_run(m, Q, 0.001, 4, phys=phys)
    out, used = _run([(m, Q, 0.001, 4)], 64, True, dg.make_phys(**phys))
    assert used[0] != B.VAR_AFFINE
    assert max(relerr_fields(out[0], ref)) < 1e-12
