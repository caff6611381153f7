"""3-D even orders in the pipelined stage: Np is odd, so an element's state,
metric and face-geometry slabs are not multiples of 16 bytes and the bulk
copies start and end on the 16-byte boundaries around them (the group that
ends an array loads its last bytes with plain loads).  Element counts are
chosen odd and even so that the last group is partial or full.

Tolerances: FP64 against the FP64 oracle 1e-12 relative L2 per field, FP32
1e-5; the pipelined batch variant against the grouped one 1e-13.
"""
import math

import numpy as np
import pytest

from conftest import cuda_available
from dg_cases import oracle_run, relerr_fields
from canary_b200 import batch as B
from canary_b200 import dg, ic
from canary_b200.metric import warp_sinusoidal

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def cube(N, n, warp=True, walls=False, seed=0):
    per = (True, True, not walls)
    m = dg.build_mesh(3, N, (np.linspace(0, 2 * math.pi, n + 1),) * 3, per,
                      meshwarp=(lambda X: warp_sinusoidal(X, 0.05)) if warp else None)
    x, y, z = m.coords()
    Q = np.zeros((m.Np, 5, m.nelem), order="F")
    for c, v in enumerate(ic.fourier_state(x, y, z, seed=seed)):
        Q[:, c] = v
    return m, Q, 0.5 * ic.fourier_dt(Q, N, h=2 * math.pi / n)


CASES = [(2, 3, True, False), (4, 3, True, True), (4, 2, True, False), (6, 2, True, True), (4, 3, False, False)]


@pytest.mark.parametrize("N,n,warp,walls", CASES)
def test_single_mesh_fused_stage(N, n, warp, walls):
    """The shape's default stage and the pipelined (1), grouped (3) and lean
    (4) stages, each against the oracle (FP64 1e-12, FP32 1e-5); the lean
    stage equals the pipelined one bit for bit."""
    from canary_b200 import CanaryError
    m, Q, dt = cube(N, n, warp, walls, seed=N)
    k = 3
    ref = oracle_run(m, Q, dt, k)
    dm = dg.DeviceMesh.upload(m)
    for prec, tol in ((64, 1e-12), (32, 1e-5)):
        out = {}
        for kernel in (0, 1, 3, 4):
            s = dg.LSRK.for_state(dm, Q, prec)
            try:
                s.set_kernel(kernel)
            except CanaryError:
                s.close()
                continue
            s.run(k, dt)
            out[kernel] = s.state()
            s.close()
            assert max(relerr_fields(out[kernel], ref)) < tol, (prec, kernel)
        if 1 in out and 4 in out:
            assert np.array_equal(out[1], out[4])


def _batch(cases, precision, variant=None, affine=True):
    b = B.Batch(precision, 16)
    b.set_affine(affine)
    if variant is not None:
        for N in {m.N for m, _, _, _ in cases}:
            b.set_variant(3, N, variant)
    meshes, slots, used = [], [], []
    for m, Q, dt, k in cases:
        bm = B.BatchMesh(dg.DeviceMesh.upload(m), precision)
        meshes.append(bm)
        s = b.add_state(bm, Q, dt, k)
        slots.append(s)
        used.append(b.slot_variant(s))
    b.run(1)
    b.run(10)
    assert not b.status().any()
    out = [b.result(s) for s in slots]
    b.close()
    return out, used


@pytest.fixture(scope="module")
def batch_cases():
    out = []
    for i, (N, n, warp, walls) in enumerate(CASES):
        m, Q, dt = cube(N, n, warp, walls, seed=10 + i)
        out.append((m, Q, dt, 2 + i % 3))
    return out


@pytest.fixture(scope="module")
def batch_refs(batch_cases):
    return [oracle_run(m, Q, dt, k) for (m, Q, dt, k) in batch_cases]


def test_batch_pipelined_variant(batch_cases, batch_refs):
    out, used = _batch(batch_cases, 64, variant=0, affine=False)
    assert all(v == 0 for v in used)
    grouped, _ = _batch(batch_cases, 64, variant=1, affine=False)
    for (m, Q, dt, k), a, g, ref in zip(batch_cases, out, grouped, batch_refs):
        assert max(relerr_fields(a, ref)) < 1e-12, (m.N, m.nelem)
        assert max(relerr_fields(a, g)) < 1e-13


def test_batch_affine_even_orders(batch_cases, batch_refs):
    """The unwarped cube runs the affine stage (copies two groups ahead)."""
    for prec, tol in ((64, 1e-12), (32, 1e-5)):
        out, used = _batch(batch_cases, prec)  # the default variant: affine where it applies
        for (m, Q, dt, k), a, v, ref in zip(batch_cases, out, used, batch_refs):
            assert max(relerr_fields(a, ref)) < tol, (prec, m.N, m.nelem)
        # the warped cubes run their shape's default per-node variant, the
        # unwarped one the affine stage
        assert used[-1] == B.VAR_AFFINE and all(v not in B.AFFINE for v in used[:-1])


def test_misaligned_state_is_rejected():
    import torch
    from canary_b200 import CanaryError
    m, Q, dt = cube(4, 2)
    bm = B.BatchMesh(dg.DeviceMesh.upload(m), 64)
    b = B.Batch(64, 2)
    buf = torch.zeros(Q.size + 1, dtype=torch.float64, device="cuda")
    with pytest.raises(CanaryError):
        b.add(bm, buf[1:], torch.zeros(Q.size, dtype=torch.float64, device="cuda"), dt, 1)
    b.close()
    bm.close()
