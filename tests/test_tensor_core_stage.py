"""The tensor-core (DMMA) stage of 3-D N=7 (FP64, and the FP32 form) against
the oracle and the CUDA-core stage.

k_stage_mma runs the D contraction as 8x8x4 FP64 tensor-core tiles with a
different summation order inside each direction; its LSRK results must still
match the oracle's left-to-right restatement at 1e-12 relative L2 per field
(full runs) and the CUDA-core stage's to round-off.  Meshes of 3^3 to 8^3
warped hexahedra put 1 to 4 element groups on each persistent block.
"""
import math
import os

import numpy as np
import pytest

from conftest import cuda_available
from oracle import pyoracle as O
from canary_b200 import dg, ic
from canary_b200._lib import CB_ERR_UNSUPPORTED, CanaryError

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

NT = os.cpu_count() or 1


def _phys(**kw):
    d = dict(dg.WORKLOAD_PHYS)
    d.update(kw)
    d["lambda"] = d.pop("lam")
    return O.make_phys(**d)


def _case(n, seed=0, walls=False):
    from canary_b200.metric import warp_sinusoidal
    L = 2 * math.pi
    per = (True, True, not walls)
    m = dg.build_mesh(3, 7, (np.linspace(0.0, L, n + 1),) * 3, per,
                      meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    Q = np.asfortranarray(np.stack(ic.fourier_state(*m.coords(), seed=seed), axis=1))
    return m, Q, ic.fourier_dt(Q, 7, h=L / n)


def _relerr(a, b):
    return max(np.linalg.norm(a[:, q] - b[:, q]) / np.linalg.norm(b[:, q]) for q in range(b.shape[1]))


@pytest.mark.parametrize("n,nsteps,walls", [(3, 2, False), (4, 7, False), (8, 4, False), (4, 3, True)])
def test_tensor_core_stage_matches_the_oracle(n, nsteps, walls):
    m, Q, dt = _case(n, seed=n, walls=walls)
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(3, 7, m.vgeo, m.sgeo, ref, rref, m.D, dt, nsteps, m.vmapM, m.vmapP, m.elemtobndy,
                   _phys(), NT)
    dm = dg.DeviceMesh.upload(m)
    out = {}
    for kernel in (1, 2):
        s = dg.LSRK.for_state(dm, Q, 64)
        s.set_kernel(kernel)
        assert s.kernel == kernel
        s.run(nsteps, dt)
        out[kernel] = s.state()
        s.close()
    assert _relerr(out[2], ref) < 1e-12
    assert _relerr(out[1], ref) < 1e-12
    assert _relerr(out[2], out[1]) < 1e-13


def test_tensor_core_stage_with_reference_physics_and_gravity():
    """The reference's gas constants, gravity 10 and walls in z (the rising
    bubble set-up of euler3d_set3c.jl:113-118) through the tensor-core stage."""
    from canary_b200.metric import warp_sinusoidal
    m = dg.build_mesh(3, 7, (np.linspace(0.0, 1000.0, 4),) * 3, (True, True, False),
                      meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    rng = np.random.default_rng(3)
    Q = np.zeros((m.Np, 5, m.nelem), order="F")
    Q[:, 3] = 1.0 + 0.01 * rng.random((m.Np, m.nelem))
    Q[:, 0:3] = 0.5 * rng.standard_normal((m.Np, 3, m.nelem))
    Q[:, 4] = 2.5e5 + 100.0 * rng.random((m.Np, m.nelem))
    rp = dict(dg.REFERENCE_PHYS)
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    orp = dict(rp)
    orp["lambda"] = orp.pop("lam")
    O.lowstorageRK(3, 7, m.vgeo, m.sgeo, ref, rref, m.D, 1e-3, 3, m.vmapM, m.vmapP, m.elemtobndy,
                   O.make_phys(**orp), NT)
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, 64, phys=dg.make_phys(**rp))
    s.set_kernel(2)
    s.run(3, 1e-3)
    assert _relerr(s.state(), ref) < 1e-12
    s.close()


@pytest.mark.parametrize("n,nsteps,walls", [(3, 3, False), (4, 5, True)])
def test_fp32_tensor_core_stage(n, nsteps, walls):
    """The FP32 form through the tensor-core stage: fluxes and update in FP32,
    the D contraction of the FP32 fluxes on the FP64 tensor pipe.  Bar: 1e-5
    relative L2 per field against the FP64 oracle (the FP32 form's bar), and
    the CUDA-core FP32 stage to within FP32 round-off (1e-6)."""
    m, Q, dt = _case(n, seed=10 + n, walls=walls)
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(3, 7, m.vgeo, m.sgeo, ref, rref, m.D, dt, nsteps, m.vmapM, m.vmapP, m.elemtobndy,
                   _phys(), NT)
    dm = dg.DeviceMesh.upload(m)
    out = {}
    for kernel in (1, 2):
        s = dg.LSRK.for_state(dm, Q, 32)
        s.set_kernel(kernel)
        assert s.kernel == kernel
        s.run(nsteps, dt)
        out[kernel] = s.state()
        s.close()
    assert _relerr(out[2], ref) < 1e-5
    assert _relerr(out[1], ref) < 1e-5
    assert _relerr(out[2], out[1]) < 1e-6


@pytest.mark.parametrize("precision,tol", [(64, 1e-12), (32, 1e-5)])
def test_every_kernel_choice_matches_the_oracle(precision, tol):
    """Kernel choices 0 (default: tensor-core stage), 1 (pipelined CUDA-core
    stage), 2 (tensor-core), 3 (unpipelined grouped stage) and 4 (lean
    pipelined stage: only the state staged) on one warped 3-D N=7 mesh: each
    against the oracle at the form's bar (FP64 1e-12, FP32 1e-5), the FP64
    ones with each other to round-off (1e-13), and the lean stage bit for
    bit with the pipelined CUDA-core one (the same arithmetic)."""
    m, Q, dt = _case(3, seed=5, walls=True)
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(3, 7, m.vgeo, m.sgeo, ref, rref, m.D, dt, 3, m.vmapM, m.vmapP, m.elemtobndy, _phys(), NT)
    dm = dg.DeviceMesh.upload(m)
    out = {}
    for kernel in (0, 1, 2, 3, 4):
        s = dg.LSRK.for_state(dm, Q, precision)
        s.set_kernel(kernel)
        assert s.kernel == (2 if kernel == 0 else kernel)
        s.run(3, dt)
        out[kernel] = s.state()
        s.close()
        assert _relerr(out[kernel], ref) < tol, kernel
    if precision == 64:
        for kernel in (1, 2, 3, 4):
            assert _relerr(out[kernel], out[0]) < 1e-13
    assert np.array_equal(out[4], out[1])


def test_kernel_choice_is_checked():
    m, Q, dt = _case(2)
    dm = dg.DeviceMesh.upload(m)
    s32 = dg.LSRK.for_state(dm, Q, 32)
    assert s32.kernel == 2
    s32.set_kernel(2)
    assert s32.kernel == 2
    s32.close()
    mv = dg.build_mesh(3, 4, (np.linspace(0.0, 1.0, 3),) * 3, (True,) * 3)
    Qv = np.zeros((mv.Np, 5, mv.nelem), order="F")
    Qv[:, 3] = 1.0
    Qv[:, 4] = 2.5
    s4 = dg.LSRK.for_state(dg.DeviceMesh.upload(mv), Qv, 64)
    assert s4.kernel == 4  # 3-D N=4 FP64 defaults to the lean pipelined stage
    with pytest.raises(CanaryError) as ei:
        s4.set_kernel(2)
    assert ei.value.code == CB_ERR_UNSUPPORTED
    s4.close()
