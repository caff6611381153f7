"""The allocation-free stage entry point (cb_lsrk_stage_noalloc).

Callers that cannot allocate device memory (a host runtime that owns every
device allocation) use this entry point; its scratch is a static device array
instead of cudaMalloc memory.  Checked here through the C-ABI against the
stateless entry points cb_volumerhs + cb_fluxrhs + cb_updatesolution on two
consecutive calls (the second one reuses the shared scratch).  The file is
named so that pytest collects it last.
"""
import math

import numpy as np
import pytest

from conftest import cuda_available
from canary_b200 import dg, ic
from canary_b200._lib import CB_ERR_ARG, CanaryError, lib, cb_phys

RKA = [0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0]
RKB = [1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0]


def _relerr(a, b):
    out = []
    for s in range(a.shape[1]):
        den = np.linalg.norm(b[:, s])
        out.append(np.linalg.norm(a[:, s] - b[:, s]) / (den if den > 0 else 1.0))
    return max(out)


def _max_elements(dim, N):
    """Largest element count the 32 MiB static scratch accepts: a sticky status
    word padded to 256 bytes, then the int32 face-neighbour table and the FP64
    stage-input state, each padded to 256 bytes."""
    Np, ns, nface = (N + 1) ** dim, 5 if dim == 3 else 4, 2 * dim
    return (dg.NOALLOC_SCRATCH_BYTES - 256 - 2 * 256) // (8 * Np * ns + 4 * nface)


def test_noalloc_rejects_meshes_beyond_the_static_scratch():
    phys = cb_phys(1.4, 1.0, 3.5, 2.5, 0.0, 0.72, -2 / 3, 0.0)
    import ctypes as C
    d = C.c_void_p(16)  # never dereferenced: the size check comes first
    for n in (10 ** 6, 2 ** 62):  # the second would wrap a naive byte count
        rc = lib().cb_lsrk_stage_noalloc(3, 7, d, d, d, d, d, d, d, d, n, C.byref(phys),
                                         0.0, 0.1, 0.1, None, None)
        assert rc == CB_ERR_ARG
        assert "scratch" in lib().cb_last_error().decode()


@pytest.mark.skipif(cuda_available(), reason="passes fake pointers past the size check: CPU only")
@pytest.mark.parametrize("dim,N", [(3, 7), (2, 4), (3, 1)])
def test_noalloc_size_boundary(dim, N):
    """One element above the limit is rejected before any device work; the
    limit itself passes the size check (without a GPU the call then fails
    at the device lookup, never with CB_ERR_ARG)."""
    import ctypes as C
    phys = cb_phys(1.4, 1.0, 3.5, 2.5, 0.0, 0.72, -2 / 3, 0.0)
    d = C.c_void_p(16)
    n = _max_elements(dim, N)
    rc = lib().cb_lsrk_stage_noalloc(dim, N, d, d, d, d, d, d, d, d, n + 1, C.byref(phys), 0.0, 0.1, 0.1,
                                     None, None)
    assert rc == CB_ERR_ARG
    assert f"exceeds the {n} elements" in lib().cb_last_error().decode()
    rc = lib().cb_lsrk_stage_noalloc(dim, N, d, d, d, d, d, d, d, d, n, C.byref(phys), 0.0, 0.1, 0.1,
                                     None, None)
    assert rc != CB_ERR_ARG


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
@pytest.mark.parametrize("dim,N,n", [(3, 7, 4), (2, 4, 10)])
def test_noalloc_stage_matches_stateless_entry_points(dim, N, n):
    import torch
    from canary_b200.metric import warp_sinusoidal
    L = 2 * math.pi
    m = dg.build_mesh(dim, N, (np.linspace(0.0, L, n + 1),) * dim, (True,) * dim,
                      meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    X = m.coords()
    if dim == 3:
        U, V, W, rho, E = ic.fourier_state(*X, seed=3)
        Q = np.stack([U, V, W, rho, E], axis=1)
    else:
        U, V, rho, E = ic.isentropic_vortex(X[0] * (10 / L), X[1] * (10 / L))
        Q = np.stack([U, V, rho, E], axis=1)
    Q = np.asfortranarray(Q)
    dm = dg.DeviceMesh.upload(m)
    dt = 1e-3
    # reference: the stateless entry points
    qa, ra = dg.to_device(Q), torch.zeros(Q.size, dtype=torch.float64, device="cuda")
    # allocation-free stage
    qb, rb = qa.clone(), ra.clone()
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    for call in range(2):  # two calls in a row share the static scratch
        dg.volumerhs(dim, N, ra, qa, dm.vgeo, dm.D, m.nelem)
        dg.fluxrhs(dim, N, ra, qa, dm.sgeo, dm.vgeo, m.nelem, dm.vmapM, dm.vmapP, dm.elemtobndy)
        dg.updatesolution(dim, N, ra, None, qa, dm.vgeo, m.nelem, RKA[call + 1], RKB[call], dt)
        dg.lsrk_stage_noalloc(dim, N, qb, rb, dm.vgeo, dm.sgeo, dm.vmapM, dm.vmapP, dm.elemtobndy,
                              dm.D, m.nelem, RKA[call + 1], RKB[call], dt, status=status)
        torch.cuda.synchronize()
        sh = Q.shape
        qa_h, qb_h = dg.from_device(qa, sh), dg.from_device(qb, sh)
        ra_h, rb_h = dg.from_device(ra, sh), dg.from_device(rb, sh)
        # tolerances of the single-call kernel tests; the fused stage sums in a
        # different (but equally accurate) order, so the small residual carry
        # is compared with a looser bound
        assert _relerr(qb_h, qa_h) < 1e-13, call
        assert _relerr(rb_h, ra_h) < 1e-11, call
    assert int(status.item()) == 0


@pytest.mark.gpu
@pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")
def test_noalloc_reports_kernel_status_with_and_without_a_status_word():
    """A face with boundary code 7 (neither connected nor wall) is skipped and
    reported: into the caller's status word when one is given, else into the
    sticky word that cb_noalloc_status reads and clears."""
    import torch
    from canary_b200._lib import CB_ERR_BC
    m = dg.build_mesh(2, 3, (np.linspace(0.0, 10.0, 5),) * 2, (True, True))
    X = m.coords()
    U, V, rho, E = ic.isentropic_vortex(X[0], X[1])
    Q = np.asfortranarray(np.stack([U, V, rho, E], axis=1))
    dm = dg.DeviceMesh.upload(m)
    bad = dm.elemtobndy.clone()
    bad[5] = 7
    q, r = dg.to_device(Q), torch.zeros(Q.size, dtype=torch.float64, device="cuda")
    try:  # start from a clear sticky word whatever ran before in this process
        dg.noalloc_status()
    except CanaryError:
        pass
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    dg.lsrk_stage_noalloc(2, 3, q, r, dm.vgeo, dm.sgeo, dm.vmapM, dm.vmapP, bad, dm.D, m.nelem,
                          RKA[1], RKB[0], 1e-3, status=status)
    torch.cuda.synchronize()
    assert int(status.item()) & 1  # ST_BC into the caller's word
    assert dg.noalloc_status() == 0  # ... and not into the sticky one
    dg.lsrk_stage_noalloc(2, 3, q, r, dm.vgeo, dm.sgeo, dm.vmapM, dm.vmapP, bad, dm.D, m.nelem,
                          RKA[1], RKB[0], 1e-3)
    with pytest.raises(CanaryError) as ei:
        dg.noalloc_status()
    assert ei.value.code == CB_ERR_BC
    assert dg.noalloc_status() == 0  # read and cleared
