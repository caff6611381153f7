"""Device-side grid and geometry (cb_computegeometry) against the host
restatement of creategrid / computemetric / computegeometry (which the
reference's own metric tests pin), and an LSRK run on a device-built mesh
against the oracle on the host-built one.

Tolerance (max abs difference per field over the field's max abs value): the
two evaluations share the operation order and differ only in the last bits of
sin and hypot.  Unwarped meshes: 1e-14 for every field.  Warped meshes: the
coordinates agree to 4e-16 (sin), and the metric terms, which subtract
products of coordinates and their derivatives, to 1e-12.  The LSRK run on a
warped device-built mesh: 1e-12 relative L2 per field against the oracle.
"""
import math

import numpy as np
import pytest

from conftest import cuda_available
from dg_cases import oracle_run, relerr_fields
from canary_b200 import dg, ic
from canary_b200.metric import warp_sinusoidal

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def _field_err(a, b, scale=None):
    scale = np.max(np.abs(b)) if scale is None else scale
    return float(np.max(np.abs(a - b)) / (scale if scale > 0 else 1.0))


@pytest.mark.parametrize("dim,N,n,amp", [(2, 1, 3, 0.0), (2, 4, 5, 0.0), (2, 8, 3, 0.05), (3, 1, 2, 0.05),
                                         (3, 3, 3, 0.05), (3, 7, 2, 0.05), (3, 4, 3, 0.0), (3, 10, 2, 0.05)])
def test_device_geometry_matches_host(dim, N, n, amp):
    L = 2 * math.pi if dim == 3 else 10.0
    x = (np.linspace(0.0, L, n + 1),) * dim
    host = dg.build_mesh(dim, N, x, (True,) * dim,
                         meshwarp=(lambda X: warp_sinusoidal(X, amp)) if amp else None)
    dm = dg.DeviceMesh.build(dim, N, x, (True,) * dim, warp_amp=amp)
    vg = dg.from_device(dm.vgeo, host.vgeo.shape)
    sg = dg.from_device(dm.sgeo, host.sgeo.shape)
    ncoord = dim * dim + 2
    # metric terms are compared on the scale of the largest one (off-diagonal
    # terms of a symmetric warp are round-off sized)
    mscale = np.max(np.abs(host.vgeo[:, :dim * dim]))
    for f in range(host.vgeo.shape[1]):
        tol = 1e-14 if amp == 0.0 else (4e-16 if f >= ncoord else 1e-12)
        sc = mscale if f < dim * dim else None
        assert _field_err(vg[:, f], host.vgeo[:, f], sc) < tol, ("vgeo", f)
    for f in range(host.sgeo.shape[0]):
        assert _field_err(sg[f], host.sgeo[f]) < (1e-14 if amp == 0.0 else 1e-12), ("sgeo", f)
    assert np.array_equal(dg.from_device(dm.vmapM, host.vmapM.shape), host.vmapM)
    assert np.array_equal(dg.from_device(dm.vmapP, host.vmapP.shape), host.vmapP)


def test_lsrk_on_device_built_mesh_matches_oracle():
    N, n = 5, 3
    x = (np.linspace(0.0, 2 * math.pi, n + 1),) * 3
    host = dg.build_mesh(3, N, x, (True,) * 3, meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    X, Y, Z = host.coords()
    Q = np.stack(ic.fourier_state(X, Y, Z, seed=3), axis=1)
    Q = np.asfortranarray(Q)
    dt = ic.fourier_dt(Q, N, h=2 * math.pi / n)
    ref = oracle_run(host, Q, dt, 6)
    dm = dg.DeviceMesh.build(3, N, x, (True,) * 3, warp_amp=0.05)
    s = dg.LSRK.for_state(dm, Q, 64)
    s.run(6, dt)
    assert max(relerr_fields(s.state(), ref)) < 1e-12
    s.close()


def test_device_initial_states_match_host():
    import torch
    m = dg.build_mesh(2, 5, (np.linspace(0, 10, 5),) * 2, (True, True))
    dm = dg.DeviceMesh.upload(m)
    x, y = dm.coords()
    dev = torch.stack(ic.isentropic_vortex_t(x, y, 3.0, 4.0, 6.0), 1)
    host = np.stack(ic.isentropic_vortex(*m.coords(), 3.0, 4.0, 6.0), 1)
    got = dev.cpu().numpy().transpose(2, 1, 0)  # (nelem, 4, Np) -> (Np, 4, nelem)
    assert np.allclose(got, host, rtol=1e-14, atol=1e-14)
    m3 = dg.build_mesh(3, 3, (np.linspace(0, 2 * math.pi, 3),) * 3, (True,) * 3)
    d3 = dg.DeviceMesh.upload(m3)
    dev3 = torch.stack(ic.fourier_state_t(*d3.coords(), seed=5), 1).cpu().numpy().transpose(2, 1, 0)
    host3 = np.stack(ic.fourier_state(*m3.coords(), seed=5), 1)
    assert np.allclose(dev3, host3, rtol=1e-13, atol=1e-13)
