"""Bounded device waits of the pipelined stage kernel.

Every mbarrier wait of the stage gives up after a poll limit instead of
hanging; the block then stores nothing, raises the timeout status and exits
once the copies it issued have landed.  The test hook cb_solver_test_timeout
runs one stage in which each block's first state copy is never issued, so
the wait runs out on an mbarrier nobody arrives on (no fault, trap or hang is
involved).  Checked through the C-ABI: the status APIs report CB_ERR_TIMEOUT,
the state and residual carry are unchanged bit for bit, and the context stays
usable — after a status reset the same solver runs LSRK steps that match the
oracle at 1e-12.
"""
import math
import os

import numpy as np
import pytest

from conftest import cuda_available
from oracle import pyoracle as O
from canary_b200 import dg, ic
from canary_b200._lib import CB_ERR_TIMEOUT, CB_ERR_UNSUPPORTED, CanaryError

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]

NT = os.cpu_count() or 1
ST_TIMEOUT = 8


def _oracle_phys():
    d = dict(dg.WORKLOAD_PHYS)
    d["lambda"] = d.pop("lam")
    return O.make_phys(**d)


def _case(dim, N, n):
    from canary_b200.metric import warp_sinusoidal
    L = 2 * math.pi
    m = dg.build_mesh(dim, N, (np.linspace(0.0, L, n + 1),) * dim, (True,) * dim,
                      meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    X = m.coords()
    if dim == 3:
        Q = np.stack(ic.fourier_state(*X, seed=1), axis=1)
        dt = ic.fourier_dt(np.asfortranarray(Q), N, h=L / n)
    else:
        Q = np.stack(ic.isentropic_vortex(X[0] * (10 / L), X[1] * (10 / L)), axis=1)
        dt = 1e-3
    return m, np.asfortranarray(Q), dt


# 3-D N=7: the tensor-core stage; 2-D N=4 and 3-D N=4 FP32: the pipelined
# one; 3-D N=4 FP64 (its default) and N=9 FP64 (no pipelined plan fits): the
# lean one
@pytest.mark.parametrize("dim,N,n,precision", [(3, 7, 6, 64), (3, 7, 4, 32), (2, 4, 12, 64),
                                               (3, 4, 4, 64), (3, 4, 4, 32), (3, 9, 3, 64)])
def test_timed_out_wait_stores_nothing_and_reports(dim, N, n, precision):
    import torch
    m, Q, dt = _case(dim, N, n)
    dm = dg.DeviceMesh.upload(m)
    s = dg.LSRK.for_state(dm, Q, precision, offset=np.zeros(Q.shape[1]))
    # a few real steps first, so the carry is non-zero and the probe starts
    # from an ordinary state
    s.run(1, dt)
    torch.cuda.synchronize()
    q0, r0 = s.Q.clone(), s.rhs.clone()
    s.test_timeout()
    torch.cuda.synchronize()
    host = torch.zeros(1, dtype=torch.int32, pin_memory=True)
    s.status_async(host)
    torch.cuda.synchronize()
    assert int(host.item()) & ST_TIMEOUT
    with pytest.raises(CanaryError) as ei:
        s.sums()
    assert ei.value.code == CB_ERR_TIMEOUT
    assert torch.equal(s.Q, q0) and torch.equal(s.rhs, r0)  # nothing stored
    # the context and the solver stay usable
    s.reset_status()
    k = 3
    s.run(k, dt)
    out = s.state()
    s.close()
    ref = Q.copy(order="F")
    rref = np.zeros_like(Q, order="F")
    O.lowstorageRK(dim, N, m.vgeo, m.sgeo, ref, rref, m.D, dt, 1 + k, m.vmapM, m.vmapP,
                   m.elemtobndy, _oracle_phys(), NT)
    errs = [np.linalg.norm(out[:, q] - ref[:, q]) / np.linalg.norm(ref[:, q]) for q in range(Q.shape[1])]
    assert max(errs) < (1e-12 if precision == 64 else 1e-5), errs


def test_timeout_hook_refuses_the_viscous_form():
    m, Q, dt = _case(2, 3, 4)
    s = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, 64, phys=dg.make_phys(visc=1e-3))
    with pytest.raises(CanaryError) as ei:
        s.test_timeout()
    assert ei.value.code == CB_ERR_UNSUPPORTED
    s.close()
