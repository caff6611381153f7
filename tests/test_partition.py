"""Element-partitioned solve (cb_solver_create_ghosted and the stage API):
several parts of one mesh advanced in lock step in this process, ghosts moved
by device copies — face traces (the minimal message) or whole elements —
with each inviscid stage split into its interior and boundary halves, give
the unpartitioned single-mesh result bit for bit: every element's arithmetic
is the same.  The inter-rank transport is covered on the host
(tests/test_partition_host.py, gloo)."""
import math

import numpy as np
import pytest

from conftest import cuda_available
from dg_cases import oracle_run, relerr_fields
from canary_b200 import dg, ic
from canary_b200 import partition as P
from canary_b200.metric import warp_sinusoidal

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not cuda_available(), reason="needs a CUDA GPU")]


def cube(N, n, walls=False):
    m = dg.build_mesh(3, N, (np.linspace(0, 2 * math.pi, n + 1),) * 3, (True, True, not walls),
                      meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    x, y, z = m.coords()
    Q = np.zeros((m.Np, 5, m.nelem), order="F")
    for c, v in enumerate(ic.fourier_state(x, y, z, seed=N)):
        Q[:, c] = v
    return m, Q, 0.5 * ic.fourier_dt(Q, N, h=2 * math.pi / n)


def square(N, n):
    m = dg.build_mesh(2, N, (np.linspace(0, 10, n + 1),) * 2, (True, False))
    x, y = m.coords()
    Q = np.zeros((m.Np, 4, m.nelem), order="F")
    for c, v in enumerate(ic.isentropic_vortex(x, y, 3.0, 5.0, 5.0)):
        Q[:, c] = v
    return m, Q, 0.002


@pytest.mark.parametrize("case,world,visc", [("cube3", 2, 0.0), ("cube3", 5, 0.0), ("cube4w", 3, 0.0),
                                             ("square", 4, 0.0), ("cube3", 3, 0.02), ("square", 2, 0.02),
                                             ("cube7", 2, 0.0), ("cube9", 2, 0.0)])
@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("faces", [True, False])
def test_parts_equal_single_mesh(case, world, visc, precision, faces):
    """Inviscid and LDG Navier–Stokes (state and gradient exchanged)."""
    import torch
    m, Q, dt = {"cube3": lambda: cube(3, 4), "cube4w": lambda: cube(4, 3, walls=True),
                "square": lambda: square(5, 6), "cube7": lambda: cube(7, 3),
                "cube9": lambda: cube(9, 3)}[case]()
    k = 3
    phys = dict(dg.WORKLOAD_PHYS, visc=visc)
    single = dg.LSRK.for_state(dg.DeviceMesh.upload(m), Q, precision, phys=dg.make_phys(**phys))
    single.run(k, dt)
    ref = single.state()
    single.close()
    stream = torch.cuda.Stream()
    parts = [P.GhostedLSRK(m, P.plan(m, r, world), Q, precision, dg.make_phys(**phys), stream=stream)
             for r in range(world)]
    if visc == 0.0:
        # interior / boundary halves in every shape here (3-D N=9 FP64: by
        # the lean stage, the pipelined plan does not fit shared memory)
        assert all(p.split for p in parts)
    P.run_parts(parts, k, dt, faces=faces)
    got = np.concatenate([p.state() for p in parts], axis=2)
    for p in parts:
        p.close()
    if case == "cube9":
        # the interior half runs the shape's default stage (grouped), the
        # boundary half the lean (FP64) or pipelined (FP32) one: the two
        # agree to rounding, not bit for bit
        assert max(relerr_fields(got, ref)) < (1e-12 if precision == 64 else 1e-5)
    else:
        assert np.array_equal(got, ref)
    if precision == 64 and faces:
        assert max(relerr_fields(got, oracle_run(m, Q, dt, k, phys=phys))) < 1e-12


def test_face_traces_are_the_minimal_message():
    """The trace exchange moves Nfp values per shared face and field; whole
    elements move Np per element."""
    m, Q, dt = cube(3, 4)
    p = P.plan(m, 0, 2)
    nfaces = sum(len(c) for _, c in p.recv_faces)
    trace_values = nfaces * 16 * 5
    element_values = sum(n for _, _, n in p.recv) * 64 * 5
    assert trace_values < element_values / 3
