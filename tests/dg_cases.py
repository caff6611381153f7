"""Shared builders of DG test cases (meshes, initial states, error norms)."""
import math

import numpy as np

from oracle import pyoracle as O
from canary_b200 import dg, ic
from canary_b200.metric import warp_sinusoidal


def oracle_phys(d):
    d = dict(d)
    d["lambda"] = d.pop("lam")
    return O.make_phys(**d)


def relerr_fields(a, b):
    """Relative L2 error per state field (axis 1)."""
    out = []
    for s in range(a.shape[1]):
        den = np.linalg.norm(b[:, s])
        out.append(np.linalg.norm(a[:, s] - b[:, s]) / (den if den > 0 else 1.0))
    return out


def vortex_case(N, n_side, beta=5.0, xc=5.0, yc=5.0):
    """2-D isentropic vortex on the periodic square [0,10]^2."""
    m = dg.build_mesh(2, N, (np.linspace(0, 10, n_side + 1),) * 2, (True, True))
    x, y = m.coords()
    U, V, rho, E = ic.isentropic_vortex(x, y, beta, xc, yc)
    Q = np.zeros((m.Np, 4, m.nelem), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3] = U, V, rho, E
    return m, Q


def fourier_case(N, n_side, seed=0):
    """3-D random Fourier state on the warped periodic cube [0,2π]^3; returns
    (mesh, Q, dt) with dt from the CFL rule of the workload."""
    m = dg.build_mesh(3, N, (np.linspace(0, 2 * math.pi, n_side + 1),) * 3, (True,) * 3,
                      meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    x, y, z = m.coords()
    U, V, W, rho, E = ic.fourier_state(x, y, z, seed=seed)
    Q = np.zeros((m.Np, 5, m.nelem), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3], Q[:, 4] = U, V, W, rho, E
    return m, Q, ic.fourier_dt(Q, N, h=2 * math.pi / n_side)


def oracle_run(m, Q, dt, nsteps, phys=None, threads=None):
    """FP64 oracle LSRK(5,4) of a host state; returns the final state."""
    import os
    ref, rref = Q.copy(order="F"), np.zeros_like(Q, order="F")
    O.lowstorageRK(m.dim, m.N, m.vgeo, m.sgeo, ref, rref, m.D, dt, nsteps, m.vmapM, m.vmapP,
                   m.elemtobndy, oracle_phys(phys or dg.WORKLOAD_PHYS), threads or os.cpu_count() or 1)
    return ref
