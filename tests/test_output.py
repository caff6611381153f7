"""VTK output of the nodal fields (the reference's writemesh sub-cell
layout) and restart checkpoints, on the host."""
import numpy as np
import pytest

from canary_b200 import dg, ic
from canary_b200.output import (VTK_PIXEL, VTK_VOXEL, load_checkpoint, read_vtu, save_checkpoint, subcells,
                                write_vtu)


@pytest.mark.parametrize("dim,N,n", [(2, 3, 2), (3, 2, 2)])
def test_vtu_layout_and_round_trip(tmp_path, dim, N, n):
    m = dg.build_mesh(dim, N, (np.linspace(0, 1, n + 1),) * dim, (True,) * dim)
    X = m.coords()
    rho = 1.0 + 0.1 * np.sin(2 * np.pi * X[0])
    f = write_vtu(str(tmp_path / "sol"), dim, N, X, [("rho", rho), ("x", X[0])])
    out = read_vtu(f)
    Np, ne = m.Np, m.nelem
    assert out["n_points"] == Np * ne and out["n_cells"] == ne * N ** dim
    assert np.array_equal(out["points"][:, 0], X[0].ravel(order="F"))
    assert np.array_equal(out["rho"], rho.ravel(order="F"))
    conn = out["connectivity"].reshape(-1, 2 ** dim)
    assert np.array_equal(conn, subcells(dim, N, ne))
    assert np.all(out["types"] == (VTK_PIXEL if dim == 2 else VTK_VOXEL))
    assert np.array_equal(out["offsets"], np.arange(1, ne * N ** dim + 1) * 2 ** dim)
    # first sub-cell: nodes (0,0), (1,0), (0,1), (1,1) [, (., ., 1)] of element 1, column-major
    Nq = N + 1
    first = [0, 1, Nq, Nq + 1] if dim == 2 else [0, 1, Nq, Nq + 1, Nq * Nq, Nq * Nq + 1, Nq * Nq + Nq,
                                                 Nq * Nq + Nq + 1]
    assert list(conn[0]) == first
    # sub-cells tile each element: every node is a corner of some sub-cell
    assert set(np.unique(conn)) == set(range(Np * ne))


def test_checkpoint_round_trip(tmp_path):
    m = dg.build_mesh(2, 3, (np.linspace(0, 10, 4),) * 2, (True, True))
    x, y = m.coords()
    Q = np.zeros((m.Np, 4, m.nelem), order="F")
    for c, v in enumerate(ic.isentropic_vortex(x, y)):
        Q[:, c] = v
    f = save_checkpoint(str(tmp_path / "ck"), Q, 17, 0.034, 0.002, dim=2, N=3, n_side=3)
    ck = load_checkpoint(f)
    assert np.array_equal(ck["Q"], Q) and ck["Q"].flags.f_contiguous
    assert ck["step"] == 17 and ck["t"] == 0.034 and ck["dt"] == 0.002 and int(ck["N"]) == 3


@pytest.mark.gpu
def test_restart_from_checkpoint_is_bit_identical(tmp_path):
    """Six steps in one run equal three steps, a checkpoint, and three more
    steps from the reloaded state (the LSRK carry is zero between steps)."""
    from conftest import cuda_available
    if not cuda_available():
        pytest.skip("needs a CUDA GPU")
    m = dg.build_mesh(2, 4, (np.linspace(0, 10, 6),) * 2, (True, True))
    x, y = m.coords()
    Q = np.zeros((m.Np, 4, m.nelem), order="F")
    for c, v in enumerate(ic.isentropic_vortex(x, y)):
        Q[:, c] = v
    dm, dt = dg.DeviceMesh.upload(m), 0.002
    s = dg.LSRK.for_state(dm, Q, 64)
    s.run(6, dt)
    full = s.state()
    s.close()
    s = dg.LSRK.for_state(dm, Q, 64)
    s.run(3, dt)
    f = save_checkpoint(str(tmp_path / "ck"), s.state(), 3, 3 * dt, dt)
    s.close()
    ck = load_checkpoint(f)
    s = dg.LSRK.for_state(dm, ck["Q"], 64)
    s.run(3, ck["dt"])
    assert np.array_equal(s.state(), full)
    s.close()
