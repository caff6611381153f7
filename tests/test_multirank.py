"""Replica mode across ranks on CPU (gloo, world size 2): each rank advances
its own seeded DG instance; the only collectives are the bookkeeping
reductions used by bench.py (max of times, sum of work)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, outdir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "canary.jl_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from canary_b200 import dg, ic, replicas
    from oracle import pyoracle as O
    seed = replicas.replica_seed(7, rank)
    rng = np.random.default_rng(seed)
    m = dg.build_mesh(2, 3, (np.linspace(0, 10, 5),) * 2, (True, True))
    x, y = m.coords()
    U, V, rho, E = ic.isentropic_vortex(x, y, beta=float(rng.uniform(1, 5)))
    Q = np.asfortranarray(np.stack([U, V, rho, E], axis=1))
    rhs = np.zeros_like(Q, order="F")
    wp = dict(dg.WORKLOAD_PHYS)
    wp["lambda"] = wp.pop("lam")
    O.lowstorageRK(2, 3, m.vgeo, m.sgeo, Q, rhs, m.D, 0.002, 5, m.vmapM, m.vmapP, m.elemtobndy,
                   O.make_phys(**wp), 1)
    t = 1.0 + rank  # stand-in per-rank time
    tmax = replicas.max_over_ranks(t)
    work = replicas.sum_over_ranks(float(m.nelem * m.Np * 4))
    replicas.barrier()
    np.save(os.path.join(outdir, f"q{rank}.npy"), Q)
    with open(os.path.join(outdir, f"r{rank}.txt"), "w") as f:
        f.write(f"{tmax} {work} {replicas.rank_and_size()}")
    dist.destroy_process_group()


def test_two_rank_replicas_gloo(tmp_path):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    r0 = open(tmp_path / "r0.txt").read().split(" ", 2)
    r1 = open(tmp_path / "r1.txt").read().split(" ", 2)
    assert float(r0[0]) == float(r1[0]) == 2.0            # max of per-rank times
    assert float(r0[1]) == float(r1[1]) == 2 * 16 * 16 * 4  # summed work
    q0, q1 = np.load(tmp_path / "q0.npy"), np.load(tmp_path / "q1.npy")
    assert np.all(np.isfinite(q0)) and not np.array_equal(q0, q1)  # distinct replicas
