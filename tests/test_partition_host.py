"""Partition plan and ghost exchange on the host: ranges, ghosts, send and
receive lists (elements and face traces) agree across ranks, own elements
are ordered interior first and the interior ones read no ghost, the local
maps name own and ghost elements only, and a two-rank gloo exchange delivers
every ghost face trace (and, in the element form, every ghost element) from
its owner (with stand-in parts on CPU tensors; the device solver is
exercised in tests/test_partition.py)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from canary_b200 import dg
from canary_b200 import partition as P
from canary_b200.metric import warp_sinusoidal


def _mesh():
    return dg.build_mesh(3, 2, (np.linspace(0, 1, 5),) * 3, (True, False, True),
                         meshwarp=lambda X: warp_sinusoidal(X, 0.02))


@pytest.mark.parametrize("world", [2, 3, 7])
def test_plans_agree_across_ranks(world):
    m = _mesh()
    plans = [P.plan(m, r, world) for r in range(world)]
    assert plans[0].lo == 0 and plans[-1].hi == m.nelem
    assert all(plans[r].hi == plans[r + 1].lo for r in range(world - 1))
    for p in plans:
        assert sum(n for _, _, n in p.recv) == p.nghost
        assert np.all((p.ghosts < p.lo) | (p.ghosts >= p.hi))
        ids = (p.vmapP - 1) // m.Np
        assert ids.min() >= 0 and ids.max() < p.nloc + p.nghost
        assert np.array_equal((p.vmapM - 1) // m.Np, np.broadcast_to(np.arange(p.nloc), p.vmapM.shape))
        assert np.array_equal(np.sort(p.order), np.arange(p.lo, p.hi))
        assert np.all(ids[:, :, :p.ninterior] < p.nloc)  # interior elements read no ghost
        assert np.all(np.any(ids[:, :, p.ninterior:] >= p.nloc, axis=(0, 1)))
        for q, first, n in p.recv:
            sent = dict(plans[q].send)[p.rank]
            assert np.array_equal(plans[q].order[sent], p.ghosts[first:first + n])
        # face traces: same (element, face) list on both sides, covering every
        # ghost node a face of this rank reads
        need = set()
        table = P.face_nodes(m.dim, m.N)
        for e in range(p.nloc):
            for f in range(2 * m.dim):
                idn = p.vmapP[:, f, e] - 1
                if idn[0] // m.Np >= p.nloc:
                    f2 = [g for g in range(2 * m.dim) if np.array_equal(table[g], idn % m.Np)]
                    need.add((int(idn[0] // m.Np - p.nloc), f2[0]))
        got = set()
        for q, rc in p.recv_faces:
            sc = dict(plans[q].send_faces)[p.rank]
            assert len(sc) == len(rc)
            assert np.array_equal(plans[q].order[sc >> 3], p.ghosts[rc >> 3])
            assert np.array_equal(sc & 7, rc & 7)
            got |= {(int(c >> 3), int(c & 7)) for c in rc}
        assert got == need


class _Rows:
    """Stand-in part: rows of a CPU tensor, own elements (local order) then
    ghosts; a face trace of element e, face f is e * 100 + f * 10 + 0..fw-1."""

    def __init__(self, p, ew=3, fw=4):
        import torch
        self.p, self.ew, self.widths, self.face_widths = p, ew, (ew, ew), (fw, fw)
        self.Q = torch.full((p.nloc + p.nghost, ew), -1.0, dtype=torch.float64)
        self.Q[:p.nloc] = torch.as_tensor(p.order, dtype=torch.float64)[:, None] * 10 + torch.arange(ew)
        self.faces = {}

    def pack(self, idx, buf, what=0):
        buf.copy_(self.Q[idx].reshape(-1))

    def unpack(self, buf, first, n, what=0):
        i = self.p.nloc + first
        self.Q[i:i + n] = buf.reshape(n, self.ew)

    def pack_faces(self, codes, buf, what=0):
        import torch
        fw = self.face_widths[what]
        for i, c in enumerate(codes.tolist()):
            e, f = int(self.p.order[c >> 3]), c & 7
            buf[i * fw:(i + 1) * fw] = e * 100.0 + f * 10.0 + torch.arange(fw, dtype=torch.float64)

    def unpack_faces(self, codes, buf, what=0):
        fw = self.face_widths[what]
        for i, c in enumerate(codes.tolist()):
            self.faces[(c >> 3, c & 7)] = buf[i * fw:(i + 1) * fw].clone()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, outdir):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "canary.jl_b200"), os.path.join(root, "tests")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from test_partition_host import _Rows, _mesh
    from canary_b200 import partition as P
    m = _mesh()
    p = P.plan(m, rank, world)
    part = _Rows(p)
    P.Exchange(p, part, torch.float64, "cpu", faces=False).fill()
    P.Exchange(p, part, torch.float64, "cpu").fill()
    np.save(os.path.join(outdir, f"g{rank}.npy"), part.Q[p.nloc:].numpy())
    np.save(os.path.join(outdir, f"ids{rank}.npy"), p.ghosts)
    ok = len(part.faces) == sum(len(c) for _, c in p.recv_faces) and len(part.faces) > 0
    for (g, f), v in part.faces.items():
        ok &= bool(np.array_equal(v.numpy(), p.ghosts[g] * 100.0 + f * 10.0 + np.arange(4)))
    np.save(os.path.join(outdir, f"faces_ok{rank}.npy"), np.array([ok]))
    dist.destroy_process_group()


def test_two_rank_ghost_exchange_gloo(tmp_path):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(2):
        g = np.load(tmp_path / f"g{r}.npy")
        ids = np.load(tmp_path / f"ids{r}.npy")
        assert len(ids) > 0
        assert np.array_equal(g, ids[:, None] * 10.0 + np.arange(3))
        assert np.load(tmp_path / f"faces_ok{r}.npy")[0]
