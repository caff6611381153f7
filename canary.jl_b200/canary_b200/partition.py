"""Element-partitioned solve of one mesh over several ranks, one GPU each.

The reference splits the Hilbert-ordered elements into contiguous ranges,
one per MPI rank (partition, src/mesh.jl:499-580), appends the neighbouring
ranks' elements that its faces touch as ghost elements (connectmesh,
:751-956), and before every RK stage sends the elements its neighbours need
and receives its ghosts (fillsendQ! / transferrecvQ! and the MPI exchange of
euler2d_set2c.jl:529-594, :707-735).  Here:

* `plan` derives every rank's range, ghosts (sorted by global element, hence
  grouped by owner), receive ranges and send lists from the global mesh,
  with no communication, and the rank's local maps (own elements first,
  ghosts after them);
* `GhostedLSRK` is the rank's solver (cb_solver_create_ghosted): it
  advances its own elements one RK stage at a time, packs the elements a
  neighbour needs from the current state and stores received ghosts into it;
* `Exchange` moves the packed elements between ranks with
  torch.distributed point-to-point operations (NCCL between GPUs; any
  backend whose tensors the solver can read);
* `PartitionedLSRK` runs the LSRK steps: exchange, then stage, five times a
  step; the viscous form (orders with the fused passes) exchanges the state,
  runs the gradient pass, exchanges the gradient, then runs the stage pass.

Every element's arithmetic is the single-mesh solver's, so the partitioned
result equals the unpartitioned one bit for bit (tests/test_partition.py
checks this with several partitions in one process).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check
from .dg import Mesh, _ptr, _stream, _torch, from_device, make_phys, nstate, to_device


def part_range(nelem: int, rank: int, world: int) -> tuple[int, int]:
    """0-based [lo, hi) of rank's elements (linearpartition, mesh.jl:13)."""
    return rank * nelem // world, (rank + 1) * nelem // world


def _ghosts(mesh: Mesh, lo: int, hi: int) -> np.ndarray:
    eP = (np.asarray(mesh.vmapP)[:, :, lo:hi] - 1) // mesh.Np
    return np.unique(eP[(eP < lo) | (eP >= hi)])


@dataclass
class PartPlan:
    rank: int
    world: int
    lo: int
    hi: int
    ghosts: np.ndarray                              # global ids, sorted
    recv: list = field(default_factory=list)        # (rank q, first ghost, count)
    send: list = field(default_factory=list)        # (rank q, local element ids)
    vmapM: np.ndarray = None                        # local maps (Nfp, nface, nloc), 1-based
    vmapP: np.ndarray = None
    elemtobndy: np.ndarray = None

    @property
    def nloc(self) -> int:
        return self.hi - self.lo

    @property
    def nghost(self) -> int:
        return len(self.ghosts)


def plan(mesh: Mesh, rank: int, world: int) -> PartPlan:
    """Rank's part of the global mesh: range, ghosts, exchange lists, local maps."""
    nelem, Np = mesh.nelem, mesh.Np
    ranges = [part_range(nelem, q, world) for q in range(world)]
    lo, hi = ranges[rank]
    gh = _ghosts(mesh, lo, hi)
    owner = np.searchsorted(np.array([r[1] for r in ranges]), gh, side="right")
    recv = []
    for q in np.unique(owner):
        first = int(np.searchsorted(owner, q, side="left"))
        recv.append((int(q), first, int(np.sum(owner == q))))
    send = []
    for q in range(world):
        if q == rank:
            continue
        g = _ghosts(mesh, *ranges[q])
        mine = g[(g >= lo) & (g < hi)]
        if len(mine):
            send.append((q, (mine - lo).astype(np.int64)))
    loc = np.full(nelem, -1, dtype=np.int64)
    loc[lo:hi] = np.arange(hi - lo)
    loc[gh] = (hi - lo) + np.arange(len(gh))
    vM = np.asarray(mesh.vmapM)[:, :, lo:hi]
    vP = np.asarray(mesh.vmapP)[:, :, lo:hi]
    vmapM = Np * np.arange(hi - lo, dtype=np.int64)[None, None, :] + (vM - 1) % Np + 1
    vmapP = Np * loc[(vP - 1) // Np] + (vP - 1) % Np + 1
    assert np.all(loc[(vP - 1) // Np] >= 0)
    return PartPlan(rank, world, lo, hi, gh, recv, send, np.asfortranarray(vmapM), np.asfortranarray(vmapP),
                    np.asfortranarray(np.asarray(mesh.elemtobndy)[:, lo:hi]))


class GhostedLSRK:
    """A rank's solver (cb_solver_create_ghosted) for its part of `mesh`,
    starting from the global host state Q (Np, nstate, nelem).  All its work
    — stages, packing, unpacking — is ordered on `stream` (a torch stream; a
    new one by default), on which the exchange of its buffers must run too."""

    def __init__(self, mesh: Mesh, p: PartPlan, Q: np.ndarray, precision=64, phys=None, stream=None,
                 device="cuda", offset=None):
        torch = _torch()
        self.mesh, self.plan, self.precision = mesh, p, precision
        self.stream = stream or torch.cuda.Stream(torch.device(device))
        self.real = torch.float64 if precision == 64 else torch.float32
        self.phys = phys or make_phys()
        ns, Np = nstate(mesh.dim), mesh.Np
        self.ew = ns * Np
        self.visc = self.phys.visc > 0
        # element width of the state and of its gradient (viscous form only)
        self.widths = (self.ew, self.ew * mesh.dim if self.visc else self.ew)
        Q = np.asarray(Q, dtype=np.float64)
        if offset is None:
            offset = Q.mean(axis=(0, 2)) if precision == 32 else np.zeros(ns)
        self.offset = np.asarray(offset, dtype=np.float64)
        with torch.cuda.stream(self.stream):
            dev = lambda a, t=torch.float64: to_device(a, t, device)
            self.vgeo = dev(np.asarray(mesh.vgeo)[:, :, p.lo:p.hi])
            self.sgeo = dev(np.asarray(mesh.sgeo)[..., p.lo:p.hi])
            self.vmapM, self.vmapP = dev(p.vmapM, torch.int64), dev(p.vmapP, torch.int64)
            self.etb, self.D = dev(p.elemtobndy, torch.int64), dev(mesh.D)
            self.Q = torch.zeros((p.nloc + p.nghost) * self.ew, dtype=self.real, device=device)
            own = Q[:, :, p.lo:p.hi] - self.offset[None, :, None]
            self.Q[:p.nloc * self.ew] = to_device(own, self.real, device)
            self.rhs = torch.zeros_like(self.Q)
        self._h = C.c_void_p()
        check(_lib.lib().cb_solver_create_ghosted(
            C.byref(self._h), mesh.dim, mesh.N, precision, p.nloc, p.nghost, _ptr(self.Q, self.real),
            _ptr(self.rhs, self.real), _ptr(self.vgeo, torch.float64), _ptr(self.sgeo, torch.float64),
            _ptr(self.vmapM, torch.int64), _ptr(self.vmapP, torch.int64), _ptr(self.etb, torch.int64),
            _ptr(self.D, torch.float64), C.byref(self.phys), _stream(self.stream)))
        arr = (C.c_double * 5)(*([float(v) for v in self.offset] + [0.0] * (5 - ns)))
        check(_lib.lib().cb_solver_set_offset(self._h, arr))

    def stage(self, st: int, dt: float, pass_: int = None) -> None:
        """RK stage st (0..4) of the own elements, or one pass of it (0: the
        viscous gradient, 1: the stage); the ghosts of what it reads must have
        been filled."""
        nxt = C.c_void_p()
        if pass_ is None:
            check(_lib.lib().cb_solver_stage(self._h, int(st), float(dt), C.byref(nxt)))
        else:
            check(_lib.lib().cb_solver_stage_pass(self._h, int(st), float(dt), int(pass_), C.byref(nxt)))

    def pack(self, idx, buf, what: int = 0) -> None:
        """Gather own elements idx (device int64) of the current state (what =
        0) or of the gradient (1) into buf."""
        check(_lib.lib().cb_solver_pack(self._h, int(what), C.c_void_p(idx.data_ptr()), int(idx.numel()),
                                        C.c_void_p(buf.data_ptr())))

    def unpack(self, buf, first: int, count: int, what: int = 0) -> None:
        """Store count received elements from buf as ghosts first.. of the
        current state (what = 0) or of the gradient (1)."""
        check(_lib.lib().cb_solver_unpack(self._h, int(what), C.c_void_p(buf.data_ptr()), int(first),
                                          int(count)))

    def state(self) -> np.ndarray:
        """Full FP64 state of the own elements (Np, nstate, nloc) on the host."""
        check(_lib.lib().cb_solver_settle(self._h))
        self.stream.synchronize()
        m, p = self.mesh, self.plan
        out = from_device(self.Q[:p.nloc * self.ew].double(), (m.Np, nstate(m.dim), p.nloc))
        return out + self.offset[None, :, None]

    def close(self) -> None:
        if self._h:
            _lib.lib().cb_solver_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Exchange:
    """Ghost exchange of one rank with torch.distributed point-to-point
    operations.  `part` provides pack(idx, buf, what) / unpack(buf, first,
    count, what) and the element widths `widths` of what = 0 (state) and 1
    (gradient); buffers live on `device` with `dtype`."""

    def __init__(self, p: PartPlan, part, dtype, device, group=None):
        torch = _torch()
        self.part, self.group = part, group
        wmax = max(part.widths)
        self.sends = [(q, torch.as_tensor(idx, dtype=torch.int64, device=device),
                       torch.empty(len(idx) * wmax, dtype=dtype, device=device)) for q, idx in p.send]
        self.recvs = [(q, first, n, torch.empty(n * wmax, dtype=dtype, device=device)) for q, first, n in p.recv]

    def fill(self, what: int = 0) -> None:
        import torch.distributed as dist
        w = self.part.widths[what]
        sends = [(q, idx, buf[:len(idx) * w]) for q, idx, buf in self.sends]
        recvs = [(q, first, n, buf[:n * w]) for q, first, n, buf in self.recvs]
        for q, idx, buf in sends:
            self.part.pack(idx, buf, what)
        if dist.get_backend(self.group) == "nccl":  # one NCCL group for all peers
            ops = [dist.P2POp(dist.isend, buf, q, self.group) for q, _, buf in sends]
            ops += [dist.P2POp(dist.irecv, buf, q, self.group) for q, _, _, buf in recvs]
            reqs = dist.batch_isend_irecv(ops) if ops else []
        else:
            reqs = [dist.isend(buf, q, self.group) for q, _, buf in sends]
            reqs += [dist.irecv(buf, q, self.group) for q, _, _, buf in recvs]
        for r in reqs:
            r.wait()
        for q, first, n, buf in recvs:
            self.part.unpack(buf, first, n, what)


class PartitionedLSRK:
    """LSRK(5,4) of this rank's part of a mesh partitioned over the ranks of
    torch.distributed (initialised by the caller; one GPU per rank)."""

    def __init__(self, mesh: Mesh, Q: np.ndarray, rank: int, world: int, precision=64, phys=None, stream=None,
                 device="cuda", group=None, offset=None):
        self.plan = plan(mesh, rank, world)
        self.part = GhostedLSRK(mesh, self.plan, Q, precision, phys, stream, device, offset)
        self.exchange = Exchange(self.plan, self.part, self.part.real, device, group)

    def run(self, nsteps: int, dt: float) -> None:
        torch = _torch()
        with torch.cuda.stream(self.part.stream):
            for _ in range(nsteps):
                for st in range(5):
                    self.exchange.fill(0)
                    if self.part.visc:
                        self.part.stage(st, dt, 0)
                        self.exchange.fill(1)
                        self.part.stage(st, dt, 1)
                    else:
                        self.part.stage(st, dt)

    def state(self) -> np.ndarray:
        return self.part.state()

    def close(self) -> None:
        self.part.close()


def run_parts(parts, nsteps: int, dt: float) -> None:
    """Advance several parts of one mesh held by this process (one GPU) in
    lock step, moving ghosts by device copies: the partitioned arithmetic
    without the inter-rank transport.  The parts must share one stream."""
    torch = _torch()
    if any(p.stream != parts[0].stream for p in parts):
        raise ValueError("run_parts: the parts must be created on one stream")
    bufs = {}
    for r, part in enumerate(parts):
        for q, first, n in part.plan.recv:
            idx = dict(parts[q].plan.send)[r]
            bufs[(r, q)] = (torch.as_tensor(idx, dtype=torch.int64, device=part.Q.device),
                            torch.empty(n * max(part.widths), dtype=part.real, device=part.Q.device), first, n)

    def fill(what):
        for r, part in enumerate(parts):
            for q, first, n in part.plan.recv:
                idx, buf, first, n = bufs[(r, q)]
                b = buf[:n * part.widths[what]]
                parts[q].pack(idx, b, what)
                part.unpack(b, first, n, what)

    with torch.cuda.stream(parts[0].stream):
        for _ in range(nsteps):
            for st in range(5):
                fill(0)
                if parts[0].visc:
                    for part in parts:
                        part.stage(st, dt, 0)
                    fill(1)
                    for part in parts:
                        part.stage(st, dt, 1)
                else:
                    for part in parts:
                        part.stage(st, dt)
