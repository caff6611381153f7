"""Element-partitioned solve of one mesh over several ranks, one GPU each.

The reference splits the Hilbert-ordered elements into contiguous ranges,
one per MPI rank (partition, src/mesh.jl:499-580), appends the neighbouring
ranks' elements that its faces touch as ghost elements (connectmesh,
:751-956), and before every RK stage sends whole elements to its neighbours
and receives its ghosts (fillsendQ! / transferrecvQ! and the MPI exchange of
euler2d_set2c.jl:529-594, :707-735), running volumerhs! while the receives
are in flight (:724-728).  Here:

* `plan` derives every rank's range, ghosts (sorted by global element, hence
  grouped by owner), exchange lists and local maps from the global mesh,
  with no communication.  The rank's own elements are ordered interior first
  (elements none of whose faces touch a ghost), then boundary; ghosts follow.
* The message is the minimal one: a stage reads a ghost element only at the
  face nodes of the faces shared with this rank, so each shared face carries
  Nfp x nstate values (x dim for the LDG gradient) — `send_faces` /
  `recv_faces` list (element, face) pairs in one canonical order on both
  sides.  Whole-element lists (`send` / `recv`) are kept for callers that
  exchange elements.
* `GhostedLSRK` is the rank's solver (cb_solver_create_ghosted): it advances
  its own elements one RK stage at a time, in two halves where the stage
  runs over element ranges (interior, then boundary once ghosts arrived),
  packs face traces of the current state and stores received ones.
* `Exchange` moves the traces between ranks with torch.distributed
  point-to-point operations (NCCL between GPUs; any backend whose tensors
  the solver can read), started before the interior half and finished before
  the boundary half, so the transfer overlaps interior work.
* `PartitionedLSRK` runs the LSRK steps; the viscous form (orders with the
  fused passes) exchanges the state, runs the gradient pass, exchanges the
  gradient, then runs the stage pass.

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


def face_nodes(dim: int, N: int) -> np.ndarray:
    """Local volume node of face node fn on face f, (nface, Nfp), as the
    reference's mappings orders them (mesh.jl:979-983)."""
    Nq = N + 1
    Nfp = Nq ** (dim - 1)
    out = np.zeros((2 * dim, Nfp), dtype=np.int64)
    for f in range(2 * dim):
        d0, side = f >> 1, (f & 1) * (Nq - 1)
        for fn in range(Nfp):
            if dim == 2:
                out[f, fn] = side + Nq * fn if d0 == 0 else fn + Nq * side
            else:
                a, b = fn % Nq, fn // Nq
                out[f, fn] = (side + Nq * (a + Nq * b), a + Nq * (side + Nq * b), a + Nq * (b + Nq * side))[d0]
    return out


def _ghost_faces(mesh: Mesh, lo: int, hi: int) -> np.ndarray:
    """Sorted unique (neighbour element, neighbour face) pairs, global ids,
    that the faces of elements lo..hi-1 read outside that range."""
    Np = mesh.Np
    vP = np.asarray(mesh.vmapP)[:, :, lo:hi] - 1  # (Nfp, nface, n)
    e2 = vP[0] // Np
    out = (e2 < lo) | (e2 >= hi)
    if not out.any():
        return np.zeros((0, 2), dtype=np.int64)
    fi, ei = np.nonzero(out)
    nodes = vP[:, fi, ei] % Np  # (Nfp, k)
    table = face_nodes(mesh.dim, mesh.N)  # (nface, Nfp)
    match = np.all(table[:, :, None] == nodes[None, :, :], axis=1)  # (nface, k)
    if not np.all(match.sum(axis=0) == 1):
        raise ValueError("vmapP does not describe conforming faces (orientation 1)")
    f2 = np.argmax(match, axis=0)
    pairs = np.stack([e2[fi, ei], f2], axis=1)
    return np.unique(pairs, axis=0)


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
    order: np.ndarray = None                        # global id of each own local element
    ninterior: int = 0                              # own local elements 0..ninterior-1 read no ghost
    send_faces: list = field(default_factory=list)  # (rank q, codes local element << 3 | face)
    recv_faces: list = field(default_factory=list)  # (rank q, codes ghost slot << 3 | face)

    @property
    def nloc(self) -> int:
        return self.hi - self.lo

    @property
    def nghost(self) -> int:
        return len(self.ghosts)


def plan(mesh: Mesh, rank: int, world: int) -> PartPlan:
    """Rank's part of the global mesh: range, local order (interior first),
    ghosts, exchange lists (faces and elements) and local maps."""
    nelem, Np = mesh.nelem, mesh.Np
    ranges = [part_range(nelem, q, world) for q in range(world)]
    lo, hi = ranges[rank]
    ends = np.array([r[1] for r in ranges])
    gfaces = _ghost_faces(mesh, lo, hi)
    gh = np.unique(gfaces[:, 0]) if len(gfaces) else np.zeros(0, dtype=np.int64)
    owner = np.searchsorted(ends, gh, side="right")
    recv = []
    for q in np.unique(owner):
        first = int(np.searchsorted(owner, q, side="left"))
        recv.append((int(q), first, int(np.sum(owner == q))))
    # own elements: interior (no face reads a ghost) first, then boundary
    e2 = (np.asarray(mesh.vmapP)[0, :, lo:hi] - 1) // Np  # (nface, nloc)
    boundary = np.any((e2 < lo) | (e2 >= hi), axis=0)
    order = np.concatenate([np.nonzero(~boundary)[0], np.nonzero(boundary)[0]]) + lo
    loc = np.full(nelem, -1, dtype=np.int64)
    loc[order] = np.arange(hi - lo)
    loc[gh] = (hi - lo) + np.arange(len(gh))
    send, send_faces = [], []
    for q in range(world):
        if q == rank:
            continue
        gf = _ghost_faces(mesh, *ranges[q])
        mine = gf[(gf[:, 0] >= lo) & (gf[:, 0] < hi)] if len(gf) else gf
        if len(mine):
            send.append((q, loc[np.unique(mine[:, 0])].astype(np.int64)))
            send_faces.append((q, (loc[mine[:, 0]] << 3) | mine[:, 1]))
    gslot = np.searchsorted(gh, gfaces[:, 0]) if len(gfaces) else np.zeros(0, dtype=np.int64)
    fowner = np.searchsorted(ends, gfaces[:, 0], side="right") if len(gfaces) else gslot
    recv_faces = [(q, ((gslot[fowner == q] << 3) | gfaces[fowner == q, 1]).astype(np.int64))
                  for q, _, _ in recv]
    vM = np.asarray(mesh.vmapM)[:, :, order]
    vP = np.asarray(mesh.vmapP)[:, :, order]
    vmapM = Np * np.arange(hi - lo, dtype=np.int64)[None, None, :] + (vM - 1) % Np + 1
    vmapP = Np * loc[(vP - 1) // Np] + (vP - 1) % Np + 1
    assert np.all(loc[(vP - 1) // Np] >= 0)
    return PartPlan(rank, world, lo, hi, gh, recv, send, np.asfortranarray(vmapM), np.asfortranarray(vmapP),
                    np.asfortranarray(np.asarray(mesh.elemtobndy)[:, order]), order, int(np.sum(~boundary)),
                    send_faces, recv_faces)


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
        # element width of the state and of its gradient (viscous form only),
        # and the face-trace width (values per shared face)
        self.widths = (self.ew, self.ew * mesh.dim if self.visc else self.ew)
        nfp = (mesh.N + 1) ** (mesh.dim - 1)
        self.face_widths = (ns * nfp, ns * nfp * mesh.dim if self.visc else ns * nfp)
        Q = np.asarray(Q, dtype=np.float64)
        if offset is None:
            offset = Q.mean(axis=(0, 2)) if precision == 32 else np.zeros(ns)
        self.offset = np.asarray(offset, dtype=np.float64)
        with torch.cuda.stream(self.stream):
            dev = lambda a, t=torch.float64: to_device(a, t, device)
            self.vgeo = dev(np.asarray(mesh.vgeo)[:, :, p.order])
            self.sgeo = dev(np.asarray(mesh.sgeo)[..., p.order])
            self.vmapM, self.vmapP = dev(p.vmapM, torch.int64), dev(p.vmapP, torch.int64)
            self.etb, self.D = dev(p.elemtobndy, torch.int64), dev(mesh.D)
            self.Q = torch.zeros((p.nloc + p.nghost) * self.ew, dtype=self.real, device=device)
            own = Q[:, :, p.order] - self.offset[None, :, None]
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
        # stages split into an interior and a boundary half where supported
        self.split = False
        if not self.visc:
            rc = _lib.lib().cb_solver_set_split(self._h, int(p.ninterior))
            self.split = rc == 0

    def stage(self, st: int, dt: float, pass_: int = None) -> None:
        """RK stage st (0..4) of the own elements, or one pass of it (0: the
        viscous gradient, 1: the stage); the ghosts of what it reads must have
        been filled."""
        nxt = C.c_void_p()
        if pass_ is None:
            check(_lib.lib().cb_solver_stage(self._h, int(st), float(dt), C.byref(nxt)))
        else:
            check(_lib.lib().cb_solver_stage_pass(self._h, int(st), float(dt), int(pass_), C.byref(nxt)))

    def stage_half(self, st: int, dt: float, half: int) -> None:
        """Half of RK stage st: 0 the interior elements (no ghost read), 1 the
        boundary elements (ghosts filled); the stage is complete after half 1."""
        nxt = C.c_void_p()
        check(_lib.lib().cb_solver_stage_split(self._h, int(st), float(dt), int(half), C.byref(nxt)))

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

    def pack_faces(self, codes, buf, what: int = 0) -> None:
        """Gather the face traces listed in codes (device int64, own element
        << 3 | face) of the current state (what = 0) or gradient (1)."""
        check(_lib.lib().cb_solver_pack_faces(self._h, int(what), C.c_void_p(codes.data_ptr()),
                                              int(codes.numel()), C.c_void_p(buf.data_ptr())))

    def unpack_faces(self, codes, buf, what: int = 0) -> None:
        """Store received face traces into the ghost slots listed in codes
        (ghost slot << 3 | face)."""
        check(_lib.lib().cb_solver_unpack_faces(self._h, int(what), C.c_void_p(codes.data_ptr()),
                                                int(codes.numel()), C.c_void_p(buf.data_ptr())))

    def state(self) -> np.ndarray:
        """Full FP64 state of the own elements (Np, nstate, nloc) on the host,
        in global element order lo..hi-1."""
        check(_lib.lib().cb_solver_settle(self._h))
        self.stream.synchronize()
        m, p = self.mesh, self.plan
        loc = from_device(self.Q[:p.nloc * self.ew].double(), (m.Np, nstate(m.dim), p.nloc))
        out = np.empty_like(loc)
        out[:, :, p.order - p.lo] = loc
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
    operations: face traces by default (`faces=True`; `part` provides
    pack_faces / unpack_faces and `face_widths`), or whole elements (pack /
    unpack and `widths`).  Buffers live on `device` with `dtype`.  start()
    packs and posts the transfers, finish() waits for them (stream-ordered
    for NCCL) and stores the received values; fill() does both."""

    def __init__(self, p: PartPlan, part, dtype, device, group=None, faces=True):
        torch = _torch()
        self.part, self.group, self.faces = part, group, faces
        if faces:
            wmax = max(part.face_widths)
            self.sends = [(q, torch.as_tensor(c, dtype=torch.int64, device=device),
                           torch.empty(len(c) * wmax, dtype=dtype, device=device)) for q, c in p.send_faces]
            self.recvs = [(q, torch.as_tensor(c, dtype=torch.int64, device=device),
                           torch.empty(len(c) * wmax, dtype=dtype, device=device)) for q, c in p.recv_faces]
        else:
            wmax = max(part.widths)
            self.sends = [(q, torch.as_tensor(idx, dtype=torch.int64, device=device),
                           torch.empty(len(idx) * wmax, dtype=dtype, device=device)) for q, idx in p.send]
            self.recvs = [(q, (first, n), torch.empty(n * wmax, dtype=dtype, device=device))
                          for q, first, n in p.recv]
        self._pending = None

    def _width(self, what):
        return (self.part.face_widths if self.faces else self.part.widths)[what]

    @staticmethod
    def _count(key):
        """Entries of a send (index / code tensor) or element receive ((first, n))."""
        return key[1] if isinstance(key, tuple) else key.numel()

    def start(self, what: int = 0) -> None:
        import torch.distributed as dist
        w = self._width(what)
        sends = [(q, key, buf[:self._count(key) * w]) for q, key, buf in self.sends]
        recvs = [(q, key, buf[:self._count(key) * w]) for q, key, buf in self.recvs]
        for q, key, buf in sends:
            if self.faces:
                self.part.pack_faces(key, buf, what)
            else:
                self.part.pack(key, buf, what)
        if dist.get_backend(self.group) == "nccl":  # one NCCL group for all peers
            ops = [dist.P2POp(dist.isend, buf, q, self.group) for q, _, buf in sends]
            ops += [dist.P2POp(dist.irecv, buf, q, self.group) for q, _, buf in recvs]
            reqs = dist.batch_isend_irecv(ops) if ops else []
        else:
            reqs = [dist.isend(buf, q, self.group) for q, _, buf in sends]
            reqs += [dist.irecv(buf, q, self.group) for q, _, buf in recvs]
        self._pending = (what, reqs, recvs)

    def finish(self) -> None:
        what, reqs, recvs = self._pending
        self._pending = None
        for r in reqs:
            r.wait()
        for q, key, buf in recvs:
            if self.faces:
                self.part.unpack_faces(key, buf, what)
            else:
                self.part.unpack(buf, key[0], key[1], what)

    def fill(self, what: int = 0) -> None:
        self.start(what)
        self.finish()


class PartitionedLSRK:
    """LSRK(5,4) of this rank's part of a mesh partitioned over the ranks of
    torch.distributed (initialised by the caller; one GPU per rank).  The
    inviscid form overlaps each stage's trace exchange with its interior
    elements where the stage runs over element ranges."""

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
                    if self.part.visc:
                        self.exchange.fill(0)
                        self.part.stage(st, dt, 0)
                        self.exchange.fill(1)
                        self.part.stage(st, dt, 1)
                    elif self.part.split:
                        self.exchange.start(0)
                        self.part.stage_half(st, dt, 0)
                        self.exchange.finish()
                        self.part.stage_half(st, dt, 1)
                    else:
                        self.exchange.fill(0)
                        self.part.stage(st, dt)

    def state(self) -> np.ndarray:
        return self.part.state()

    def close(self) -> None:
        self.part.close()


def run_parts(parts, nsteps: int, dt: float, faces: bool = True) -> None:
    """Advance several parts of one mesh held by this process (one GPU) in
    lock step, moving ghosts by device copies — face traces (default) or
    whole elements: the partitioned arithmetic without the inter-rank
    transport, including the interior / boundary halves of each stage.  The
    parts must share one stream."""
    torch = _torch()
    if any(p.stream != parts[0].stream for p in parts):
        raise ValueError("run_parts: the parts must be created on one stream")
    links = []  # (receiver r, sender q, sender key, receiver key, buffer)
    for r, part in enumerate(parts):
        dev = part.Q.device
        if faces:
            for q, rcodes in part.plan.recv_faces:
                scodes = dict(parts[q].plan.send_faces)[r]
                links.append((r, q, torch.as_tensor(scodes, dtype=torch.int64, device=dev),
                              torch.as_tensor(rcodes, dtype=torch.int64, device=dev),
                              torch.empty(len(rcodes) * max(part.face_widths), dtype=part.real, device=dev)))
        else:
            for q, first, n in part.plan.recv:
                idx = dict(parts[q].plan.send)[r]
                links.append((r, q, torch.as_tensor(idx, dtype=torch.int64, device=dev), (first, n),
                              torch.empty(n * max(part.widths), dtype=part.real, device=dev)))

    def fill(what):
        for r, q, skey, rkey, buf in links:
            if faces:
                b = buf[:skey.numel() * parts[r].face_widths[what]]
                parts[q].pack_faces(skey, b, what)
                parts[r].unpack_faces(rkey, b, what)
            else:
                b = buf[:rkey[1] * parts[r].widths[what]]
                parts[q].pack(skey, b, what)
                parts[r].unpack(b, rkey[0], rkey[1], what)

    split = all(p.split for p in parts)
    with torch.cuda.stream(parts[0].stream):
        for _ in range(nsteps):
            for st in range(5):
                if parts[0].visc:
                    fill(0)
                    for part in parts:
                        part.stage(st, dt, 0)
                    fill(1)
                    for part in parts:
                        part.stage(st, dt, 1)
                elif split:
                    for part in parts:  # interior halves read no ghost
                        part.stage_half(st, dt, 0)
                    fill(0)  # packs read the state the stage started from
                    for part in parts:
                        part.stage_half(st, dt, 1)
                else:
                    fill(0)
                    for part in parts:
                        part.stage(st, dt)
