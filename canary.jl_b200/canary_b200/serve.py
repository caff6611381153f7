"""Serving loop over a stream of solve requests (continuous batching).

A request names a problem (2-D isentropic vortex, 3-D periodic Euler with the
seeded Fourier state, or its LDG Navier–Stokes variant), its order and mesh
size, its initial-condition parameters and a final time.  The server keeps
every admitted state resident on the device, admits requests in arrival order
while their memory fits an HBM budget, and advances all inviscid requests
together in one Batch (one graph launch per LSRK step, each instance with its
own dt and step count) and all Navier–Stokes requests in a second, viscous
Batch on its own stream, overlapping the first on the device.  Finished
instances are retired
and copied to pinned host memory without stopping the others, and their slots
and memory go to the next requests.  Latency is arrival -> final state on the
host, timed with CUDA events on the device clock.

The per-instance arithmetic is that of a single solve: an instance's result
does not depend on what else is being served (tests/test_serve.py).
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import ic
from .batch import Batch, BatchMesh
from .dg import LSRK, DeviceMesh, _torch, make_phys, nstate

GAMMA = 1.4
KINDS = ("vortex", "euler3d", "ns3d")
VISC = 1e-3  # LDG Navier–Stokes requests: mu (the `visc` multiplier) and Pr = 0.72


@dataclass
class Request:
    rid: int
    kind: str
    N: int
    n_side: int
    t_final: float
    arrival: float
    beta: float = 5.0
    xc: float = 5.0
    yc: float = 5.0
    seed: int = 0
    # 3-D requests: peak magnitude each velocity component's Fourier sum is
    # scaled to (None: the literal sums, amplitudes a_k ~ U(0, 0.1) per mode)
    vel_peak: float = None

    @property
    def dim(self) -> int:
        return 2 if self.kind == "vortex" else 3


def request_stream(count: int, rate: float, seed: int = 0, mix=(0.70, 0.15, 0.15), vel_peak=None):
    """`count` requests with Poisson arrivals of rate `rate` per second (all
    at t = 0 when rate <= 0).  Parameters are drawn from numpy's PCG64(seed)
    (the same requests at every rate), arrival gaps from PCG64(seed + 2^32):
    kind by `mix` (vortex, 3-D Euler, 3-D Navier–Stokes); vortex N ~ U{3..8},
    n_side ~ U{8..64}, beta ~ U(1,5), centre ~ U([2,8]^2); 3-D N ~ U{3..7},
    n_side ~ U{4..16}, Fourier seed = request id; t_final ~ U(0.5, 2).

    The literal 3-D state (257 modes, velocity amplitudes up to 0.1 each)
    steepens into shocks that the unlimited scheme does not survive to
    t = 0.5; with `vel_peak` (e.g. 0.1) every 3-D request's velocity sums are
    normalised to that peak magnitude, and those requests complete."""
    rng = np.random.Generator(np.random.PCG64(seed))
    arr = np.random.Generator(np.random.PCG64(seed + 2 ** 32))
    t, out = 0.0, []
    for i in range(count):
        if rate > 0:
            t += float(arr.exponential(1.0 / rate))
        u = float(rng.random())
        kind = "vortex" if u < mix[0] else ("euler3d" if u < mix[0] + mix[1] else "ns3d")
        if kind == "vortex":
            N, n = int(rng.integers(3, 9)), int(rng.integers(8, 65))
            beta = float(rng.uniform(1.0, 5.0))
            xc, yc = (float(v) for v in rng.uniform(2.0, 8.0, 2))
            r = Request(i, kind, N, n, 0.0, t, beta, xc, yc)
        else:
            N, n = int(rng.integers(3, 8)), int(rng.integers(4, 17))
            r = Request(i, kind, N, n, 0.0, t, seed=i, vel_peak=vel_peak)
        r.t_final = float(rng.uniform(0.5, 2.0))
        out.append(r)
    return out


@dataclass
class _Mesh:
    dmesh: DeviceMesh
    bytes: int
    batch: dict = field(default_factory=dict)  # precision -> BatchMesh
    users: int = 0
    last: float = 0.0


class MeshPool:
    """Device meshes shared by requests with the same (kind, N, n_side):
    [0,10]^2 for the vortex, the warped cube [0,2π]^3 (x_i += 0.05 sin x sin y
    sin z) otherwise; geometry computed on the device.  Unused meshes are
    evicted least-recently-used when memory is needed."""

    def __init__(self, device, stream):
        self.device, self.stream = device, stream
        self.meshes = {}

    @staticmethod
    def key(req: Request):
        return ("square" if req.dim == 2 else "cube", req.N, req.n_side)

    @staticmethod
    def nbytes(dim, N, n, precision):
        Nq = N + 1
        nelem, Np, Nfp = n ** dim, Nq ** dim, Nq ** (dim - 1)
        nvg, nsg = (14, 5) if dim == 3 else (8, 4)
        b64 = 8 * nelem * (Np * nvg + nsg * Nfp * 2 * dim + 2 * Nfp * 2 * dim + 2 * dim)
        b32 = 4 * nelem * (Np * nvg + nsg * Nfp * 2 * dim + 2 * dim)
        return b64 + (b32 if precision == 32 else 0)

    def get(self, req: Request, precision: int, batch: bool = True):
        """The request's mesh; with `batch`, also its batch mesh (cb_mesh) of
        that precision."""
        torch = _torch()
        k = self.key(req)
        m = self.meshes.get(k)
        if m is None:
            L = 10.0 if req.dim == 2 else 2 * math.pi
            x = (np.linspace(0.0, L, req.n_side + 1),) * req.dim
            with torch.cuda.stream(self.stream):
                dm = DeviceMesh.build(req.dim, req.N, x, (True,) * req.dim,
                                      warp_amp=0.0 if req.dim == 2 else 0.05, device=self.device,
                                      stream=self.stream)
            m = self.meshes[k] = _Mesh(dm, self.nbytes(req.dim, req.N, req.n_side, precision))
        if batch and precision not in m.batch:
            m.batch[precision] = BatchMesh(m.dmesh, precision, stream=self.stream)
        m.users += 1
        m.last = time.perf_counter()
        return m

    def release(self, req: Request):
        self.meshes[self.key(req)].users -= 1

    def resident_bytes(self):
        return sum(m.bytes for m in self.meshes.values())

    def evict(self, need: int, budget: int, in_use: int) -> bool:
        """Evict unused meshes (LRU) until in_use + resident + need <= budget."""
        while in_use + self.resident_bytes() + need > budget:
            idle = [(m.last, k) for k, m in self.meshes.items() if m.users == 0]
            if not idle:
                return False
            _, k = min(idle)
            for bm in self.meshes[k].batch.values():
                bm.close()
            del self.meshes[k]
        return True


class _Lane:
    """One batch (inviscid or viscous) with its stream and the asynchronous
    copy of its per-slot status words."""

    def __init__(self, batch: Batch, stream, max_instances: int):
        torch = _torch()
        self.batch, self.stream = batch, stream
        self.stat = torch.zeros(max_instances, dtype=torch.int32, pin_memory=True)
        self.stat_ev, self.stat_tick, self.live = None, 0, 0


@dataclass
class _Prep:
    """A request whose mesh and initial state are being set up on the setup
    stream; `speed` (pinned) receives its max wave speed, `event` marks the
    end of the set-up."""
    req: Request
    mesh: _Mesh
    bytes: int
    offset: np.ndarray
    Q: object
    rhs: object
    speed: object
    event: object


@dataclass
class _Live:
    req: Request
    mesh: _Mesh
    nsteps: int
    dt: float
    bytes: int
    offset: np.ndarray
    lane: _Lane = None
    Q: object = None
    rhs: object = None
    slot: int = -1
    left: int = 0
    admitted: float = 0.0
    failed: bool = False
    tick0: int = 0  # loop tick at admission


def _pcts(lat):
    # no completed request: the statistics are undefined (None, JSON null)
    if not len(lat):
        return {"p50_s": None, "p99_s": None, "mean_s": None}
    a = np.asarray(lat)
    return {"p50_s": float(np.percentile(a, 50)), "p99_s": float(np.percentile(a, 99)), "mean_s": float(a.mean())}


@dataclass
class Report:
    latencies: dict  # request id -> arrival-to-final-state seconds (completed and failed requests)
    results: dict
    start: float
    end: float
    dof_stage: float  # all device work, failed requests included
    peak_bytes: int
    max_live: int
    failed: set = field(default_factory=set)  # requests whose final state is not finite
    kinds: dict = field(default_factory=dict)  # request id -> kind, every request offered
    rejected: dict = field(default_factory=dict)  # request id -> reason (never admitted)
    cancelled: set = field(default_factory=set)  # withdrawn by the client before they finished
    work: dict = field(default_factory=dict)  # request id -> DOF·stage updates of its solve

    def completed(self):
        return {r: t for r, t in self.latencies.items() if r not in self.failed and r not in self.cancelled}

    def summary(self) -> dict:
        """Throughput and latency over the requests that completed with a
        finite final state; failed, rejected and cancelled requests are
        counted separately and enter no rate or percentile."""
        done = self.completed()
        span = self.end - self.start
        ok = span > 0
        out = {"requests": len(self.kinds) or len(self.latencies), "completed": len(done),
               "failed": len(self.failed), "rejected": len(self.rejected), "cancelled": len(self.cancelled)}
        out.update(_pcts(list(done.values())))
        out.update({"solves_per_s": len(done) / span if ok else None, "span_s": span,
                    "dof_stage_per_s": self.dof_stage / span if ok else None,
                    "completed_dof_stage_per_s":
                        sum(self.work.get(r, 0.0) for r in done) / span if ok else None,
                    "peak_hbm_bytes": self.peak_bytes, "max_concurrent": self.max_live})
        if self.kinds:
            per = {}
            for k in KINDS:
                ids = [r for r, kk in self.kinds.items() if kk == k]
                if not ids:
                    continue
                lat = [done[r] for r in ids if r in done]
                per[k] = {"requests": len(ids), "completed": len(lat),
                          "failed": sum(1 for r in ids if r in self.failed),
                          "rejected": sum(1 for r in ids if r in self.rejected),
                          "cancelled": sum(1 for r in ids if r in self.cancelled)}
                per[k].update(_pcts(lat))
            out["per_kind"] = per
        return out


def plan(req: Request, speed: float):
    """dt = 0.2 h / (N^2 max(|u|+c)) with h the element size, rounded down so
    that an integer number of steps reaches t_final."""
    h = (10.0 if req.dim == 2 else 2 * math.pi) / req.n_side
    dt = 0.2 * h / (req.N * req.N * speed)
    n = max(1, math.ceil(req.t_final / dt))
    return n, req.t_final / n


def wave_speed(fields, dim, gamma=GAMMA):
    """Device max over nodes of |u| + c of conserved fields (U, V, [W], ρ, E)."""
    torch = _torch()
    mom = fields[:dim]
    rho, E = fields[dim], fields[dim + 1]
    m2 = sum(m * m for m in mom)
    p = (gamma - 1.0) * (E - m2 / (2.0 * rho))
    return torch.max(torch.sqrt(m2) / rho + torch.sqrt(gamma * p / rho))


class Server:
    """Continuous-batching server on one GPU.  precision 32 is the served
    form (FP32 state and arithmetic, FP64 geometry rounded once, per-field
    state offsets); tick_steps steps are launched per loop iteration, with at
    most two ticks in flight."""

    def __init__(self, precision=32, hbm_budget=120e9, max_instances=4096, tick_steps=8, device="cuda",
                 admit_slice=0.02):
        torch = _torch()
        self.torch = torch
        self.device = torch.device(device)
        self.precision = precision
        self.real = torch.float32 if precision == 32 else torch.float64
        self.budget = int(hbm_budget)
        self.tick = tick_steps
        # host seconds of admissions (mesh set-up, initial states) between two
        # ticks while requests are resident, so that device work overlaps them
        self.admit_slice = admit_slice
        # meshes and initial states; high priority, so that set-up kernels get
        # SMs between the batches' persistent stage kernels
        self.sstream = torch.cuda.Stream(self.device, priority=-1)
        self.max_instances = max_instances
        # the inviscid and the viscous batch, each on its own stream (with
        # their admissions and retirements)
        self.lanes = {}
        for visc in (False, True):
            st = torch.cuda.Stream(self.device)
            phys = make_phys(visc=VISC) if visc else make_phys()
            self.lanes[visc] = _Lane(Batch(precision, max_instances, phys, stream=st), st, max_instances)
        self.batch = self.lanes[False].batch
        self.pool = MeshPool(self.device, self.sstream)
        self.in_use = 0
        # fault injection on the host: request ids whose next set-up fails
        # as a device allocation beyond the HBM actually available would
        # (a simulated HBM-budget overflow)
        self.fail_alloc = set()

    # ---------------------------------------------------------------- requests
    def request_bytes(self, req: Request) -> int:
        Nq = req.N + 1
        n = (req.n_side ** req.dim) * (Nq ** req.dim) * nstate(req.dim)
        w = 4 if self.precision == 32 else 8
        if req.kind == "ns3d":  # Q, rhs, batch-owned twin and gradient (dim x state)
            return w * n * (3 + req.dim)
        return 3 * w * n  # Q, rhs, batch-owned twin

    def never_fits(self, req: Request) -> bool:
        """Whether the request's own memory and its mesh exceed the whole
        budget (it can never be admitted)."""
        return self.request_bytes(req) + MeshPool.nbytes(req.dim, req.N, req.n_side, self.precision) > self.budget

    def prepare(self, req: Request) -> _Prep:
        """Reserve the request's memory and enqueue its mesh (if not cached)
        and initial state on the setup stream, without waiting for them.
        Raises torch.cuda.OutOfMemoryError when a device allocation fails (or
        is made to fail by `fail_alloc`); nothing stays reserved then."""
        torch = self.torch
        if req.rid in self.fail_alloc:
            self.fail_alloc.discard(req.rid)
            raise torch.cuda.OutOfMemoryError(f"request {req.rid}: simulated device allocation failure")
        m = self.pool.get(req, self.precision)
        try:
            return self._prepare_on(req, m)
        except torch.cuda.OutOfMemoryError:
            self.pool.release(req)
            raise

    def _prepare_on(self, req: Request, m: _Mesh) -> _Prep:
        torch = self.torch
        with torch.cuda.stream(self.sstream):
            x = m.dmesh.coords()
            if req.kind == "vortex":
                f = ic.isentropic_vortex_t(x[0], x[1], req.beta, req.xc, req.yc)
                off = np.array([1.0, 0.0, 1.0, 1.0 / (GAMMA - 1.0) + 0.5])
            else:
                f = ic.fourier_state_t(x[0], x[1], x[2], seed=req.seed, vel_peak=req.vel_peak)
                off = np.array([0.0, 0.0, 0.0, 1.0, 1.0 / (GAMMA - 1.0)])
            speed = torch.empty(1, dtype=torch.float64, pin_memory=True)
            speed.copy_(wave_speed(f, req.dim).reshape(1), non_blocking=True)
            if self.precision == 64:
                off = np.zeros(nstate(req.dim))
            Q = ic.device_state(list(f), self.real, off)
            rhs = torch.zeros_like(Q)
        ev = torch.cuda.Event()
        ev.record(self.sstream)
        nb = self.request_bytes(req)
        self.in_use += nb
        return _Prep(req, m, nb, off, Q, rhs, speed, ev)

    def admit(self, pr: _Prep, now: float) -> _Live:
        """Admit a prepared request (its set-up event has completed) into its
        batch."""
        req, Q, rhs = pr.req, pr.Q, pr.rhs
        nsteps, dt = plan(req, float(pr.speed[0]))
        lane = self.lanes[req.kind == "ns3d"]
        live = _Live(req, pr.mesh, nsteps, dt, pr.bytes, pr.offset, lane, Q, rhs, left=nsteps, admitted=now)
        lane.stream.wait_stream(self.sstream)
        Q.record_stream(lane.stream)
        rhs.record_stream(lane.stream)
        live.slot = lane.batch.add(pr.mesh.batch[self.precision], Q, rhs, dt, nsteps, pr.offset)
        lane.live += 1
        return live

    def _fits(self, req: Request) -> bool:
        k = MeshPool.key(req)
        mesh_new = 0 if k in self.pool.meshes else MeshPool.nbytes(req.dim, req.N, req.n_side, self.precision)
        return self.pool.evict(self.request_bytes(req) + mesh_new, self.budget, self.in_use)

    # ---------------------------------------------------------------- loop
    def serve(self, requests, realtime=True, cancel=None) -> Report:
        """Serve `requests` (arrival times in seconds from the start); with
        realtime=False every request is present at t = 0 and admitted in
        arrival order (a closed-loop capacity run; latencies count from 0).

        `cancel` maps request ids to the time (seconds from the start) at
        which their client withdraws them: a request not yet admitted is
        dropped, an admitted one is retired without a result, one already
        finished is unaffected.  A request whose memory alone exceeds the
        budget is rejected at arrival; one whose set-up fails to allocate
        waits for memory to free up, or is rejected if nothing else holds
        memory.  The other requests continue in every case."""
        torch = self.torch
        reqs = deque(sorted(requests, key=lambda r: (r.arrival, r.rid)))
        kinds = {r.rid: r.kind for r in requests}
        cancel = dict(cancel or {})
        waiting, preparing, live, retiring = deque(), deque(), {}, []
        lat, results, failed, rejected, cancelled, work = {}, {}, set(), {}, set(), {}
        flight = {}  # stream -> events of the ticks in flight
        ticks = 0
        dof_stage, peak, max_live = 0.0, 0, 0
        base = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(self.device)
        base.record(self.lanes[False].stream)
        t0 = time.perf_counter()

        def tick_done(stream):
            ev = torch.cuda.Event()
            ev.record(stream)
            q = flight.setdefault(stream, deque())
            q.append(ev)
            if len(q) > 2:  # at most two ticks in flight per stream
                q.popleft().synchronize()

        def withdrawn(rid, now):
            return rid in cancel and cancel[rid] <= now

        while reqs or waiting or preparing or live or retiring:
            now = time.perf_counter() - t0
            while reqs and (not realtime or reqs[0].arrival <= now):
                r = reqs.popleft()
                if self.never_fits(r):
                    rejected[r.rid] = "its memory alone exceeds the HBM budget"
                else:
                    waiting.append(r)
            # cancellations of requests not yet admitted, and of live ones
            for r in [r for r in waiting if withdrawn(r.rid, now)]:
                waiting.remove(r)
                cancelled.add(r.rid)
            for rid, lv in list(live.items()):
                if withdrawn(rid, now):
                    cancelled.add(rid)
                    retiring.append(self._retire(lv, copy=False))
                    del live[rid]
            # set-up of arriving requests (asynchronous), then admission of
            # those whose set-up has completed, in arrival order
            t_adm = time.perf_counter()
            while waiting and self._fits(waiting[0]):
                try:
                    preparing.append(self.prepare(waiting[0]))
                except torch.cuda.OutOfMemoryError:
                    if live or preparing or retiring:
                        break  # retry once memory has been freed
                    rejected[waiting.popleft().rid] = "device allocation failed with nothing else resident"
                    continue
                waiting.popleft()
                if time.perf_counter() - t_adm > self.admit_slice:
                    break
            if preparing and not live:
                preparing[0].event.synchronize()
            while preparing and preparing[0].event.query():
                pr = preparing.popleft()
                if withdrawn(pr.req.rid, time.perf_counter() - t0):
                    cancelled.add(pr.req.rid)
                    self.in_use -= pr.bytes
                    self.pool.release(pr.req)
                    continue
                lv = self.admit(pr, time.perf_counter() - t0)
                lv.tick0 = ticks
                live[pr.req.rid] = lv
            if waiting and not live and not retiring and not preparing and not self._fits(waiting[0]):
                # nothing resident can be evicted any further
                rejected[waiting.popleft().rid] = "does not fit the HBM budget next to the cached meshes"
            peak = max(peak, self.in_use + self.pool.resident_bytes())
            max_live = max(max_live, len(live))
            # non-finite states (status copied after an earlier tick): retire early as failed
            for lane in self.lanes.values():
                if lane.stat_ev is not None and lane.stat_ev.query():
                    bits = lane.stat.numpy()
                    for lv in live.values():
                        # a slot's word is reset at admission: only instances admitted
                        # before the copied tick are described by it
                        if lv.lane is lane and lv.tick0 < lane.stat_tick and bits[lv.slot] & 2:
                            lv.failed = True
                    lane.stat_ev = None
            if live:
                # one tick: K steps of both batches (concurrent streams)
                for lane in self.lanes.values():
                    if lane.live:
                        lane.batch.run(self.tick)
                for rid, lv in list(live.items()):
                    Nq = lv.req.N + 1
                    dofs = nstate(lv.req.dim) * (lv.req.n_side ** lv.req.dim) * Nq ** lv.req.dim
                    done, target = lv.lane.batch.info(lv.slot)
                    dof_stage += 5 * dofs * (lv.left - (target - done))
                    lv.left = target - done
                    if lv.left <= 0 or lv.failed:
                        if lv.failed:
                            failed.add(rid)
                        else:
                            work[rid] = 5.0 * dofs * lv.nsteps
                        retiring.append(self._retire(lv))
                        del live[rid]
                ticks += 1
                for lane in self.lanes.values():
                    if lane.stat_ev is None and lane.live:
                        lane.batch.status_async(lane.stat)
                        lane.stat_ev = torch.cuda.Event()
                        lane.stat_ev.record(lane.stream)
                        lane.stat_tick = ticks
                    tick_done(lane.stream)
            elif reqs and realtime:
                time.sleep(max(0.0, min(reqs[0].arrival - (time.perf_counter() - t0), 0.002)))
            for item in list(retiring):
                ev, lv, host = item
                if ev.query():
                    if host is not None:
                        lat[lv.req.rid] = base.elapsed_time(ev) * 1e-3 - (lv.req.arrival if realtime else 0.0)
                        results[lv.req.rid] = host.numpy().reshape(
                            (lv.req.n_side ** lv.req.dim, nstate(lv.req.dim), (lv.req.N + 1) ** lv.req.dim)
                        ).transpose(2, 1, 0) + lv.offset[None, :, None]
                        if not np.all(np.isfinite(results[lv.req.rid])):
                            failed.add(lv.req.rid)
                            work.pop(lv.req.rid, None)
                    self.in_use -= lv.bytes
                    self.pool.release(lv.req)
                    retiring.remove(item)
            if not live and retiring:
                retiring[0][0].synchronize()
        torch.cuda.synchronize(self.device)
        arrival = {r.rid: (r.arrival if realtime else 0.0) for r in requests}
        first = min(arrival.values()) if arrival else 0.0
        last = max((lat[k] + arrival[k] for k in lat), default=first)
        return Report(lat, results, first, last, dof_stage, peak, max_live, failed, kinds, rejected, cancelled,
                      work)

    def _retire(self, lv: _Live, copy=True):
        """Release the instance's slot; with `copy`, read its final state back
        to pinned host memory (stream-ordered)."""
        torch = self.torch
        lv.lane.batch.release(lv.slot)  # places the final state in lv.Q (stream-ordered)
        lv.lane.live -= 1
        stream = lv.lane.stream
        host = None
        if copy:
            host = torch.empty(lv.Q.numel(), dtype=torch.float64, pin_memory=True)
            with torch.cuda.stream(stream):
                host.copy_(lv.Q, non_blocking=True) if lv.Q.dtype == torch.float64 else \
                    host.copy_(lv.Q.double(), non_blocking=True)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        return (ev, lv, host)

    def close(self):
        for lane in self.lanes.values():
            lane.batch.close()
        for m in self.pool.meshes.values():
            for bm in m.batch.values():
                bm.close()
        self.pool.meshes.clear()


def serve_one_at_a_time(requests, precision=64, device="cuda"):
    """The same requests through the plain single-mesh path, one solve at a
    time in arrival order (FP64 fused LSRK driver; viscous requests through
    its LDG form), on the same device clock.  Returns a Report."""
    torch = _torch()
    dev = torch.device(device)
    stream = torch.cuda.Stream(dev)
    pool = MeshPool(dev, stream)
    lat, results, failed, work = {}, {}, set(), {}
    dof_stage = 0.0
    real = torch.float64 if precision == 64 else torch.float32
    base = torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    base.record(stream)
    t0 = time.perf_counter()
    for r in sorted(requests, key=lambda q: (q.arrival, q.rid)):
        while time.perf_counter() - t0 < r.arrival:
            time.sleep(min(0.002, r.arrival - (time.perf_counter() - t0)))
        m = pool.get(r, precision, batch=False)
        x = m.dmesh.coords()
        with torch.cuda.stream(stream):
            if r.kind == "vortex":
                f = ic.isentropic_vortex_t(x[0], x[1], r.beta, r.xc, r.yc)
            else:
                f = ic.fourier_state_t(x[0], x[1], x[2], seed=r.seed, vel_peak=r.vel_peak)
            speed = float(wave_speed(f, r.dim).item())
            Q = ic.device_state(list(f), real)
            rhs = torch.zeros_like(Q)
        nsteps, dt = plan(r, speed)
        s = LSRK(m.dmesh, Q, rhs, precision, make_phys(visc=VISC) if r.kind == "ns3d" else make_phys(),
                 stream=stream)
        s.run(nsteps, dt)
        host = torch.empty(Q.numel(), dtype=torch.float64, pin_memory=True)
        with torch.cuda.stream(stream):
            host.copy_(Q.double(), non_blocking=True)
        ev = torch.cuda.Event(enable_timing=True)
        ev.record(stream)
        ev.synchronize()
        s.close()
        lat[r.rid] = base.elapsed_time(ev) * 1e-3 - r.arrival
        results[r.rid] = host.numpy().reshape((r.n_side ** r.dim, nstate(r.dim), (r.N + 1) ** r.dim)).transpose(2, 1, 0)
        w = 5.0 * nstate(r.dim) * (r.n_side ** r.dim) * (r.N + 1) ** r.dim * nsteps
        if not np.all(np.isfinite(results[r.rid])):
            failed.add(r.rid)
        else:
            work[r.rid] = w
        dof_stage += w
        pool.release(r)
    first = min(r.arrival for r in requests)
    last = max(lat[r.rid] + r.arrival for r in requests)
    for m in pool.meshes.values():
        for bm in m.batch.values():
            bm.close()
    return Report(lat, results, first, last, dof_stage, 0, 1, failed, {r.rid: r.kind for r in requests},
                  work=work)


def benchmark(count=2000, seed=0, precision=32, hbm_budget=120e9, tick_steps=8, load=0.8,
              baseline_count=100, device="cuda"):
    """The served stream: (1) capacity = solves/s of the closed loop with all
    `count` requests present at t = 0; (2) the same requests arriving as a
    Poisson stream at `load` x capacity, served in real time (p50/p99 latency,
    solves/s); (3) the first `baseline_count` of them one at a time through
    the plain FP64 path, and the same subset through the server, on the same
    arrival times."""
    out = {"requests": count, "seed": seed, "precision": precision, "hbm_budget_bytes": int(hbm_budget),
           "tick_steps": tick_steps, "load": load,
           "note": "rates and percentiles count completed requests only (finite final state at t_final); "
                   "failed, rejected and cancelled requests are counted separately"}
    # the normalised 3-D mix (velocity sums scaled to peak 0.1, every request
    # completes) in full, and the literal one (its 3-D requests turn
    # non-finite before t_final and are retired as failed) beside it
    for name, vel_peak, full in (("normalised_3d", 0.1, True), ("literal", None, False)):
        cap_reqs = request_stream(count, 0.0, seed, vel_peak=vel_peak)
        srv = Server(precision, hbm_budget, tick_steps=tick_steps, device=device)
        cap = srv.serve(cap_reqs, realtime=False).summary()
        srv.close()
        rate = load * (cap["solves_per_s"] or 0.0)  # completed solves only (0: all arrive at once)
        reqs = request_stream(count, rate, seed, vel_peak=vel_peak)
        srv = Server(precision, hbm_budget, tick_steps=tick_steps, device=device)
        served = srv.serve(reqs, realtime=True)
        srv.close()
        sec = {"vel_peak": vel_peak, "mix": {k: sum(1 for r in reqs if r.kind == k) for k in KINDS},
               "capacity": cap, "rate_per_s": rate, "served": served.summary()}
        if full:
            sub = reqs[:baseline_count]
            srv = Server(precision, hbm_budget, tick_steps=tick_steps, device=device)
            sub_served = srv.serve(sub, realtime=True).summary()
            srv.close()
            seq = serve_one_at_a_time(sub, 64, device).summary()
            sec["subset"] = {"requests": len(sub), "served": sub_served, "one_at_a_time_fp64": seq}
        out[name] = sec
    return out


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="served stream of DG solve requests")
    ap.add_argument("--requests", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--precision", type=int, default=32, choices=[32, 64])
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--tick", type=int, default=8)
    ap.add_argument("--load", type=float, default=0.8)
    ap.add_argument("--baseline", type=int, default=100)
    a = ap.parse_args(argv)
    out = benchmark(a.requests, a.seed, a.precision, a.budget_gb * 1e9, a.tick, a.load, a.baseline)
    print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
