"""Batched LSRK(5,4) over many independent DG instances (cb_mesh_* and
cb_batch_* of include/canary_b200.h).

The reference advances one mesh per `lowstorageRK` call
(euler2d_set3c.jl:1109-1282, euler3d_set3c.jl:1361-1523); a `Batch` advances
many instances of uneven order and size in one graph launch per step, each
with its own dt, step count and state, and admits and releases instances
between runs (continuous batching).  An instance's result does not depend on
what else is in the batch.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check
from .dg import DeviceMesh, _ptr, _stream, _torch, from_device, make_phys, nstate, to_device

MAX_ORDER = {2: 8, 3: 7}  # orders compiled into the batched stage
# stage variants of one (dim, N): 0 = pipelined bulk-copy staging (where the
# slabs are 16-byte multiples), 1 / 2 = grouped stage with ~256 / ~512 nodes
# per block, 3 / 4 = pipelined staging compiled for 3 / 4 resident blocks per
# SM (blocks of up to 256 threads), 6 = pipelined staging with copies two
# element groups ahead, 7 = pipelined staging with twice the elements per
# group on 512-thread blocks, 8 = pipelined staging with two nodes per thread;
# 5 / 9 = the affine-element stage (copies two groups ahead) with one / two
# nodes per thread, for meshes whose elements are all affine; 10 = the
# tensor-core stage (3-D N = 7); 11 = the lean pipelined stage (only the state
# staged in shared memory, geometry and carry read from L2)
VARIANTS = (0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11)
PIPELINED = (0, 3, 4, 6, 7, 8, 11)  # per-node geometry, bit-identical among themselves
AFFINE = (5, 9)  # affine-element geometry, bit-identical among themselves
VAR_AFFINE = 5
VAR_DEEP = 6
VAR_WIDE = 7
VAR_NPT2 = 8
VAR_AFFINE_NPT2 = 9
VAR_MMA = 10
VAR_LEAN = 11


class BatchMesh:
    """Geometry and face-neighbour table shared by all batch instances on one
    mesh (cb_mesh): the FP64 device arrays of `dmesh` for precision 64, rounded
    FP32 copies for precision 32.  Keep it alive while instances use it."""

    def __init__(self, dmesh: DeviceMesh, precision: int = 64, stream=None):
        torch = _torch()
        m = dmesh.mesh
        self.dmesh, self.precision = dmesh, precision
        self.dim, self.N, self.nelem = m.dim, m.N, m.nelem
        self._h = C.c_void_p()
        check(_lib.lib().cb_mesh_create(
            C.byref(self._h), m.dim, m.N, precision, m.nelem, _ptr(dmesh.vgeo, torch.float64),
            _ptr(dmesh.sgeo, torch.float64), _ptr(dmesh.vmapM, torch.int64), _ptr(dmesh.vmapP, torch.int64),
            _ptr(dmesh.elemtobndy, torch.int64), _ptr(dmesh.D, torch.float64), _stream(stream)))

    @property
    def Np(self) -> int:
        return (self.N + 1) ** self.dim

    @property
    def affine(self) -> bool:
        """Whether every element is affine (the batch then uses the
        affine-element stage for it, see Batch.set_affine)."""
        v = C.c_int(0)
        check(_lib.lib().cb_mesh_affine(self._h, C.byref(v)))
        return bool(v.value)

    def close(self) -> None:
        if self._h:
            _lib.lib().cb_mesh_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """A batch of up to `max_instances` slots (cb_batch).  All work is ordered
    on `stream` (the current torch stream by default)."""

    def __init__(self, precision: int = 64, max_instances: int = 1024, phys=None, stream=None):
        self.precision = precision
        self.max_instances = max_instances
        self.phys = phys or make_phys()
        self._h = C.c_void_p()
        check(_lib.lib().cb_batch_create(C.byref(self._h), precision, max_instances, C.byref(self.phys),
                                         _stream(stream)))
        self._inst = {}  # slot -> (mesh, Q, rhs, offset)

    def variant(self, dim: int, N: int) -> int:
        """Stage variant used for instances of (dim, N) admitted from now on."""
        v = C.c_int(-1)
        check(_lib.lib().cb_batch_get_variant(self._h, dim, N, C.byref(v)))
        return v.value

    def variant_info(self, dim: int, N: int, variant: int) -> dict:
        """Launch configuration of a stage variant: elements per CTA, threads
        per CTA, nodes per thread, element groups staged ahead (0: grouped
        staging), resident CTAs per SM, shared memory per CTA."""
        a = (C.c_int64 * 6)()
        check(_lib.lib().cb_batch_variant_info(self._h, dim, N, variant, a))
        return {"elements_per_cta": a[0], "threads_per_cta": a[1], "nodes_per_thread": a[2],
                "staging_depth": a[3], "ctas_per_sm": a[4], "smem_per_cta": a[5]}

    def set_variant(self, dim: int, N: int, variant: int) -> None:
        """Stage variant for instances of (dim, N) admitted from now on
        (VARIANTS); raises CanaryError for a variant not built for it.  A
        chosen variant runs as chosen (an affine one only on meshes that
        allow it, the shape's default per-node variant elsewhere); without a
        choice the batch runs VAR_AFFINE where the affine stage applies."""
        check(_lib.lib().cb_batch_set_variant(self._h, dim, N, variant))

    def set_affine(self, on: bool) -> None:
        """Whether instances admitted from now on may use the affine-element
        stage where it applies (affine mesh, gravity 0; on by default for
        precision 32, off for 64): it reads one geometry record per element
        instead of the per-node metric and face geometry, and agrees with
        them to round-off."""
        check(_lib.lib().cb_batch_set_affine(self._h, 1 if on else 0))

    def set_concurrent(self, on: bool) -> None:
        """Step-graph order of the shapes present: True (default) = one chain
        per shape, the chains concurrent; False = every RK stage of every
        shape in turn, each stage kernel with the whole GPU.  Results do not
        depend on it."""
        check(_lib.lib().cb_batch_set_concurrent(self._h, 1 if on else 0))

    def add(self, mesh: BatchMesh, Q, rhs, dt: float, nsteps: int, qref=None) -> int:
        """Admit the caller's device state Q and zeroed carry rhs (flat tensors
        of the batch precision); returns the slot."""
        torch = _torch()
        real = torch.float64 if self.precision == 64 else torch.float32
        n = mesh.nelem * mesh.Np * nstate(mesh.dim)
        ns = nstate(mesh.dim)
        off = np.zeros(ns) if qref is None else np.asarray(qref, dtype=np.float64)[:ns]
        arr = (C.c_double * 5)(*([float(v) for v in off] + [0.0] * (5 - ns)))
        slot = C.c_int(-1)
        check(_lib.lib().cb_batch_add(self._h, mesh._h, _ptr(Q, real, n, "Q"), _ptr(rhs, real, n, "rhs"),
                                      float(dt), int(nsteps), arr, C.byref(slot)))
        self._inst[slot.value] = (mesh, Q, rhs, off)
        return slot.value

    def add_state(self, mesh: BatchMesh, Q: np.ndarray, dt: float, nsteps: int, offset=None) -> int:
        """Admit a host state Q (Np, nstate, nelem).  For precision 32 the
        device state holds Q - qref with qref = per-field mean of Q (unless
        `offset` is given); `result` returns the full FP64 state."""
        torch = _torch()
        Q = np.asarray(Q, dtype=np.float64)
        if offset is None:
            offset = Q.mean(axis=(0, 2)) if self.precision == 32 else np.zeros(Q.shape[1])
        offset = np.asarray(offset, dtype=np.float64)
        real = torch.float64 if self.precision == 64 else torch.float32
        dQ = to_device(Q - offset[None, :, None], real, mesh.dmesh.vgeo.device)
        return self.add(mesh, dQ, torch.zeros_like(dQ), dt, nsteps, offset)

    def run(self, nsteps: int) -> None:
        """Advance every admitted instance by nsteps steps (each stops at its
        own step count)."""
        check(_lib.lib().cb_batch_run(self._h, int(nsteps)))

    def info(self, slot: int) -> tuple[int, int]:
        """(steps taken, steps to take) of a slot."""
        done, target = C.c_int64(), C.c_int64()
        check(_lib.lib().cb_batch_info(self._h, slot, C.byref(done), C.byref(target)))
        return done.value, target.value

    def slot_variant(self, slot: int) -> int:
        """Stage variant the slot runs with (VAR_AFFINE: the affine-element
        stage)."""
        v = C.c_int(-1)
        check(_lib.lib().cb_batch_slot_variant(self._h, slot, C.byref(v)))
        return v.value

    def release(self, slot: int):
        """Retire a slot; its final state is placed in the caller's Q.
        Returns (Q, rhs) tensors."""
        check(_lib.lib().cb_batch_release(self._h, slot))
        mesh, Q, rhs, off = self._inst.pop(slot)
        return Q, rhs

    def result(self, slot: int) -> np.ndarray:
        """Retire a slot admitted by `add_state` and return its full FP64
        state (Np, nstate, nelem) on the host."""
        mesh, _, _, off = self._inst[slot]
        Q, _ = self.release(slot)
        shape = (mesh.Np, nstate(mesh.dim), mesh.nelem)
        return from_device(Q.double(), shape) + off[None, :, None]

    def status(self) -> np.ndarray:
        """Per-slot sticky status bits (bit 2: non-finite state); synchronises."""
        out = (C.c_uint * self.max_instances)()
        check(_lib.lib().cb_batch_status(self._h, out))
        return np.array(out[:], dtype=np.uint32)

    def status_async(self, host) -> None:
        """Enqueue a copy of the per-slot status bits into `host` (a pinned
        int32 tensor of max_instances entries) on the batch stream."""
        check(_lib.lib().cb_batch_status_async(self._h, C.c_void_p(host.data_ptr())))

    def close(self) -> None:
        if self._h:
            _lib.lib().cb_batch_destroy(self._h)
            self._h = C.c_void_p()
            self._inst.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ------------------------------------------------------------------ ensembles
class MeshCache:
    """Host meshes, device geometry and batch meshes shared by all instances
    with the same (dim, N, n_side) (the geometry does not depend on the
    initial state)."""

    def __init__(self, device="cuda"):
        self.device = device
        self._host, self._dev, self._batch = {}, {}, {}

    def host(self, dim: int, N: int, n_side: int, L: float = 10.0, warp=None):
        from .dg import build_mesh
        key = (dim, N, n_side, L, warp is not None)
        if key not in self._host:
            x = (np.linspace(0.0, L, n_side + 1),) * dim
            self._host[key] = build_mesh(dim, N, x, (True,) * dim, meshwarp=warp)
        return self._host[key]

    def batch_mesh(self, precision: int, dim: int, N: int, n_side: int, L: float = 10.0, warp=None):
        key = (precision, dim, N, n_side, L, warp is not None)
        if key not in self._batch:
            hkey = key[1:]
            if hkey not in self._dev:
                self._dev[hkey] = DeviceMesh.upload(self.host(dim, N, n_side, L, warp), self.device)
            self._batch[key] = BatchMesh(self._dev[hkey], precision)
        return self._batch[key]

    def close(self) -> None:
        for bm in self._batch.values():
            bm.close()
        self._batch.clear()
        self._dev.clear()


def vortex_state(mesh, beta: float, xc: float, yc: float) -> np.ndarray:
    """Conserved (U, V, ρ, E) of the isentropic vortex on a 2-D mesh."""
    from .ic import isentropic_vortex
    x, y = mesh.coords()
    U, V, rho, E = isentropic_vortex(x, y, beta, xc, yc)
    Q = np.empty((mesh.Np, 4, mesh.nelem), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3] = U, V, rho, E
    return Q


class VortexEnsemble:
    """Independent 2-D isentropic-vortex instances (parameters from
    ic.vortex_ensemble) advancing together in one Batch.  For precision 32
    each instance stores its deviation from the free stream (U, V, ρ, E) =
    (1, 0, 1, 1/(γ-1) + 1/2)."""

    FREE_STREAM = (1.0, 0.0, 1.0, 1.0 / 0.4 + 0.5)

    def __init__(self, params, precision=64, dt=0.002, nsteps=500, phys=None, tuning=None, cache=None):
        self.params, self.precision, self.dt, self.nsteps = list(params), precision, dt, nsteps
        self.cache = cache or MeshCache()
        self.batch = Batch(precision, max_instances=max(len(self.params), 1), phys=phys)
        for (dim, N), v in (tuning or {}).items():
            self.batch.set_variant(dim, N, v)
        off = np.array(self.FREE_STREAM) if precision == 32 else np.zeros(4)
        self.slots = []
        self.nodes = 0
        for p in self.params:
            bm = self.cache.batch_mesh(precision, 2, p["N"], p["n_side"])
            Q = vortex_state(self.cache.host(2, p["N"], p["n_side"]), p["beta"], p["xc"], p["yc"])
            self.slots.append(self.batch.add_state(bm, Q, dt, nsteps, off))
            self.nodes += bm.Np * bm.nelem

    @property
    def dof(self) -> int:
        return 4 * self.nodes

    def variants(self) -> dict:
        """Stage variant used per (dim, N) present."""
        return {(2, p["N"]): self.batch.variant(2, p["N"]) for p in self.params}

    def run(self, nsteps=None) -> None:
        self.batch.run(self.nsteps if nsteps is None else nsteps)

    def results(self):
        """Retire every instance; final FP64 host states in parameter order."""
        return [self.batch.result(s) for s in self.slots]

    def close(self) -> None:
        self.batch.close()


# ------------------------------------------------------------------ autotuner
def _time_variants(precision, dim, N, meshes, steps, repeat, affine):
    """Step time of each stage variant of (dim, N) on the given instances
    (pairs of a BatchMesh and a device state factory), all admitted to one
    batch; {variant: ms per step} over the variants built for the shape (the
    affine ones only when `affine`: every mesh affine and the affine stage
    allowed)."""
    torch = _torch()
    timings = {}
    for var in VARIANTS:
        if var in AFFINE and not affine:
            continue
        b = Batch(precision, max(len(meshes), 1))
        try:
            b.set_variant(dim, N, var)  # a chosen variant runs as chosen
        except Exception:
            b.close()
            continue
        b.set_affine(var in AFFINE)
        slots = []
        for bm, make, dt in meshes:
            Q = make()
            slots.append(b.add(bm, Q, torch.zeros_like(Q), dt, 10 ** 9))
        b.run(1)  # build the graph, warm up
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ts = []
        for _ in range(repeat):
            torch.cuda.synchronize()
            ev0.record()
            b.run(steps)
            ev1.record()
            torch.cuda.synchronize()
            ts.append(ev0.elapsed_time(ev1) / steps)
        timings[var] = min(ts)
        for s in slots:
            b.release(s)
        b.close()
    return timings


def tuning_picks(instances, dim: int, N: int, nodes_target: int):
    """The instances the tuner times for (dim, N): the workload's own
    (n_side of each (dim, N, n_side) entry of that shape), in order, up to
    about `nodes_target` nodes, then the same ones again in order while they
    hold fewer.  Returns (n_side list, distinct workload instances, nodes)."""
    picks, nodes = [], 0
    for d, n, ns in instances:
        if (d, n) == (dim, N) and nodes < nodes_target:
            picks.append(ns)
            nodes += ns ** dim * (N + 1) ** dim
    distinct = len(picks)
    k = 0
    while picks and nodes < nodes_target:  # the same instances again, in order
        ns = picks[k % distinct]
        picks.append(ns)
        nodes += ns ** dim * (N + 1) ** dim
        k += 1
    return picks, distinct, nodes


def autotune(precision: int, shapes, nodes_target: int = 8_000_000, steps: int = 4, repeat: int = 3,
             stream=None, instances=None, report=None, affine=None) -> dict:
    """Choose the stage variant of each (dim, N) — pipelined staging at one of
    several occupancies, two element groups ahead, twice the elements per
    group or two nodes per thread, per-node or (affine meshes, `affine`:
    default on for precision 32 as in Batch) affine-element geometry, or
    grouped staging with about 256 / 512 nodes per block, i.e. elements per
    CTA, threads and nodes per thread, and staging depth — by timing the
    batched step.

    With `instances` (the workload's (dim, N, n_side) list) each shape is
    timed on the workload's own instances of that shape, taken in order up to
    about `nodes_target` nodes (its actual size mix) and repeated in the same
    order while they hold fewer — so that the timed state does not stay in
    L2 between stages, as it does not in the whole workload; otherwise on one
    synthetic instance of about `nodes_target` nodes: the 2-D vortex / the
    3-D Fourier state on periodic meshes built on the device.  Returns
    {(dim, N): variant}; `report` (a dict) receives, per shape, the timings
    and the chosen variant's launch configuration."""
    torch = _torch()
    from . import ic
    if affine is None:
        affine = precision == 32
    best = {}
    if instances is not None:
        for dim, N in shapes:
            L = 10.0 if dim == 2 else 2 * np.pi
            picks, distinct, nodes = tuning_picks(instances, dim, N, nodes_target)
            dms = {}
            meshes = []
            real = torch.float64 if precision == 64 else torch.float32
            for ns in picks:
                if ns not in dms:
                    dm = DeviceMesh.build(dim, N, (np.linspace(0.0, L, ns + 1),) * dim, (True,) * dim)
                    dms[ns] = (dm, BatchMesh(dm, precision))
                dm, bm = dms[ns]
                X = dm.coords()
                if dim == 2:
                    make = (lambda X=X: ic.device_state(list(ic.isentropic_vortex_t(X[0], X[1], 5.0, 5.0, 5.0)), real))
                    dt = 1e-4
                else:
                    make = (lambda X=X: ic.device_state(list(ic.fourier_state_t(X[0], X[1], X[2], seed=0)), real))
                    dt = 1e-5
                meshes.append((bm, make, dt))
            aff = affine and all(bm.affine for bm, _, _ in meshes)
            timings = _time_variants(precision, dim, N, meshes, steps, repeat, aff)
            for dm, bm in dms.values():
                bm.close()
            best[(dim, N)] = min(timings, key=timings.get)
            if report is not None:
                info = Batch(precision, 1)
                report[(dim, N)] = {"variant": best[(dim, N)], "instances": distinct, "admitted": len(picks),
                                    "nodes": nodes,
                                    "ms_per_step": timings,
                                    "config": info.variant_info(dim, N, best[(dim, N)])}
                info.close()
        return best
    for dim, N in shapes:
        Np = (N + 1) ** dim
        n_side = max(2, int(round((nodes_target / Np) ** (1.0 / dim))))
        L = 10.0 if dim == 2 else 2 * np.pi
        dm = DeviceMesh.build(dim, N, (np.linspace(0.0, L, n_side + 1),) * dim, (True,) * dim)
        X = dm.coords()
        if dim == 2:
            f = ic.isentropic_vortex_t(X[0], X[1], 5.0, 5.0, 5.0)
            dt = 1e-4
        else:
            f = ic.fourier_state_t(X[0], X[1], X[2], seed=0)
            dt = 1e-5
        real = torch.float64 if precision == 64 else torch.float32
        bm = BatchMesh(dm, precision)
        aff = affine and bm.affine
        timings = {}
        for var in VARIANTS:
            if var in AFFINE and not aff:
                continue
            b = Batch(precision, 1)
            try:
                b.set_variant(dim, N, var)
            except Exception:
                b.close()
                continue
            b.set_affine(var in AFFINE)
            Q = ic.device_state(list(f), real)
            slot = b.add(bm, Q, torch.zeros_like(Q), dt, 10 ** 9)
            b.run(1)  # build the graph, warm up
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ts = []
            for _ in range(repeat):
                torch.cuda.synchronize()
                ev0.record()
                b.run(steps)
                ev1.record()
                torch.cuda.synchronize()
                ts.append(ev0.elapsed_time(ev1) / steps)
            timings[var] = min(ts)
            b.release(slot)
            b.close()
        bm.close()
        best[(dim, N)] = min(timings, key=timings.get)
        if report is not None:
            info = Batch(precision, 1)
            report[(dim, N)] = {"variant": best[(dim, N)], "instances": 1, "admitted": 1,
                                "nodes": bm.Np * bm.nelem, "ms_per_step": timings,
                                "config": info.variant_info(dim, N, best[(dim, N)])}
            info.close()
    return best
