#!/usr/bin/env python
"""Throughput of the nodal-DG hot path (volume + Rusanov face + LSRK(5,4)
update) in DOF·stage updates per second.

Default workload: 3-D compressible Euler on the periodic cube [0,2π]^3,
32^3 hexes at N=7 (16.8 M nodes, 83.9 M DOF), coordinates warped by
x_i += 0.05 sin x sin y sin z, seeded random Fourier initial state (p = 1),
dt = 0.2 h / (N^2 max(|u|+c)), FP64.  One "step" is one LSRK(5,4) step
(5 fused stage launches) over the whole mesh.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--precision 64|32] [--n-side 32] [--order 7]

Under torchrun each rank advances its own copy of the workload (independent
replicas, "weak" scaling); the timed region is bracketed by a barrier and a
device synchronisation and the slowest rank's time is reported.
`--impl reference` times the CPU restatement of the reference's CPU path on
the host cores instead (rank 0 only), on the same workload.

After the timed region (one GPU) the line also carries:
  * e2e: the same steps through the public API with the state uploaded from
    and read back to pinned host memory every step;
  * parity.timed_workload: the timed workload advanced by 200 steps on the GPU and
    by the oracle from the same device-built mesh and state (bar 1e-12); the
    oracle's timing on all host cores is the cpu_baseline;
  * fp32_form: the timed workload in the FP32 form, timed the same way;
  * precision_form: FP32 against FP64 at 32^3, N = 4, 7, 10, 1000 steps, the
    LDG Navier-Stokes variant and the 2-D vortex (bar 1e-5);
  * batched: 512 vortex instances in one batch per precision, with a roofline
    and 16 instances checked against the oracle;
  * served: the served request stream.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "canary.jl_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "DOF·stage updates/s"


def bytes_per_node(dim, N, w):
    """Algorithmic HBM bytes per node and stage: Q read+write, residual carry
    read+write, metric (dim² terms, MJ, MJI) and the face normals + sMJ
    spread over the nodes (2·dim/Nq face nodes per node)."""
    ns = 5 if dim == 3 else 4
    return w * (4 * ns + (dim * dim + 2) + (2.0 * dim / (N + 1)) * (dim + 1))


L2_BYTES = 126e6
STAGE_KERNELS = {1: "k_stage_pipe2", 2: "k_stage_mma", 3: "k_stage", 4: "k_stage_lean"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_traffic(key):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(key)
    return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    FIELDS = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.proc = None
        self.path = None
        self.skip = 0

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "50",
                                          "-f", self.path],
                                         stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def _lines(self):
        try:
            with open(self.path) as f:
                return sum(1 for _ in f)
        except Exception:
            return 0

    def mark(self):
        """Wait (up to 3 s) until the sampler has written a first sample, then
        remember how many were taken before the timed region."""
        if self.proc is None:
            return
        t = time.time()
        while self._lines() == 0 and time.time() - t < 3.0:
            time.sleep(0.01)
        self.skip = self._lines()

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        try:
            with open(self.path) as f:
                for line in f:
                    parts = [p.strip() for p in line.split(",")]
                    if len(parts) < 9:
                        continue
                    if self.uuid and self.uuid not in parts[0]:
                        continue
                    rows.append(parts)
            os.unlink(self.path)
        except Exception:
            return None
        if not rows:
            return None
        # samples taken during (and just after) the timed region; the last one
        # if the region was shorter than the sampling interval
        rows = rows[self.skip:] if len(rows) > self.skip else rows[-1:]
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v.lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


def setup_workload(n_side, N, device="cuda", seed=0):
    from canary_b200 import dg, ic
    from canary_b200.metric import warp_sinusoidal
    L = 2 * math.pi
    mesh = dg.build_mesh(3, N, (np.linspace(0.0, L, n_side + 1),) * 3, (True,) * 3,
                         meshwarp=lambda X: warp_sinusoidal(X, 0.05))
    x, y, z = mesh.coords()
    U, V, W, rho, E = ic.fourier_state(x, y, z, seed=seed, device=device)
    Q = np.zeros((mesh.Np, 5, mesh.nelem), order="F")
    Q[:, 0], Q[:, 1], Q[:, 2], Q[:, 3], Q[:, 4] = U, V, W, rho, E
    dt = ic.fourier_dt(Q, N, h=L / n_side)
    return mesh, Q, dt


def setup_device_workload(n_side, N, precision, device="cuda", seed=0):
    """The same workload built on the device: connectivity on the host, grid,
    warp and geometry by cb_computegeometry, the Fourier state by torch.
    Returns (DeviceMesh, Q, rhs, dt, offset) with Q, rhs in the working
    precision (for FP32 Q holds the state minus its per-field mean)."""
    import torch
    from canary_b200 import dg, ic, serve
    L = 2 * math.pi
    x = (np.linspace(0.0, L, n_side + 1),) * 3
    dm = dg.DeviceMesh.build(3, N, x, (True,) * 3, warp_amp=0.05, device=device)
    f = ic.fourier_state_t(*dm.coords(), seed=seed)
    dt = 0.2 * (L / n_side) / (N * N * float(serve.wave_speed(f, 3).item()))
    off = np.array([float(t.mean().item()) for t in f]) if precision == 32 else np.zeros(5)
    real = torch.float64 if precision == 64 else torch.float32
    Q = ic.device_state(list(f), real, off)
    return dm, Q, torch.zeros_like(Q), dt, off


def _oracle_rate(N, seconds, n_side, max_steps, cores):
    """DOF·stage/s of the oracle on an n_side^3 sample of the workload with
    `cores` OpenMP threads, LSRK steps until `seconds` elapse; (rate, steps,
    seconds)."""
    from canary_b200 import dg
    from oracle import pyoracle as O
    mesh, Q, dt = setup_workload(n_side, N, device=None)
    wp = dict(dg.WORKLOAD_PHYS)
    wp["lambda"] = wp.pop("lam")
    phys = O.make_phys(**wp)
    rhs = np.zeros_like(Q, order="F")
    O.lowstorageRK(3, N, mesh.vgeo, mesh.sgeo, Q, rhs, mesh.D, dt, 1, mesh.vmapM, mesh.vmapP,
                   mesh.elemtobndy, phys, cores)  # warm-up
    t0 = time.perf_counter()
    steps = 0
    while steps < max_steps and (time.perf_counter() - t0) < seconds:
        O.lowstorageRK(3, N, mesh.vgeo, mesh.sgeo, Q, rhs, mesh.D, dt, 1, mesh.vmapM, mesh.vmapP,
                       mesh.elemtobndy, phys, cores)
        steps += 1
    el = time.perf_counter() - t0
    return mesh.nelem * mesh.Np * 5 * 5 * steps / el, steps, el


def cpu_sample(N, seconds=10.0, n_side=16, max_steps=40):
    """Oracle (CPU restatement of the reference's CPU path) on a bounded
    sample of the workload: same N, warp and initial-state law on an
    n_side^3 mesh, all host threads, LSRK steps until `seconds` elapse; and,
    mirroring the reference's single-threaded Julia loop, one thread on an
    8^3 sample."""
    cores = os.cpu_count() or 1
    rate, steps, el = _oracle_rate(N, seconds, n_side, max_steps, cores)
    r1, s1, e1 = _oracle_rate(N, seconds / 2, 8, 4, 1)
    return {"value": rate, "unit": METRIC, "cores": cores, "kind": "port",
            "sample": f"{n_side}^3 hexes N={N} (same warp/IC law), {steps} LSRK steps "
                      f"({5 * steps} stages) in {el:.1f} s, C oracle with {cores} OpenMP threads",
            "single_thread": {"value": r1, "unit": METRIC, "cores": 1,
                              "sample": f"8^3 hexes N={N}, {s1} LSRK steps in {e1:.1f} s, one thread"}}


def _oracle_phys():
    from canary_b200 import dg
    from oracle import pyoracle as O
    wp = dict(dg.WORKLOAD_PHYS)
    wp["lambda"] = wp.pop("lam")
    return O.make_phys(**wp)


def _rel_l2(a, b):
    """Relative L2 error per state field (axis 1 of (Np, nstate, nelem))."""
    return [float(np.linalg.norm(a[:, q] - b[:, q]) / np.linalg.norm(b[:, q])) for q in range(b.shape[1])]


class Config1Parity:
    """Full-size parity of the bench workload: the FP64 GPU solver and the
    oracle (the CPU restatement of the reference's lowstorageRK,
    euler3d_set3c.jl:1361-1523) each advance the same initial state on the
    same mesh (the device-built geometry and maps, copied to the host) by the
    stated step count; the relative L2 error per field is compared with 1e-12.
    The oracle runs on all host cores in a background thread (ctypes releases
    the GIL), so the GPU sections that follow overlap it; its timing over the
    whole workload is the CPU baseline."""

    NAMES = ("U", "V", "W", "rho", "E")

    def __init__(self, dm, Q0, dt, steps, stream, threads):
        import torch
        from canary_b200 import dg
        m = dm.mesh
        Nfp = (m.N + 1) ** 2
        self.steps, self.threads, self.dt = steps, threads, dt
        shape = (m.Np, 5, m.nelem)
        q = Q0.clone()
        r = torch.zeros_like(q)
        s = dg.LSRK(dm, q, r, 64, dg.make_phys(), stream)
        s.run(steps, dt)
        torch.cuda.synchronize()
        self.gpu = dg.from_device(q, shape)
        s.close()
        del q, r
        self.m = m
        self.vgeo = dg.from_device(dm.vgeo, (m.Np, 14, m.nelem))
        self.sgeo = dg.from_device(dm.sgeo, (5, Nfp, 6, m.nelem))
        self.vmapM = dg.from_device(dm.vmapM, (Nfp, 6, m.nelem))
        self.vmapP = dg.from_device(dm.vmapP, (Nfp, 6, m.nelem))
        self.etb = dg.from_device(dm.elemtobndy, (6, m.nelem))
        self.Q = np.asfortranarray(dg.from_device(Q0, shape))
        self.out = None
        self.thread = threading.Thread(target=self._oracle, daemon=True)
        self.thread.start()

    def _oracle(self):
        from oracle import pyoracle as O
        rhs = np.zeros_like(self.Q, order="F")
        t0 = time.perf_counter()
        O.lowstorageRK(3, self.m.N, self.vgeo, self.sgeo, self.Q, rhs, self.m.D, self.dt, self.steps,
                       self.vmapM, self.vmapP, self.etb, _oracle_phys(), self.threads)
        self.seconds = time.perf_counter() - t0

    def result(self):
        self.thread.join()
        err = _rel_l2(self.gpu, self.Q)
        dof = self.m.nelem * self.m.Np * 5
        return {
            "workload": "the bench workload (32^3 hexes, N=7, warped, seeded Fourier state) as timed, "
                        "device-built mesh and state copied to the oracle",
            "steps": self.steps, "dt": self.dt, "bar": 1e-12,
            "rel_l2": dict(zip(self.NAMES, err)), "max_rel_l2": max(err), "pass": max(err) <= 1e-12,
            "finite": bool(np.all(np.isfinite(self.gpu))),
            "oracle_seconds": self.seconds, "oracle_threads": self.threads,
            "oracle_value": dof * 5 * self.steps / self.seconds,
        }


def precision_section(steps=1000, orders=(4, 7, 10), n_side=32, ns_n_side=16, device="cuda"):
    """The precision form at full size: FP32 against the FP64 form (itself
    pinned to the oracle) after `steps` steps on the same mesh and initial
    state, inviscid 3-D at n_side^3, the LDG Navier-Stokes variant
    (mu = 1e-3, Pr = 0.72) at ns_n_side^3 and the 2-D vortex."""
    from canary_b200 import precision as P
    cases = []
    for c in P.report(orders, n_side, steps, ns_n_side, device=device):
        cases.append({"dim": c["dim"], "N": c["N"], "n_side": c["n_side"], "visc": c["visc"], "steps": steps,
                      "dt": c["dt"], "rel_l2": c["fp32_rel_l2_vs_fp64"], "max_rel_l2": c["max_rel_l2"],
                      "fp64_dof_stage_per_s": c["fp64"]["dof_stage_per_s"],
                      "fp32_dof_stage_per_s": c["fp32"]["dof_stage_per_s"],
                      "fp32_mass_drift_rel": c["fp32"]["mass_drift_rel"],
                      "finite": c["fp64"]["finite"] and c["fp32"]["finite"]})
    worst = max(c["max_rel_l2"] for c in cases)
    return {"workload": f"warped [0,2π]^3 {n_side}^3 (LDG NS {ns_n_side}^3) and 2-D vortex 10^2, FP32 vs FP64, "
                        f"dt = min(CFL rule, 0.08/steps)",
            "bar": 1e-5, "max_rel_l2": worst, "pass": worst <= 1e-5, "cases": cases}


def ensemble_parity(params, cache, finals, sample=16, steps=500, dt=0.002, threads=None):
    """The first `sample` instances of the batched ensemble through the
    oracle (FP64, `steps` steps from the same host mesh and initial state)
    against the FP64 batch (bar 1e-12) and the FP32 batch (bar 1e-5)."""
    from canary_b200 import batch as B
    from oracle import pyoracle as O
    threads = threads or os.cpu_count() or 1
    e64 = np.zeros(4)
    e32 = np.zeros(4)
    t0 = time.perf_counter()
    for i, p in enumerate(params[:sample]):
        m = cache.host(2, p["N"], p["n_side"])
        Q = B.vortex_state(m, p["beta"], p["xc"], p["yc"])
        rhs = np.zeros_like(Q, order="F")
        O.lowstorageRK(2, p["N"], m.vgeo, m.sgeo, Q, rhs, m.D, dt, steps, m.vmapM, m.vmapP, m.elemtobndy,
                       _oracle_phys(), threads)
        e64 = np.maximum(e64, _rel_l2(finals[64][i], Q))
        e32 = np.maximum(e32, _rel_l2(finals[32][i], Q))
    names = ("U", "V", "rho", "E")
    return {"instances": min(sample, len(params)), "steps": steps,
            "shapes": [(p["N"], p["n_side"]) for p in params[:sample]],
            "fp64_vs_oracle": dict(zip(names, e64.tolist())), "fp64_bar": 1e-12,
            "fp32_vs_oracle": dict(zip(names, e32.tolist())), "fp32_bar": 1e-5,
            "pass": bool(e64.max() <= 1e-12 and e32.max() <= 1e-5),
            "oracle_seconds": time.perf_counter() - t0}


def batched_ensemble(count=512, seed=0, steps=500, device="cuda", parity_sample=16, precisions=(64, 32),
                     tune=True):
    """The batched workload: `count` independent 2-D vortex instances (N, mesh,
    strength and centre drawn per instance from PCG64(seed + i)), dt = 0.002,
    `steps` LSRK(5,4) steps each, advanced together by one Batch per precision
    (one graph launch per step).  Returns throughput, solves/s, the roofline
    of the step, the FP32 form's relative L2 error per field against the FP64
    batch and a sample of instances checked against the oracle."""
    import torch
    from canary_b200 import batch as B, ic
    params = ic.vortex_ensemble(count, seed)
    cache = B.MeshCache(device)
    t0 = time.time()
    for p in params:
        cache.host(2, p["N"], p["n_side"])
    out = {"workload": f"{count} independent 2-D isentropic vortices on [0,10]^2, N~U{{3..8}}, "
                       f"n_side~U{{4..48}}, beta~U(1,5), centre~U([2,8]^2), PCG64(seed+i), dt=0.002, "
                       f"{steps} steps each", "instances": count, "steps": steps,
           "host_mesh_setup_s": round(time.time() - t0, 2)}
    finals = {}
    shapes = sorted({(2, p["N"]) for p in params})
    for prec in precisions:
        t1 = time.time()
        # stage variant per (dim, N), timed on this GPU on the ensemble's own
        # instances of each shape (its size mix); the batch's defaults without it
        rep = {}
        tuning = B.autotune(prec, shapes, instances=[(2, p["N"], p["n_side"]) for p in params],
                            report=rep) if tune else {}
        out[f"autotune_fp{prec}_s"] = round(time.time() - t1, 2)
        out[f"autotune_fp{prec}"] = {f"{d},{n}": {"variant": r["variant"], **r["config"],
                                                   "instances": r["instances"], "admitted": r["admitted"],
                                                   "nodes": r["nodes"],
                                                   "ms_per_step": {str(v): round(t, 4) for v, t in r["ms_per_step"].items()}}
                                     for (d, n), r in rep.items()}
        ens = B.VortexEnsemble(params, prec, nsteps=steps, cache=cache, tuning=tuning)
        torch.cuda.synchronize()
        ens.run(1)  # builds the step graph
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        ens.run(steps - 1)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        st = ens.batch.status()
        # algorithmic HBM bytes of one step: per instance nodes x bytes per
        # node and stage of the stage variant it runs (the affine-element
        # stage reads one geometry record per element instead of the
        # per-node metric and face geometry)
        w = 8 if prec == 64 else 4
        step_bytes = 0.0
        for p, slot in zip(params, ens.slots):
            Np = (p["N"] + 1) ** 2
            nodes = Np * p["n_side"] ** 2
            if ens.batch.slot_variant(slot) in B.AFFINE:
                bpn = w * (4 * 4 + 17.0 / Np)  # state + carry, record of 17 values per element
            else:
                bpn = bytes_per_node(2, p["N"], w)
            step_bytes += 5 * nodes * bpn
        peak, peak_kind = measured_peaks()
        achieved = step_bytes / (ms * 1e-3 / (steps - 1)) / 1e9
        finals[prec] = ens.results()
        out[f"fp{prec}"] = {"value": ens.dof * 5 * (steps - 1) / (ms * 1e-3), "unit": METRIC,
                            "ms_per_step": ms / (steps - 1), "dof": ens.dof,
                            "solves_per_s": count / (ms * 1e-3 * steps / (steps - 1)),
                            "state_finite": not bool(st.any()),
                            "variants": {f"{d},{n}": v for (d, n), v in ens.variants().items()},
                            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                         "frac": achieved / peak, "peak_kind": peak_kind,
                                         "bytes_per_step": step_bytes,
                                         "kernel": "k_stage_pipe2 (one persistent kernel per shape, "
                                                   "five stage launches per step)"}}
        ens.close()
    if 32 in finals and 64 in finals:
        err = np.zeros(4)
        for a, b in zip(finals[32], finals[64]):
            for q in range(4):
                err[q] = max(err[q], np.linalg.norm(a[:, q] - b[:, q]) / np.linalg.norm(b[:, q]))
        out["fp32_rel_l2_vs_fp64_max_over_instances"] = {"U": err[0], "V": err[1], "rho": err[2], "E": err[3]}
        if parity_sample:
            out["parity_vs_oracle"] = ensemble_parity(params, cache, finals, parity_sample, steps)
    cache.close()
    return out


def fp32_form(args, dev, stream):
    """The timed workload in the FP32 form (state stored as its deviation
    from the per-field mean, FP32 arithmetic), args.warmup + args.steps steps
    with CUDA events around args.steps of them; throughput and roofline."""
    import torch
    from canary_b200 import dg
    dm, dQ, drhs, dt, off = setup_device_workload(args.n_side, args.order, 32, device=dev)
    s = dg.LSRK(dm, dQ, drhs, 32, dg.make_phys(), stream)
    s.set_offset(off)
    s.run(args.warmup, dt)
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s.run(args.steps, dt)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    ms = e0.elapsed_time(e1)
    kernel = STAGE_KERNELS[s.kernel]
    finite = bool(np.all(np.isfinite(s.sums())))
    s.close()
    mesh = dm.mesh
    dof = mesh.nelem * mesh.Np * 5
    t_launch = ms * 1e-3 / (5 * args.steps)
    bpn = bytes_per_node(3, args.order, 4)
    peak, peak_kind = measured_peaks()
    achieved = mesh.nelem * mesh.Np * bpn / t_launch / 1e9
    return {"value": dof * 5 * args.steps / (ms * 1e-3), "unit": METRIC, "ms_per_step": ms / args.steps,
            "steps": args.steps, "dtype": "f32", "state_finite": finite,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "bytes_per_node": bpn, "kernel": kernel,
                         "launch_ms": t_launch * 1e3}}


def dist_init():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    if ws <= 1:
        return 0, 1, 0, None
    import datetime
    import torch
    import torch.distributed as tdist
    rank = int(os.environ["RANK"])
    local = int(os.environ.get("LOCAL_RANK", rank))
    torch.cuda.set_device(local)
    tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                             device_id=torch.device("cuda", local))
    return rank, ws, local, tdist


def reference_workload(n_side, N, seed=0):
    """The bench workload built for the CPU path alone: the oracle's
    restatement of the reference's set-up (brickmesh -> partition ->
    connectmesh -> mappings -> computegeometry with the sinusoidal warp) and
    the seeded Fourier state (257 modes, evaluated by torch: on a GPU where
    one is present, else on the host cores; set-up only, never timed)."""
    import torch
    from canary_b200 import ic
    from oracle import pyoracle as O
    L = 2 * math.pi
    S = O.setup(3, N, (np.linspace(0.0, L, n_side + 1),) * 3, (True,) * 3, warp=1, warp_amp=0.05)
    X = [np.ascontiguousarray(S.vgeo[:, 11 + c, :]) for c in range(3)]
    f = ic.fourier_state(*X, seed=seed, device="cuda" if torch.cuda.is_available() else "cpu")
    Q = np.asfortranarray(np.stack(f, axis=1))
    dt = ic.fourier_dt(Q, N, h=L / n_side)
    return S, Q, dt


def run_reference(args, rank):
    """--impl reference: the CPU path on the host cores (rank 0 only), on the
    same workload as the GPU arm."""
    if rank != 0:
        return
    from oracle import pyoracle as O
    O.build()
    n_side = args.ref_n_side or args.n_side
    mesh, Q, dt = reference_workload(n_side, args.order)
    phys = _oracle_phys()
    rhs = np.zeros_like(Q, order="F")
    cores = os.cpu_count() or 1
    for _ in range(args.warmup):
        O.lowstorageRK(3, args.order, mesh.vgeo, mesh.sgeo, Q, rhs, mesh.D, dt, 1, mesh.vmapM,
                       mesh.vmapP, mesh.elemtobndy, phys, cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.lowstorageRK(3, args.order, mesh.vgeo, mesh.sgeo, Q, rhs, mesh.D, dt, 1, mesh.vmapM,
                       mesh.vmapP, mesh.elemtobndy, phys, cores)
    el = time.perf_counter() - t0
    dof = mesh.nelem * (args.order + 1) ** 3 * 5
    val = dof * 5 * args.steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": METRIC,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * el / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"3-D Euler, periodic [0,2π]^3, {n_side}^3 hexes, N={args.order}, "
                               "warped x_i += 0.05 sin x sin y sin z, seeded Fourier state (seed 0)",
                   "n_side": n_side, "order": args.order, "nelem": mesh.nelem, "dof": dof, "dt": dt,
                   "same_config": n_side == args.n_side},
        "cpu_baseline": {"value": val, "unit": METRIC, "cores": cores, "kind": "port",
                         "sample": f"{n_side}^3 hexes, N={args.order}, {args.steps} timed LSRK steps "
                                   f"after {args.warmup} untimed; the reference's Julia CPU path cannot run "
                                   "here (no Julia toolchain), so its C restatement (oracle/) is timed"},
        "e2e": {"value": val, "unit": METRIC, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--precision", type=int, default=64, choices=[64, 32])
    ap.add_argument("--n-side", type=int, default=32)
    ap.add_argument("--order", type=int, default=7)
    ap.add_argument("--stage-kernel", type=int, default=0, choices=[0, 1, 2, 3, 4],
                    help="stage kernel: 0 the shape's default, 1 CUDA-core pipelined, 2 tensor-core "
                         "(3-D N=7), 3 grouped, 4 lean pipelined")
    ap.add_argument("--ref-n-side", type=int, default=None,
                    help="mesh of the reference arm (default: --n-side, the same workload)")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--parity-steps", type=int, default=200,
                    help="steps of the full-size parity run against the oracle (0: skip)")
    ap.add_argument("--precision-steps", type=int, default=1000,
                    help="steps of the precision-form section (0: skip)")
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched-ensemble measurement (run on 1 GPU only)")
    ap.add_argument("--batched-instances", type=int, default=512)
    ap.add_argument("--batched-steps", type=int, default=500)
    ap.add_argument("--batched-precisions", type=int, nargs="+", default=[64, 32], choices=[64, 32])
    ap.add_argument("--no-autotune", action="store_true",
                    help="batched section: the batch's default stage variants instead of the autotuner's")
    ap.add_argument("--no-fp32-form", action="store_true",
                    help="skip the FP32 form of the timed workload (run on 1 GPU, FP64 arm only)")
    ap.add_argument("--no-served", action="store_true",
                    help="skip the served-stream measurement (run on 1 GPU only)")
    ap.add_argument("--served-requests", type=int, default=150)
    ap.add_argument("--served-baseline", type=int, default=30)
    args = ap.parse_args()

    rank, world, local, tdist = dist_init()
    if args.impl == "reference":
        run_reference(args, rank)
        if tdist is not None:
            tdist.destroy_process_group()
        return

    import torch
    from canary_b200 import dg

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    N, dim = args.order, 3
    dm, dQ, drhs, dt, off = setup_device_workload(args.n_side, N, args.precision, device=dev)
    mesh = dm.mesh
    real = torch.float64 if args.precision == 64 else torch.float32
    solver = dg.LSRK(dm, dQ, drhs, args.precision, dg.make_phys(), stream)
    solver.set_offset(off)
    solver.set_kernel(args.stage_kernel)
    kernel_name = STAGE_KERNELS[solver.kernel]
    dof = mesh.nelem * mesh.Np * 5
    dQ0 = dQ.clone()  # initial state, for the parity run

    solver.run(args.warmup, dt)
    torch.cuda.synchronize(dev)
    try:
        uuid = str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        uuid = None
    clocks = ClockSampler(uuid)
    clocks.start()
    clocks.mark()
    if tdist is not None:
        tdist.barrier()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    solver.run(args.steps, dt)
    e1.record(stream)
    torch.cuda.synchronize(dev)
    if tdist is not None:
        tdist.barrier()
    clk = clocks.stop()
    from canary_b200 import replicas
    t_ms = replicas.max_over_ranks(e0.elapsed_time(e1), device=dev)
    sums = solver.sums()
    finite = bool(np.all(np.isfinite(sums)))

    # end to end through the public API with host buffers: every step copies
    # the state from pinned host memory, advances one step and reads the
    # state back (the step's input is the state alone: the 2N-storage carry
    # is zero at a step boundary, scaled by RKA[0] = 0 after the fifth stage).
    # Three device states, each with its own solver on the compute stream, and
    # one copy stream per direction: the upload of step k+1 and the read-back
    # of step k overlap step k's compute and each other, and the upload of
    # step k+3 waits only for the read-back of step k (with two states the
    # cycle upload -> step -> read-back of every second step serialises).
    NB = 3
    hQ = torch.empty(dQ.numel(), dtype=real, pin_memory=True)
    hQ.copy_(dQ)
    hout = [torch.empty_like(hQ, pin_memory=True) for _ in range(NB)]
    dQ2 = [dQ] + [torch.empty_like(dQ) for _ in range(NB - 1)]
    rhs2 = [drhs] + [torch.zeros_like(drhs) for _ in range(NB - 1)]
    solvers = [solver] + [dg.LSRK(dm, dQ2[i], rhs2[i], args.precision, dg.make_phys(), stream) for i in range(1, NB)]
    for sv in solvers[1:]:
        sv.set_offset(off)
        sv.set_kernel(args.stage_kernel)
    up, down = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    torch.cuda.synchronize(dev)
    if tdist is not None:
        tdist.barrier()
    ev = lambda: torch.cuda.Event(enable_timing=False)
    loaded, stepped, stored = [], [], []
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(up)
    for k in range(args.e2e_steps):
        b = k % NB
        if k >= NB:
            up.wait_event(stored[k - NB])  # state buffer b has been read back
        with torch.cuda.stream(up):
            dQ2[b].copy_(hQ, non_blocking=True)
        loaded.append(ev())
        loaded[k].record(up)
        stream.wait_event(loaded[k])
        solvers[b].run(1, dt)
        stepped.append(ev())
        stepped[k].record(stream)
        down.wait_event(stepped[k])
        with torch.cuda.stream(down):
            hout[b].copy_(dQ2[b], non_blocking=True)
        stored.append(ev())
        stored[k].record(down)
    f1.record(down)
    torch.cuda.synchronize(dev)
    e2e_ms = replicas.max_over_ranks(f0.elapsed_time(f1), device=dev)
    e2e_ok = bool(torch.equal(hout[(args.e2e_steps - 1) % NB], hout[(args.e2e_steps - 2) % NB]))
    for sv in solvers:
        sv.close()
    del dQ2, rhs2, hout

    # full-size parity of the timed workload (FP64 form): the oracle runs on
    # the host cores in the background while the precision section uses the GPU
    par = None
    if rank == 0 and world == 1 and args.precision == 64 and args.parity_steps > 0:
        par = Config1Parity(dm, dQ0, dt, args.parity_steps, stream, os.cpu_count() or 1)
    # the FP32 form of the same workload (offsets, FP32 state and arithmetic,
    # FP64-computed geometry rounded once), timed like the FP64 line
    fp32 = None
    if world == 1 and args.precision == 64 and not args.no_fp32_form:
        fp32 = fp32_form(args, dev, stream)
    prec_sec = None
    if world == 1 and args.precision_steps > 0:
        prec_sec = precision_section(args.precision_steps, device=dev)

    w = 8 if args.precision == 64 else 4
    bpn = bytes_per_node(dim, N, w)
    nodes = mesh.nelem * mesh.Np
    launches = 5 * args.steps
    t_launch = t_ms * 1e-3 / launches
    peak, peak_kind = measured_peaks()
    achieved = nodes * bpn / t_launch / 1e9
    key = f"{kernel_name}_3d_N{N}_fp{args.precision}_n{args.n_side}"
    state_gb = dQ.numel() * w / 1e9
    geo_gb = nodes * (bpn - 4 * 5 * w) / 1e9  # metric and face geometry
    l2_note = (f"inputs {'larger' if nodes * bpn > L2_BYTES else 'smaller'} than L2 "
               f"(state {state_gb:.2f} GB, geometry {geo_gb:.2f} GB in FP{args.precision})")
    traffic = load_traffic(key)
    value = world * dof * 5 * args.steps / (t_ms * 1e-3)
    bi = dQ.numel() * w
    bo = dQ.numel() * w
    line = {
        "metric": METRIC, "value": value, "unit": METRIC, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == 64 else "f32",
        "data": "synthetic",
        "config": {"workload": f"3-D Euler, periodic [0,2π]^3, {args.n_side}^3 hexes, N={N}, "
                               "warped x_i += 0.05 sin x sin y sin z, seeded Fourier state (seed 0)",
                   "n_side": args.n_side, "order": N, "nelem": mesh.nelem, "dof": dof, "dt": dt,
                   "parallelism": f"replicas{world}",
                   "l2": l2_note,
                   "state_finite": finite},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_kind": peak_kind,
                     "traffic": traffic, "bytes_per_node": bpn, "kernel": kernel_name,
                     "launch_ms": t_launch * 1e3},
        "e2e": {"value": world * dof * 5 * args.e2e_steps / (e2e_ms * 1e-3), "unit": METRIC,
                "h2d_bytes_per_step": bi, "d2h_bytes_per_step": bo, "steps": args.e2e_steps,
                "ms_per_step": e2e_ms / args.e2e_steps, "results_repeat": e2e_ok,
                "how": "cb_solver per state buffer; H2D, step and D2H on three streams, three states in flight"},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if fp32 is not None:
        fp32["over_fp64_plain"] = fp32["value"] / value
        line["fp32_form"] = fp32
    if prec_sec is not None:
        line["precision_form"] = prec_sec
    if par is not None:
        res = par.result()
        line["parity"] = {"timed_workload": res}
        if not args.no_cpu_baseline:
            r1, s1, e1 = _oracle_rate(N, args.cpu_seconds / 2, 8, 4, 1)
            line["cpu_baseline"] = {
                "value": res["oracle_value"], "unit": METRIC, "cores": res["oracle_threads"], "kind": "port",
                "sample": f"the whole timed workload ({args.n_side}^3 hexes, N={N}), all {args.parity_steps} "
                          f"steps of the parity run in {res['oracle_seconds']:.1f} s, C oracle with "
                          f"{res['oracle_threads']} OpenMP threads (overlapping GPU work of this process)",
                "single_thread": {"value": r1, "unit": METRIC, "cores": 1,
                                  "sample": f"8^3 hexes N={N}, {s1} LSRK steps in {e1:.1f} s, one thread"}}
    elif rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_sample(N, args.cpu_seconds)
    if world == 1 and not args.no_batched:
        bat = batched_ensemble(args.batched_instances, steps=args.batched_steps, device=dev,
                               parity_sample=16 if args.parity_steps > 0 else 0,
                               precisions=tuple(args.batched_precisions), tune=not args.no_autotune)
        if args.precision == 64 and "fp32" in bat:
            # against the headline FP64 single-mesh stage (3-D, another workload)
            bat["fp32_over_fp64_plain"] = bat["fp32"]["value"] / value
        if "fp32" in bat and "fp64" in bat:
            # against the FP64 form of the same ensemble
            bat["fp32_over_fp64_batched"] = bat["fp32"]["value"] / bat["fp64"]["value"]
        line["batched"] = bat
    if world == 1 and not args.no_served:
        from canary_b200 import serve
        line["served"] = serve.benchmark(args.served_requests, seed=0, precision=32,
                                         baseline_count=args.served_baseline, device=str(dev))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if tdist is not None:
        tdist.barrier()
        tdist.destroy_process_group()


if __name__ == "__main__":
    main()
