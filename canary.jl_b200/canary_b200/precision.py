"""Precision form report: the FP32 working form (FP32 state, volume, surface
and RK arithmetic; FP64 geometry computed on the device and rounded once;
per-field state offsets; compensated FP64 conservation sums) against the FP64
form on the same mesh and initial state, after the same number of steps.

    python -m canary_b200.precision [--steps 1000] [--n-side 32] [--orders 4 7 10]

Cases: the warped periodic cube [0,2π]^3 (x_i += 0.05 sin x sin y sin z)
with the seeded Fourier state, inviscid and with the LDG Navier–Stokes terms
(mu = 1e-3, Pr = 0.72); the 2-D isentropic vortex on [0,10]^2 (10x10 quads).
The FP64 form is itself pinned to the CPU oracle at 1e-12 on smaller meshes
(tests/test_gpu_parity.py, tests/test_geometry.py).  Errors are relative L2
norms per state field, evaluated on the device in FP64.

The seeded Fourier state steepens into shocks, which the unlimited DG scheme
(the reference's as well) does not survive: on the oracle it turns non-finite
by t = 0.09-0.15 on 4^3-8^3 meshes.  The 3-D time step is therefore
min(0.2 h / (N^2 max(|u|+c)), t_smooth / steps) with t_smooth = 0.08, so that
the requested number of steps (the accumulation of FP32 rounding that the
report measures) stays in the smooth regime.
"""
from __future__ import annotations

import math
import time

import numpy as np

from . import ic
from .dg import LSRK, DeviceMesh, _torch, make_phys, viscous_fused


def _rel_l2(a, b):
    torch = _torch()
    return [float(torch.linalg.vector_norm(a[:, s] - b[:, s]) / torch.linalg.vector_norm(b[:, s]))
            for s in range(b.shape[1])]


T_SMOOTH = 0.08


def run_case(dim, N, n_side, steps, visc=0.0, seed=0, device="cuda", t_smooth=T_SMOOTH):
    torch = _torch()
    from .serve import wave_speed
    if dim == 3:
        L = 2 * math.pi
        x = (np.linspace(0.0, L, n_side + 1),) * 3
        dm = DeviceMesh.build(3, N, x, (True,) * 3, warp_amp=0.05, device=device)
        f = ic.fourier_state_t(*dm.coords(), seed=seed)
        dt = min(0.2 * (L / n_side) / (N * N * float(wave_speed(f, 3).item())), t_smooth / steps)
    else:
        x = (np.linspace(0.0, 10.0, n_side + 1),) * 2
        dm = DeviceMesh.build(2, N, x, (True,) * 2, device=device)
        f = ic.isentropic_vortex_t(*dm.coords())
        dt = 0.002
    ns = len(f)
    phys = make_phys(visc=visc)
    m = dm.mesh
    dof = m.nelem * m.Np * ns
    out = {"dim": dim, "N": N, "n_side": n_side, "nelem": m.nelem, "dof": dof, "steps": steps, "dt": dt,
           "visc": visc}
    finals = {}
    for prec in (64, 32):
        real = torch.float64 if prec == 64 else torch.float32
        use_off = prec == 32 and (visc == 0.0 or viscous_fused(dim, N))
        off = np.array([float(t.mean().item()) for t in f]) if use_off else np.zeros(ns)
        Q = ic.device_state(list(f), real, off)
        rhs = torch.zeros_like(Q)
        s = LSRK(dm, Q, rhs, prec, phys)
        if use_off:
            s.set_offset(off)
        s0 = s.sums()
        torch.cuda.synchronize()
        t = time.perf_counter()
        s.run(steps, dt)
        torch.cuda.synchronize()
        el = time.perf_counter() - t
        s1 = s.sums()
        finals[prec] = (Q.double().view(m.nelem, ns, m.Np) +
                        torch.as_tensor(off, dtype=torch.float64, device=Q.device).view(1, -1, 1))
        out[f"fp{prec}"] = {"dof_stage_per_s": dof * 5 * steps / el, "seconds": el,
                            "finite": bool(torch.isfinite(finals[prec]).all().item()),
                            "mass_drift_rel": float(abs(s1[0][ns - 2] - s0[0][ns - 2]) / abs(s0[0][ns - 2])),
                            "energy_drift_rel": float(abs(s1[0][ns - 1] - s0[0][ns - 1]) / abs(s0[0][ns - 1]))}
        s.close()
    names = ("U", "V", "W", "rho", "E") if dim == 3 else ("U", "V", "rho", "E")
    err = _rel_l2(finals[32], finals[64])
    out["fp32_rel_l2_vs_fp64"] = dict(zip(names, err))
    out["max_rel_l2"] = max(err)
    return out


def report(orders=(4, 7, 10), n_side=32, steps=1000, ns_n_side=16, device="cuda"):
    """Inviscid 3-D cases on n_side^3 hexes, the viscous variant on
    ns_n_side^3 hexes (its LDG passes cost several times the fused inviscid
    stage), and the 2-D vortex; yields one dict per case."""
    for N in orders:
        yield run_case(3, N, n_side, steps, device=device)
    for N in orders:
        yield run_case(3, N, ns_n_side, steps, visc=1e-3, device=device)
    for N in orders:
        yield run_case(2, N, 10, steps, device=device)


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(description="FP32 precision form against FP64")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--n-side", type=int, default=32)
    ap.add_argument("--orders", type=int, nargs="+", default=[4, 7, 10])
    ap.add_argument("--ns-n-side", type=int, default=16)
    a = ap.parse_args(argv)
    for c in report(tuple(a.orders), a.n_side, a.steps, a.ns_n_side):
        print(json.dumps(c), flush=True)


if __name__ == "__main__":
    main()
