"""Initial conditions and time-step rules of the benchmark workloads.

These are written from the workload definitions (not from the reference,
whose drivers only run a rising thermal bubble):

  * isentropic vortex on the periodic square [0,10]^2 (free stream ρ=1, u=1,
    v=0, p=1, strength β, centre (xc, yc));
  * seeded random Fourier initial state on the periodic cube [0,2π]^3;
  * time step dt = 0.2 h / (N^2 max(|u|+c)).

Conserved variables are returned in the reference's state order:
2-D (U, V, ρ, E), 3-D (U, V, W, ρ, E), with E = p/(γ-1) + ρ|u|²/2.
"""
from __future__ import annotations

import math

import numpy as np

GAMMA = 1.4


def isentropic_vortex(x, y, beta=5.0, xc=5.0, yc=5.0, gamma=GAMMA, t=0.0, L=10.0):
    """Conserved state of the isentropic vortex advected by u=1 for time t on
    a periodic box of side L.  Returns (U, V, ρ, E)."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    cx = xc + t
    dx = np.mod(x - cx + L / 2, L) - L / 2 if t != 0.0 else x - cx
    dy = y - yc
    r2 = dx * dx + dy * dy
    g1 = gamma - 1.0
    dT = -g1 * beta * beta / (8.0 * gamma * math.pi ** 2) * np.exp(1.0 - r2)
    f = beta / (2.0 * math.pi) * np.exp((1.0 - r2) / 2.0)
    u = 1.0 - f * dy
    v = f * dx
    rho = (1.0 + dT) ** (1.0 / g1)
    p = rho ** gamma
    E = p / g1 + 0.5 * rho * (u * u + v * v)
    return rho * u, rho * v, rho, E


def fourier_wavevectors(kmax: int = 4) -> np.ndarray:
    """All k in Z^3 with 0 < |k|_2 <= kmax, lexicographic order."""
    r = range(-kmax, kmax + 1)
    ks = [(a, b, c) for a in r for b in r for c in r if 0 < a * a + b * b + c * c <= kmax * kmax]
    return np.array(ks, dtype=np.float64)


def fourier_coefficients(seed: int = 0, kmax: int = 4, amp_rho=0.01, amp_vel=0.1):
    """Amplitudes a_k ~ U(0, amp) and phases φ_k ~ U(0, 2π) for ρ, u, v, w,
    drawn in that order from numpy's PCG64(seed)."""
    ks = fourier_wavevectors(kmax)
    rng = np.random.Generator(np.random.PCG64(seed))
    coef = []
    for amp in (amp_rho, amp_vel, amp_vel, amp_vel):
        a = rng.uniform(0.0, amp, len(ks))
        phi = rng.uniform(0.0, 2.0 * math.pi, len(ks))
        coef.append((a, phi))
    return ks, coef


def fourier_state(x, y, z, seed=0, kmax=4, gamma=GAMMA, device=None, dtype=None):
    """Conserved (U, V, W, ρ, E) of the random Fourier state with p = 1:
    ρ = 1 + Σ a_k sin(k·x + φ_k), (u, v, w) = Σ a_k sin(k·x + φ_k).

    Evaluated in float64 with torch on `device` (e.g. "cuda") when given,
    summing 16 wave vectors per batch, else with numpy one wave vector at a
    time; the two orders of summation agree to round-off."""
    ks, coef = fourier_coefficients(seed, kmax)
    if device is not None:
        import torch
        X = [torch.as_tensor(np.asarray(c), dtype=torch.float64, device=device).reshape(-1)
             for c in (x, y, z)]
        K = torch.as_tensor(ks, dtype=torch.float64, device=device)
        out = []
        chunk = 16
        for a, phi in coef:
            A = torch.as_tensor(a, dtype=torch.float64, device=device)
            PH = torch.as_tensor(phi, dtype=torch.float64, device=device)
            acc = torch.zeros_like(X[0])
            for q0 in range(0, len(ks), chunk):
                sl = slice(q0, min(q0 + chunk, len(ks)))
                arg = (K[sl, 0:1] * X[0] + K[sl, 1:2] * X[1]) + K[sl, 2:3] * X[2] + PH[sl, None]
                acc = acc + (A[sl, None] * torch.sin(arg)).sum(0)
            out.append(acc.reshape(np.shape(x)))
        rho = 1.0 + out[0]
        u, v, w = out[1], out[2], out[3]
        E = 1.0 / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
        res = (rho * u, rho * v, rho * w, rho, E)
        return tuple(t.cpu().numpy() for t in res)
    X = [np.asarray(c, dtype=np.float64) for c in (x, y, z)]
    out = []
    for a, phi in coef:
        acc = np.zeros_like(X[0])
        for q in range(len(ks)):
            arg = (ks[q, 0] * X[0] + ks[q, 1] * X[1]) + ks[q, 2] * X[2] + phi[q]
            acc = acc + a[q] * np.sin(arg)
        out.append(acc)
    rho = 1.0 + out[0]
    u, v, w = out[1], out[2], out[3]
    E = 1.0 / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return rho * u, rho * v, rho * w, rho, E


def max_wave_speed(Q, dim, gamma=GAMMA):
    """max over nodes of |u| + c for a conserved state Q (Np, nstate, nelem)."""
    Q = np.asarray(Q)
    ir, ie = (3, 4) if dim == 3 else (2, 3)
    rho = Q[:, ir, :]
    mom = [Q[:, c, :] for c in range(dim)]
    ke = sum(m * m for m in mom) / (2.0 * rho)
    p = (gamma - 1.0) * (Q[:, ie, :] - ke)
    speed = np.sqrt(sum(m * m for m in mom)) / rho + np.sqrt(gamma * p / rho)
    return float(speed.max())


def fourier_dt(Q, N, h=2 * math.pi / 32, gamma=GAMMA):
    """dt = 0.2 h / (N^2 max(|u| + c))."""
    return 0.2 * h / (N * N * max_wave_speed(Q, 3, gamma))


def vortex_ensemble(count: int = 512, seed: int = 0):
    """Parameters of an ensemble of independent 2-D vortex instances on
    [0,10]^2: instance i draws, from numpy's PCG64(seed + i) in this order,
    N ~ U{3..8}, elements per side ~ U{4..48}, β ~ U(1,5) and the centre
    (xc, yc) ~ U([2,8]^2).  Every other setting is that of the single vortex
    (free stream ρ=1, u=1, v=0, p=1, dt=0.002, 500 steps)."""
    out = []
    for i in range(count):
        rng = np.random.Generator(np.random.PCG64(seed + i))
        N = int(rng.integers(3, 9))
        n_side = int(rng.integers(4, 49))
        beta = float(rng.uniform(1.0, 5.0))
        xc, yc = (float(v) for v in rng.uniform(2.0, 8.0, 2))
        out.append(dict(N=N, n_side=n_side, beta=beta, xc=xc, yc=yc))
    return out


# ----------------------------------------------------------- device forms
def isentropic_vortex_t(x, y, beta=5.0, xc=5.0, yc=5.0, gamma=GAMMA):
    """Torch form of isentropic_vortex at t = 0 for device tensors x, y;
    returns (U, V, ρ, E) tensors."""
    import torch
    dx, dy = x - xc, y - yc
    r2 = dx * dx + dy * dy
    g1 = gamma - 1.0
    dT = (-g1 * beta * beta / (8.0 * gamma * math.pi ** 2)) * torch.exp(1.0 - r2)
    f = (beta / (2.0 * math.pi)) * torch.exp((1.0 - r2) / 2.0)
    u = 1.0 - f * dy
    v = f * dx
    rho = (1.0 + dT) ** (1.0 / g1)
    p = rho ** gamma
    E = p / g1 + 0.5 * rho * (u * u + v * v)
    return rho * u, rho * v, rho, E


_FOURIER = {}


def fourier_state_t(x, y, z, seed=0, kmax=4, gamma=GAMMA, vel_peak=None):
    """Torch form of fourier_state for device tensors x, y, z (FP64), summing
    16 wave vectors per batch; returns (U, V, W, ρ, E) tensors.  With
    `vel_peak`, each velocity component's Fourier sum is scaled so that its
    largest magnitude over the given nodes is vel_peak (on the device, no
    host synchronisation)."""
    import torch
    from .dg import to_device
    key = (kmax, str(x.device))
    ks, coef = fourier_coefficients(seed, kmax)
    if key not in _FOURIER:
        _FOURIER[key] = to_device(ks, torch.float64, x.device).reshape(ks.shape[1], ks.shape[0]).t()
    K = _FOURIER[key]
    # the amplitudes and phases of the four fields in one upload
    cf = to_device(np.array([v for pair in coef for v in pair]).T, torch.float64, x.device).reshape(8, -1)
    C = [(cf[2 * q], cf[2 * q + 1]) for q in range(4)]
    X = [c.reshape(-1) for c in (x, y, z)]
    out = []
    for A, PH in C:
        acc = torch.zeros_like(X[0])
        for q0 in range(0, K.shape[0], 16):
            sl = slice(q0, min(q0 + 16, K.shape[0]))
            arg = (K[sl, 0:1] * X[0] + K[sl, 1:2] * X[1]) + K[sl, 2:3] * X[2] + PH[sl, None]
            acc = acc + (A[sl, None] * torch.sin(arg)).sum(0)
        out.append(acc.reshape(x.shape))
    rho = 1.0 + out[0]
    u, v, w = out[1], out[2], out[3]
    if vel_peak is not None:
        u, v, w = (c * (vel_peak / torch.amax(torch.abs(c))) for c in (u, v, w))
    E = 1.0 / (gamma - 1.0) + 0.5 * rho * (u * u + v * v + w * w)
    return rho * u, rho * v, rho * w, rho, E


def device_state(fields, dtype=None, offset=None):
    """Pack per-field device tensors (nelem, Np) into the flat (Np, nstate,
    nelem) column-major state, minus the per-field `offset`, cast to dtype."""
    import torch
    Q = torch.stack(fields, dim=1)  # (nelem, nstate, Np) C order == (Np, nstate, nelem) F order
    if offset is not None:  # per-field scalars (no host-to-device copy)
        for s, o in enumerate(offset):
            if o != 0.0:
                Q[:, s] -= float(o)
    return Q.to(dtype or Q.dtype).contiguous().reshape(-1)
