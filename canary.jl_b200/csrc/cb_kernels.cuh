// Kernel templates of the nodal-DG hot path and their host launchers.
// Included once per (dim, precision) translation unit; see cb_inst.cuh.
#pragma once
#include "cb_dg.cuh"

namespace cb {

// Face-neighbour code of the fused path: for an interior face
// (e2 << 3) | f2 with 0-based neighbour element e2 and face f2;
// NBR_WALL for a reflective wall (elemtobndy == 1).
constexpr int32_t NBR_WALL = -1;

template <typename T>
__device__ __forceinline__ void load_D(T *Ds, const T *__restrict__ D, int nq2) {
  for (int t = threadIdx.x; t < nq2; t += blockDim.x) Ds[t] = D[t];
}

// Reflective wall state (euler3d_set3c.jl:382-389).
template <int DIM, typename T>
__device__ __forceinline__ void wall_state(const T *qM, const T *nrm, T *qP) {
  constexpr int NS = Lay<DIM>::NS;
  T un = nrm[0] * qM[0] + nrm[1] * qM[1];
  if (DIM == 3) un = un + nrm[2] * qM[2];
#pragma unroll
  for (int s = 0; s < NS; ++s) qP[s] = qM[s];
#pragma unroll
  for (int c = 0; c < DIM; ++c) qP[c] = qM[c] - T(2) * un * nrm[c];
}

// ======================================================================
// Stateless volume RHS: rhs += volume integral (volumerhs!).
// ======================================================================
template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS)
k_volumerhs(T *__restrict__ rhs, const T *__restrict__ Q,
            const T *__restrict__ vgeo, const T *__restrict__ D, int64_t nelem,
            PhysT<T> p) {
  using C = Cfg<DIM, Nq>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, Np = C::Np;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *Ds = reinterpret_cast<T *>(smem_raw);
  T *sF = Ds + Nq * Nq;
  load_D(Ds, D, Nq * Nq);
  const int64_t e0 = (int64_t)blockIdx.x * C::EPB;
  T R[C::NPT][NS];
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < C::SLOTS && e < nelem) {
      T q[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        q[s] = Q[n + Np * (s + NS * e)];
        R[u][s] = rhs[n + Np * (s + NS * e)];
      }
      pointwise_euler<DIM, Nq, C::EPB, T>(q, vgeo + (int64_t)Np * NVG * e, n, el, sF, p, R[u]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < C::SLOTS && e < nelem) {
      contract<DIM, Nq, C::EPB, T>(sF, Ds, el, n, R[u]);
#pragma unroll
      for (int s = 0; s < NS; ++s) rhs[n + Np * (s + NS * e)] = R[u][s];
    }
  }
}

// ======================================================================
// Stateless face RHS with the reference's int64 vmaps (fluxrhs!).
// Face fluxes of the block's elements go to shared memory first and are then
// subtracted per node in face order, which reproduces the reference's
// sequential f = 1..nface update without atomics.
// ======================================================================
template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS)
k_fluxrhs(T *__restrict__ rhs, const T *__restrict__ Q,
          const T *__restrict__ sgeo, const T *__restrict__ vgeo,
          int64_t nelem, const int64_t *__restrict__ vmapM,
          const int64_t *__restrict__ vmapP,
          const int64_t *__restrict__ elemtobndy, PhysT<T> p,
          unsigned *status) {
  using C = Cfg<DIM, Nq>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, FS = C::EPB * Nfp;
  constexpr int GC = DIM * DIM + 2 + DIM - 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *FF = reinterpret_cast<T *>(smem_raw);  // [NF][NS][EPB*Nfp]
  const int64_t e0 = (int64_t)blockIdx.x * C::EPB;
#pragma unroll
  for (int u = 0; u < C::FPT; ++u) {
    const int fs = threadIdx.x + u * C::THREADS;
    if (fs >= C::FSLOTS) break;
    const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
    const int64_t e = e0 + el;
    if (e >= nelem) continue;
    const int64_t fidx = fn + (int64_t)Nfp * (f + NF * e);
    const T *sg = sgeo + (int64_t)NSG * fidx;
    T nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
    const T sMJ = sg[DIM];
    const int64_t idM = vmapM[fidx], idP = vmapP[fidx];
    const int64_t vM = (idM - 1) % Np, eP = (idP - 1) / Np, vP = (idP - 1) % Np;
    T qM[NS], qP[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qM[s] = Q[vM + Np * (s + NS * e)];
    const T gM = p.grav != T(0) ? vgeo[vM + Np * (GC + NVG * e)] : T(0);
    const T PM = pressure<DIM, T>(qM, gM, p);
    T PP;
    const int64_t bc = elemtobndy[f + NF * e];
    T out[NS];
    if ((idM - 1) / Np != e || idM < 1 || (bc == 0 && (idP < 1 || eP >= nelem))) {
      atomicOr(status, ST_MESH);  // vmapP points outside the mesh: skip the face
#pragma unroll
      for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = T(0);
      continue;
    }
    if (bc == 0) {
#pragma unroll
      for (int s = 0; s < NS; ++s) qP[s] = Q[vP + Np * (s + NS * eP)];
      const T gP = p.grav != T(0) ? vgeo[vP + Np * (GC + NVG * eP)] : T(0);
      PP = pressure<DIM, T>(qP, gP, p);
    } else if (bc == 1) {
      wall_state<DIM, T>(qM, nrm, qP);
      PP = PM;
    } else {
      atomicOr(status, ST_BC);
#pragma unroll
      for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = T(0);
      continue;
    }
    rusanov<DIM, T>(qM, PM, qP, PP, nrm, p, out);
#pragma unroll
    for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = sMJ * out[s];
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < C::SLOTS && e < nelem) {
      const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
      const bool onface = i == 0 || i == Nq - 1 || j == 0 || j == Nq - 1 ||
                          (DIM == 3 && (k == 0 || k == Nq - 1));
      if (!onface) continue;
      T R[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) R[s] = rhs[n + Np * (s + NS * e)];
      gather_face_terms<DIM, Nq, C::EPB, T>(FF, el, n, R);
#pragma unroll
      for (int s = 0; s < NS; ++s) rhs[n + Np * (s + NS * e)] = R[s];
    }
  }
}

// ======================================================================
// Stateless update (updatesolution!).  Elementwise.
// ======================================================================
template <int DIM, typename T>
__global__ void k_update(T *__restrict__ rhs, const T *__restrict__ rhs_gradQ,
                         T *__restrict__ Q, const T *__restrict__ vgeo,
                         int64_t nelem, int Np, T rka, T rkb, T dt, T visc) {
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, MJI = DIM * DIM + 1;
  const int64_t total = (int64_t)Np * NS * nelem;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = q % Np, e = q / ((int64_t)Np * NS);
    const int s = (int)((q / Np) % NS);
    T r = rhs[q];
    if (rhs_gradQ) r += visc * rhs_gradQ[n + Np * (s + (int64_t)NS * DIM * e)];
    Q[q] += rkb * dt * r * vgeo[n + Np * (MJI + (int64_t)NVG * e)];
    rhs[q] = r * rka;
  }
}

// ======================================================================
// Fused LSRK stage: volume + face + update in one pass over the element.
//   Qin   state at the start of the stage (read, also for neighbour traces)
//   Qout  state after the stage (distinct buffer)
//   rhs   residual carry: read, then overwritten with rka_next * residual
// ======================================================================
template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS)
k_stage(const T *__restrict__ Qin, T *__restrict__ Qout, T *__restrict__ rhs,
        const T *__restrict__ vgeo, const T *__restrict__ sgeo,
        const int32_t *__restrict__ nbr, const T *__restrict__ D,
        int64_t nelem, PhysT<T> p, Offs<T, Lay<DIM>::NS> qref, T rka, T rkbdt,
        unsigned *status) {
  using C = Cfg<DIM, Nq>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, SP = C::SLOTS;
  constexpr int FS = C::EPB * Nfp, MJI = DIM * DIM + 1;
  constexpr int GC = DIM * DIM + 2 + DIM - 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *Ds = reinterpret_cast<T *>(smem_raw);
  T *sQ = Ds + ((Nq * Nq + 1) & ~1);  // [NS][SP]
  T *sF = sQ + NS * SP;               // [DIM][NS][SP], reused as FF
  load_D(Ds, D, Nq * Nq);
  const int64_t e0 = (int64_t)blockIdx.x * C::EPB;
  T R[C::NPT][NS];
  // ---- pointwise fluxes
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < C::SLOTS && e < nelem) {
      T q[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const T d = Qin[n + Np * (s + NS * e)];
        sQ[s * SP + slot] = d;
        q[s] = d + qref.v[s];
        R[u][s] = rhs[n + Np * (s + NS * e)];
      }
      pointwise_euler<DIM, Nq, C::EPB, T>(q, vgeo + (int64_t)Np * NVG * e, n, el, sF, p, R[u]);
    }
  }
  __syncthreads();
  // ---- volume contraction
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    if (slot < C::SLOTS && e0 + el < nelem) contract<DIM, Nq, C::EPB, T>(sF, Ds, el, n, R[u]);
  }
  __syncthreads();
  // ---- face fluxes (sF reused as FF[NF][NS][EPB*Nfp])
  T *FF = sF;
#pragma unroll
  for (int u = 0; u < C::FPT; ++u) {
    const int fs = threadIdx.x + u * C::THREADS;
    if (fs >= C::FSLOTS) break;
    const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
    const int64_t e = e0 + el;
    if (e >= nelem) continue;
    const int vM = face_node<DIM, Nq>(f, fn);
    const T *sg = sgeo + (int64_t)NSG * (fn + (int64_t)Nfp * (f + NF * e));
    T nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
    const T sMJ = sg[DIM];
    T qM[NS], qP[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qM[s] = sQ[s * SP + el * Np + vM] + qref.v[s];
    const T gM = p.grav != T(0) ? vgeo[vM + Np * (GC + NVG * e)] : T(0);
    const T PM = pressure<DIM, T>(qM, gM, p);
    const int32_t nb = nbr[f + NF * e];
    T PP;
    if (nb >= 0) {
      const int64_t e2 = nb >> 3;
      const int vP = face_node<DIM, Nq>(nb & 7, fn);
#pragma unroll
      for (int s = 0; s < NS; ++s) qP[s] = Qin[vP + Np * (s + NS * e2)] + qref.v[s];
      const T gP = p.grav != T(0) ? vgeo[vP + Np * (GC + NVG * e2)] : T(0);
      PP = pressure<DIM, T>(qP, gP, p);
    } else {
      wall_state<DIM, T>(qM, nrm, qP);
      PP = PM;
    }
    T out[NS];
    rusanov<DIM, T>(qM, PM, qP, PP, nrm, p, out);
#pragma unroll
    for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = sMJ * out[s];
  }
  __syncthreads();
  // ---- face accumulation and LSRK update
  bool bad = false;
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < C::SLOTS && e < nelem) {
      gather_face_terms<DIM, Nq, C::EPB, T>(FF, el, n, R[u]);
      const T mji = vgeo[n + Np * (MJI + (int64_t)NVG * e)];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const T qn = sQ[s * SP + slot] + rkbdt * R[u][s] * mji;
        bad |= !isfinite(qn);
        Qout[n + Np * (s + NS * e)] = qn;
        rhs[n + Np * (s + NS * e)] = R[u][s] * rka;
      }
    }
  }
  if (bad) atomicOr(status, ST_NONFINITE);
}

// Build the compact face-neighbour table from the reference vmaps and
// validate that they describe a conforming mesh with orientation 1.
template <int DIM, int Nq>
__global__ void k_build_nbr(int32_t *__restrict__ nbr,
                            const int64_t *__restrict__ vmapM,
                            const int64_t *__restrict__ vmapP,
                            const int64_t *__restrict__ elemtobndy,
                            int64_t nelem, int64_t nall, unsigned *status) {
  // nall: elements a neighbour may be (nelem, plus the ghost elements that a
  // partitioned solve appends after its own)
  using C = Cfg<DIM, Nq>;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE;
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nelem * NF) return;
  const int64_t e = t / NF;
  const int f = (int)(t % NF);
  const int64_t bc = elemtobndy[t];
  const int64_t *vm = vmapM + (int64_t)Nfp * t, *vp = vmapP + (int64_t)Nfp * t;
  bool ok = true;
  for (int fn = 0; fn < Nfp; ++fn)
    ok &= vm[fn] == Np * e + face_node<DIM, Nq>(f, fn) + 1;
  if (bc == 1) {
    nbr[t] = NBR_WALL;
  } else if (bc == 0) {
    const int64_t id0 = vp[0] - 1;
    const int64_t e2 = id0 / Np;
    int f2 = -1;
    for (int g = 0; g < NF; ++g)
      if (face_node<DIM, Nq>(g, 0) == (int)(id0 % Np)) {
        bool m = true;
        for (int fn = 0; fn < Nfp; ++fn) m &= vp[fn] == Np * e2 + face_node<DIM, Nq>(g, fn) + 1;
        if (m) { f2 = g; break; }
      }
    ok &= f2 >= 0 && e2 >= 0 && e2 < nall && e2 < (1ll << 28);
    nbr[t] = ok ? (int32_t)((e2 << 3) | f2) : NBR_WALL;
  } else {
    atomicOr(status, ST_BC);
    nbr[t] = NBR_WALL;
  }
  if (!ok) atomicOr(status, ST_MESH);
}

// ======================================================================
// LDG Navier–Stokes passes (nse2d.jl / nse3d.jl).  Stateless.
// ======================================================================

// primitives (u, v, [w], ρ, T) in state slots (nse3d.jl:509-522)
template <int DIM, typename T>
__device__ __forceinline__ void primitives(const T *q, T gc, const PhysT<T> &p, T *prim) {
  constexpr int IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  const T P = pressure<DIM, T>(q, gc, p);
#pragma unroll
  for (int c = 0; c < DIM; ++c) prim[c] = q[c] / q[IR];
  prim[IR] = q[IR];
  prim[IE] = P / (p.R * q[IR]);
}

// volume_grad!: rhs[:, s, c, e] = -Σ Dᵀ (MJ ξ_c prim_s) per reference direction.
template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS)
k_volume_grad(T *__restrict__ rhs, const T *__restrict__ Q,
              const T *__restrict__ vgeo, const T *__restrict__ D,
              int64_t nelem, PhysT<T> p) {
  using C = Cfg<DIM, Nq>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, Np = C::Np, SP = C::SLOTS;
  constexpr int GC = DIM * DIM + 2 + DIM - 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *Ds = reinterpret_cast<T *>(smem_raw);
  T *sF = Ds + ((Nq * Nq + 1) & ~1);
  load_D(Ds, D, Nq * Nq);
  const int64_t e0 = (int64_t)blockIdx.x * C::EPB;
  T prim[C::NPT][NS], met[C::NPT][DIM][DIM], MJ[C::NPT];
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < C::SLOTS && e < nelem) {
      T q[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) q[s] = Q[n + Np * (s + NS * e)];
      const T *vg = vgeo + (int64_t)Np * NVG * e;
      load_metric<DIM, T>(vg, n, Np, met[u], MJ[u]);
      const T gc = p.grav != T(0) ? vg[n + Np * GC] : T(0);
      primitives<DIM, T>(q, gc, p, prim[u]);
    }
  }
  for (int c = 0; c < DIM; ++c) {
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = threadIdx.x + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      if (slot < C::SLOTS && e0 + el < nelem)
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int s = 0; s < NS; ++s)
            sF[(r * NS + s) * SP + el * Np + n] = MJ[u] * (met[u][r][c] * prim[u][s]);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = threadIdx.x + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      const int64_t e = e0 + el;
      if (slot < C::SLOTS && e < nelem) {
        T R[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) R[s] = T(0);
        contract_sub<DIM, Nq, C::EPB, T>(sF, Ds, el, n, R);
#pragma unroll
        for (int s = 0; s < NS; ++s) rhs[n + Np * (s + NS * (c + (int64_t)DIM * e))] = R[s];
      }
    }
    __syncthreads();
  }
}

// flux_grad!: rhs[vM, s, c] += sMJ n_c (prim⁻ + prim⁺)/2 in face order.
template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS)
k_flux_grad(T *__restrict__ rhs, const T *__restrict__ Q,
            const T *__restrict__ sgeo, const T *__restrict__ vgeo,
            int64_t nelem, const int64_t *__restrict__ vmapM,
            const int64_t *__restrict__ vmapP,
            const int64_t *__restrict__ elemtobndy, PhysT<T> p,
            unsigned *status) {
  using C = Cfg<DIM, Nq>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, FS = C::EPB * Nfp;
  constexpr int GC = DIM * DIM + 2 + DIM - 1, IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *FF = reinterpret_cast<T *>(smem_raw);  // [NF][NS*DIM][FS]
  const int64_t e0 = (int64_t)blockIdx.x * C::EPB;
  for (int fs = threadIdx.x; fs < C::FSLOTS; fs += C::THREADS) {
    const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
    const int64_t e = e0 + el;
    if (e >= nelem) continue;
    const int64_t fidx = fn + (int64_t)Nfp * (f + NF * e);
    const T *sg = sgeo + (int64_t)NSG * fidx;
    T nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
    const T sMJ = sg[DIM];
    const int64_t idM = vmapM[fidx], idP = vmapP[fidx];
    const int64_t vM = (idM - 1) % Np, eP = (idP - 1) / Np, vP = (idP - 1) % Np;
    T qM[NS], pM[NS], pP[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qM[s] = Q[vM + Np * (s + NS * e)];
    const T gM = p.grav != T(0) ? vgeo[vM + Np * (GC + NVG * e)] : T(0);
    primitives<DIM, T>(qM, gM, p, pM);
    const int64_t bc = elemtobndy[f + NF * e];
    if ((idM - 1) / Np != e || idM < 1 || (bc == 0 && (idP < 1 || eP >= nelem))) {
      atomicOr(status, ST_MESH);
      for (int s = 0; s < NS * DIM; ++s) FF[(f * NS * DIM + s) * FS + el * Nfp + fn] = T(0);
      continue;
    }
    if (bc == 0) {
      T qP[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) qP[s] = Q[vP + Np * (s + NS * eP)];
      const T gP = p.grav != T(0) ? vgeo[vP + Np * (GC + NVG * eP)] : T(0);
      primitives<DIM, T>(qP, gP, p, pP);
    } else if (bc == 1) {
      T qP[NS];
      wall_state<DIM, T>(qM, nrm, qP);
#pragma unroll
      for (int c = 0; c < DIM; ++c) pP[c] = qP[c] / qM[IR];
      pP[IR] = qM[IR];
      pP[IE] = pM[IE];
    } else {
      atomicOr(status, ST_BC);
      for (int s = 0; s < NS * DIM; ++s) FF[(f * NS * DIM + s) * FS + el * Nfp + fn] = T(0);
      continue;
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const T fsv = T(0.5) * (pM[s] + pP[s]);
#pragma unroll
      for (int c = 0; c < DIM; ++c)
        FF[(f * NS * DIM + s * DIM + c) * FS + el * Nfp + fn] = sMJ * nrm[c] * fsv;
    }
  }
  __syncthreads();
  for (int slot = threadIdx.x; slot < C::SLOTS; slot += C::THREADS) {
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (e >= nelem) continue;
    const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
    int fl[3], fnl[3], nf = 0;
    if (i == 0) { fl[nf] = 0; fnl[nf++] = DIM == 3 ? j + Nq * k : j; }
    if (i == Nq - 1) { fl[nf] = 1; fnl[nf++] = DIM == 3 ? j + Nq * k : j; }
    if (j == 0) { fl[nf] = 2; fnl[nf++] = DIM == 3 ? i + Nq * k : i; }
    if (j == Nq - 1) { fl[nf] = 3; fnl[nf++] = DIM == 3 ? i + Nq * k : i; }
    if (DIM == 3 && k == 0) { fl[nf] = 4; fnl[nf++] = i + Nq * j; }
    if (DIM == 3 && k == Nq - 1) { fl[nf] = 5; fnl[nf++] = i + Nq * j; }
    if (nf == 0) continue;
    for (int s = 0; s < NS; ++s)
      for (int c = 0; c < DIM; ++c) {
        T *dst = rhs + n + Np * (s + NS * (c + (int64_t)DIM * e));
        T v = *dst;
        for (int a = 0; a < nf; ++a) v += FF[(fl[a] * NS * DIM + s * DIM + c) * FS + el * Nfp + fnl[a]];
        *dst = v;
      }
  }
}

// update_gradQ!: gradQ = rhs * MJI (elementwise)
template <int DIM, typename T>
__global__ void k_update_gradQ(T *__restrict__ gradQ, const T *__restrict__ rhs,
                               const T *__restrict__ vgeo, int64_t nelem, int Np) {
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, MJI = DIM * DIM + 1;
  const int64_t total = (int64_t)Np * NS * DIM * nelem;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = q % Np, e = q / ((int64_t)Np * NS * DIM);
    gradQ[q] = rhs[q] * vgeo[n + Np * (MJI + (int64_t)NVG * e)];
  }
}

// Viscous flux of one node (nse3d.jl:717-742 / nse2d.jl:598-614).
// g[s][c] = gradient component c of primitive slot s; vel = (u,v,[w]).
template <int DIM, typename T>
__device__ __forceinline__ void visc_flux(const T (*g)[DIM], const T *vel,
                                          const PhysT<T> &p, T (*out)[DIM]) {
  constexpr int IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  T div = g[0][0] + g[1][1];
  if (DIM == 3) div = div + g[2][DIM - 1];
#pragma unroll
  for (int c = 0; c < DIM; ++c) out[IR][c] = T(0) * g[IR][c];
  // momentum rows: τ_ac = ∂_c u_a + ∂_a u_c (+ λ div δ_ac); reference order
#pragma unroll
  for (int a = 0; a < DIM; ++a)
#pragma unroll
    for (int c = 0; c < DIM; ++c)
      out[a][c] = a == c ? T(2) * g[a][a] + p.lambda * div : g[a][c] + g[c][a];
#pragma unroll
  for (int c = 0; c < DIM; ++c) {
    T e = vel[0] * out[0][c] + vel[1] * out[1][c];
    if (DIM == 3) e = e + vel[2] * out[2][c];
    out[IE][c] = e + p.cpPr * g[IE][c];
  }
}

// volume_div!: rhs[:, s, 1, e] = -Σ Dᵀ (MJ ξ·F_visc); other components zeroed.
template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS)
k_volume_div(T *__restrict__ rhs, const T *__restrict__ gradQ,
             const T *__restrict__ Q, const T *__restrict__ vgeo,
             const T *__restrict__ D, int64_t nelem, PhysT<T> p) {
  using C = Cfg<DIM, Nq>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, Np = C::Np, SP = C::SLOTS;
  constexpr int IR = Lay<DIM>::IR;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *Ds = reinterpret_cast<T *>(smem_raw);
  T *sF = Ds + ((Nq * Nq + 1) & ~1);
  load_D(Ds, D, Nq * Nq);
  const int64_t e0 = (int64_t)blockIdx.x * C::EPB;
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < C::SLOTS && e < nelem) {
      T g[NS][DIM], out[NS][DIM], vel[DIM], met[DIM][DIM], MJ;
#pragma unroll
      for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int c = 0; c < DIM; ++c) g[s][c] = gradQ[n + Np * (s + NS * (c + (int64_t)DIM * e))];
      const T rho = Q[n + Np * (IR + NS * e)];
#pragma unroll
      for (int c = 0; c < DIM; ++c) vel[c] = Q[n + Np * (c + NS * e)] / rho;
      load_metric<DIM, T>(vgeo + (int64_t)Np * NVG * e, n, Np, met, MJ);
      visc_flux<DIM, T>(g, vel, p, out);
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          T a = met[r][0] * out[s][0] + met[r][1] * out[s][1];
          if (DIM == 3) a = a + met[r][2] * out[s][2];
          sF[(r * NS + s) * SP + el * Np + n] = MJ * a;
        }
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * C::THREADS;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < C::SLOTS && e < nelem) {
      T R[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) R[s] = T(0);
      contract_sub<DIM, Nq, C::EPB, T>(sF, Ds, el, n, R);
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        rhs[n + Np * (s + NS * (0 + (int64_t)DIM * e))] = R[s];
#pragma unroll
        for (int c = 1; c < DIM; ++c) rhs[n + Np * (s + NS * (c + (int64_t)DIM * e))] = T(0);
      }
    }
  }
}

// flux_div!: rhs[vM, s, 1] += sMJ · n·(F⁻+F⁺)/2 in face order.
template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS)
k_flux_div(T *__restrict__ rhs, const T *__restrict__ gradQ,
           const T *__restrict__ Q, const T *__restrict__ sgeo,
           int64_t nelem, const int64_t *__restrict__ vmapM,
           const int64_t *__restrict__ vmapP,
           const int64_t *__restrict__ elemtobndy, PhysT<T> p,
           unsigned *status) {
  using C = Cfg<DIM, Nq>;
  constexpr int NS = Lay<DIM>::NS, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, FS = C::EPB * Nfp;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *FF = reinterpret_cast<T *>(smem_raw);  // [NF][NS][FS]
  const int64_t e0 = (int64_t)blockIdx.x * C::EPB;
  for (int fs = threadIdx.x; fs < C::FSLOTS; fs += C::THREADS) {
    const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
    const int64_t e = e0 + el;
    if (e >= nelem) continue;
    const int64_t fidx = fn + (int64_t)Nfp * (f + NF * e);
    const T *sg = sgeo + (int64_t)NSG * fidx;
    T nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
    const T sMJ = sg[DIM];
    const int64_t idM = vmapM[fidx], idP = vmapP[fidx];
    const int64_t vM = (idM - 1) % Np, eP = (idP - 1) / Np, vP = (idP - 1) % Np;
    T gm[NS][DIM], gp[NS][DIM], vM_[DIM], vP_[DIM];
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int c = 0; c < DIM; ++c) gm[s][c] = gradQ[vM + Np * (s + NS * (c + (int64_t)DIM * e))];
    const T rhoM = Q[vM + Np * (IR + NS * e)];
#pragma unroll
    for (int c = 0; c < DIM; ++c) vM_[c] = Q[vM + Np * (c + NS * e)] / rhoM;
    const int64_t bc = elemtobndy[f + NF * e];
    if ((idM - 1) / Np != e || idM < 1 || (bc == 0 && (idP < 1 || eP >= nelem))) {
      atomicOr(status, ST_MESH);
      for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = T(0);
      continue;
    }
    if (bc == 0) {
#pragma unroll
      for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int c = 0; c < DIM; ++c) gp[s][c] = gradQ[vP + Np * (s + NS * (c + (int64_t)DIM * eP))];
      const T rhoP = Q[vP + Np * (IR + NS * eP)];
#pragma unroll
      for (int c = 0; c < DIM; ++c) vP_[c] = Q[vP + Np * (c + NS * eP)] / rhoP;
    } else if (bc == 1) {
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        T sn = nrm[0] * gm[s][0] + nrm[1] * gm[s][1];
        if (DIM == 3) sn = sn + nrm[2] * gm[s][2];
#pragma unroll
        for (int c = 0; c < DIM; ++c) gp[s][c] = gm[s][c] - T(2) * sn * nrm[c];
      }
      T un = nrm[0] * vM_[0] + nrm[1] * vM_[1];
      if (DIM == 3) un = un + nrm[2] * vM_[2];
#pragma unroll
      for (int c = 0; c < DIM; ++c) vP_[c] = vM_[c] - T(2) * un * nrm[c];
#pragma unroll
      for (int c = 0; c < DIM; ++c) gp[IE][c] = gm[IE][c];
    } else {
      atomicOr(status, ST_BC);
      for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = T(0);
      continue;
    }
    T fM[NS][DIM], fP[NS][DIM];
    visc_flux<DIM, T>(gm, vM_, p, fM);
    visc_flux<DIM, T>(gp, vP_, p, fP);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      T a = nrm[0] * (fM[s][0] + fP[s][0]) + nrm[1] * (fM[s][1] + fP[s][1]);
      if (DIM == 3) a = a + nrm[2] * (fM[s][2] + fP[s][2]);
      FF[(f * NS + s) * FS + el * Nfp + fn] = sMJ * (T(0.5) * a);
    }
  }
  __syncthreads();
  for (int slot = threadIdx.x; slot < C::SLOTS; slot += C::THREADS) {
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (e >= nelem) continue;
    const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
    const bool onface = i == 0 || i == Nq - 1 || j == 0 || j == Nq - 1 ||
                        (DIM == 3 && (k == 0 || k == Nq - 1));
    if (!onface) continue;
    // rhs += Σ_f FF, faces in reference order
    for (int s = 0; s < NS; ++s) {
      T *dst = rhs + n + Np * (s + NS * (0 + (int64_t)DIM * e));
      T v = *dst;
      if (i == 0) v += FF[(0 * NS + s) * FS + el * Nfp + (DIM == 3 ? j + Nq * k : j)];
      if (i == Nq - 1) v += FF[(1 * NS + s) * FS + el * Nfp + (DIM == 3 ? j + Nq * k : j)];
      if (j == 0) v += FF[(2 * NS + s) * FS + el * Nfp + (DIM == 3 ? i + Nq * k : i)];
      if (j == Nq - 1) v += FF[(3 * NS + s) * FS + el * Nfp + (DIM == 3 ? i + Nq * k : i)];
      if (DIM == 3 && k == 0) v += FF[(4 * NS + s) * FS + el * Nfp + i + Nq * j];
      if (DIM == 3 && k == Nq - 1) v += FF[(5 * NS + s) * FS + el * Nfp + i + Nq * j];
      *dst = v;
    }
  }
}

// Compensated FP64 sums of MJ·Q and MJ·Q² per state field.  Every thread
// keeps Neumaier (sum, compensation) pairs; pairs are merged with an exact
// two-sum across the warp and the block, and each block writes 4*NS doubles
// (sum, comp for MJ·Q and for MJ·Q²) that the host merges the same way.
__device__ __forceinline__ void neu_add(double &sum, double &comp, double v) {
  const double t = sum + v;
  if (fabs(sum) >= fabs(v)) comp += (sum - t) + v;
  else comp += (v - t) + sum;
  sum = t;
}
__device__ __forceinline__ void neu_merge(double &sum, double &comp, double s2, double c2) {
  neu_add(sum, comp, s2);
  comp += c2;
}
template <int DIM, typename T>
__global__ void __launch_bounds__(256) k_cons_sums(const T *__restrict__ Q, const T *__restrict__ vgeo,
                                                   int64_t nelem, int Np, Offs<double, Lay<DIM>::NS> qref,
                                                   double *__restrict__ part) {
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, MJ = DIM * DIM;
  double acc[4 * NS];
  for (int s = 0; s < 4 * NS; ++s) acc[s] = 0.0;
  const int64_t total = (int64_t)Np * nelem;
  for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total;
       q += (int64_t)gridDim.x * blockDim.x) {
    const int64_t n = q % Np, e = q / Np;
    const double mj = (double)vgeo[n + Np * (MJ + (int64_t)NVG * e)];
    for (int s = 0; s < NS; ++s) {
      const double v = (double)Q[n + Np * (s + (int64_t)NS * e)] + qref.v[s];
      neu_add(acc[4 * s + 0], acc[4 * s + 1], mj * v);
      neu_add(acc[4 * s + 2], acc[4 * s + 3], mj * (v * v));
    }
  }
  for (int off = 16; off > 0; off >>= 1)
    for (int s = 0; s < 2 * NS; ++s) {
      const double so = __shfl_down_sync(0xffffffffu, acc[2 * s], off);
      const double co = __shfl_down_sync(0xffffffffu, acc[2 * s + 1], off);
      neu_merge(acc[2 * s], acc[2 * s + 1], so, co);
    }
  __shared__ double red[8][4 * NS];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0)
    for (int s = 0; s < 4 * NS; ++s) red[warp][s] = acc[s];
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    for (int w = 1; w < nw; ++w)
      for (int s = 0; s < 2 * NS; ++s) neu_merge(red[0][2 * s], red[0][2 * s + 1], red[w][2 * s], red[w][2 * s + 1]);
    for (int s = 0; s < 4 * NS; ++s) part[blockIdx.x * (int64_t)(4 * NS) + s] = red[0][s];
  }
}

// Rounds an FP64 array to FP32.
__global__ void k_round_f32(float *__restrict__ dst, const double *__restrict__ src, int64_t n);

}  // namespace cb
#include "cb_pipe.cuh"
#include "cb_pipe2.cuh"
#include "cb_mma.cuh"
#include "cb_ns_pipe.cuh"
#include "cb_lean.cuh"
namespace cb {

// ---------------------------------------------------------------- launchers
template <int DIM, int Nq, typename T>
struct Launch {
  using C = Cfg<DIM, Nq>;
  static constexpr int NS = Lay<DIM>::NS;
  static size_t smem_volume() { return sizeof(T) * (((Nq * Nq + 1) & ~1) + (size_t)DIM * NS * C::SLOTS); }
  static size_t smem_stage() { return sizeof(T) * (((Nq * Nq + 1) & ~1) + (size_t)NS * C::SLOTS + (size_t)DIM * NS * C::SLOTS); }
  static size_t smem_face() { return sizeof(T) * (size_t)C::NFACE * NS * C::EPB * C::Nfp; }
  static size_t smem_face_grad() { return sizeof(T) * (size_t)C::NFACE * NS * DIM * C::EPB * C::Nfp; }
  static int grid(int64_t nelem) { return (int)((nelem + C::EPB - 1) / C::EPB); }

  template <typename K>
  static cudaError_t prep(K kernel, size_t smem) {
    if (smem > 48 * 1024) return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    return cudaSuccess;
  }

  static cudaError_t volumerhs(T *rhs, const T *Q, const T *vgeo, const T *D, int64_t nelem,
                               const PhysT<T> &p, cudaStream_t st) {
    size_t sm = smem_volume();
    cudaError_t err = prep(k_volumerhs<DIM, Nq, T>, sm);
    if (err != cudaSuccess) return err;
    k_volumerhs<DIM, Nq, T><<<grid(nelem), C::THREADS, sm, st>>>(rhs, Q, vgeo, D, nelem, p);
    return cudaGetLastError();
  }
  static cudaError_t fluxrhs(T *rhs, const T *Q, const T *sgeo, const T *vgeo, int64_t nelem,
                             const int64_t *vmapM, const int64_t *vmapP, const int64_t *bnd,
                             const PhysT<T> &p, unsigned *status, cudaStream_t st) {
    size_t sm = smem_face();
    cudaError_t err = prep(k_fluxrhs<DIM, Nq, T>, sm);
    if (err != cudaSuccess) return err;
    k_fluxrhs<DIM, Nq, T><<<grid(nelem), C::THREADS, sm, st>>>(rhs, Q, sgeo, vgeo, nelem, vmapM,
                                                                vmapP, bnd, p, status);
    return cudaGetLastError();
  }
  // Whether the tensor-core (DMMA) stage is built for this shape.
  static constexpr bool MMA_OK = DIM == 3 && Nq == 8;
  // Whether kernel 0 (the shape's default) is the tensor-core stage: the
  // faster of the two on B200 at the benchmark size.
  static constexpr bool MMA_DEFAULT = MMA_OK && PipeMT<T>::DEFAULT;
  // Whether the lean pipelined stage is built for this shape, and whether it
  // is the shape's default (where the tensor-core stage is not).
  static constexpr bool LEAN_OK = Lean<DIM, Nq, T>::OK;
  // Default stage kernel per shape, from B200 timings of one mesh (ms per
  // step, warped 3-D cubes of 7-17 M nodes; pipelined CUDA-core / grouped /
  // lean): FP64 N=3 3.66 / 3.34 / 2.76, N=4 4.95 / 4.20 / 3.78, N=5 2.37 /
  // 3.45 / 2.67, N=6 3.37 / 5.13 / 3.83, N=8 5.78 / 5.71 / 5.33; FP32 N=3
  // 1.34 / 1.31 / 1.66, N=4 2.61 / 1.75 / 2.26, N=5 1.65 / 1.44 / 1.72, N=6
  // 2.02 / 1.68 / 2.61, N=8 3.08 / 2.61 / 3.44, N=9 2.22 / 1.93 / 2.45 (the
  // FP32 pipelined plans fit fewer blocks per SM than the grouped stage;
  // FP64 N=8, 9 have no pipelined plan that fits shared memory, so their
  // first figure is the grouped stage as well).  3-D N=7 runs the
  // tensor-core stage in both precisions.
  static constexpr int DEFAULT_KERNEL =
      MMA_DEFAULT ? 2
      : DIM == 3 && sizeof(T) == 8 && LEAN_OK && (Nq == 4 || Nq == 5 || Nq == 9) ? 4
      : DIM == 3 && sizeof(T) == 4 && Nq >= 4 && Nq <= 10 ? 3
      : 1;
  static constexpr bool LEAN_DEFAULT = DEFAULT_KERNEL == 4;
  // Resident blocks per SM of a kernel at `smem` bytes, from the occupancy
  // calculator, cached per device in `cache`.
  template <typename K>
  static cudaError_t blocks_per_sm(K kernel, int threads, size_t smem, int *cache, int *out) {
    int dev = 0;
    cudaError_t err = cudaGetDevice(&dev);
    if (err != cudaSuccess) return err;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    if (!cache[dev]) {
      err = prep(kernel, smem);
      if (err != cudaSuccess) return err;
      int v = 0;
      err = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, kernel, threads, smem);
      if (err != cudaSuccess) return err;
      cache[dev] = v < 1 ? 1 : v;
    }
    *out = cache[dev];
    return cudaSuccess;
  }
  // kernel: 0 = the default for the shape (DEFAULT_KERNEL), 1 = the
  // CUDA-core stages only, 2 = the tensor-core stage (cudaErrorNotSupported
  // where it is not built), 3 = the unpipelined grouped stage k_stage, 4 =
  // the lean pipelined stage k_stage_lean (state-only staging; the pipelined
  // stage where the arrays are not 16-byte aligned).  probe != 0: the timeout
  // test hook of the pipelined, lean and tensor-core stages (see MeshSrc);
  // shapes without one return cudaErrorNotSupported for it.
  // ebeg: the launch covers elements ebeg .. nelem - 1 (neighbour indices
  // stay absolute); only the pipelined, lean and tensor-core stages take
  // ebeg > 0, the others return cudaErrorNotSupported for it.
  static cudaError_t stage(const T *Qin, T *Qout, T *rhs, const T *vgeo, const T *sgeo,
                           const int32_t *nbr, const T *D, int64_t nelem, const PhysT<T> &p,
                           const Offs<T, NS> &qref, T rka, T rkbdt, unsigned *status,
                           cudaStream_t st, int probe = 0, int kernel = 0, int64_t ebeg = 0) {
    constexpr bool pipe_ok = Pipe<DIM, Nq, T>::OK;
    const bool aligned = ((reinterpret_cast<uintptr_t>(Qin) | reinterpret_cast<uintptr_t>(vgeo)) & 15) == 0;
    const bool aligned2 = aligned && ((reinterpret_cast<uintptr_t>(rhs) | reinterpret_cast<uintptr_t>(sgeo)) & 15) == 0;
    // the shape's default; the grouped stage takes no element range and no
    // test hook: those calls take the pipelined stage, or the lean one where
    // the pipelined plan does not fit shared memory (3-D N=9 FP64, N=10 FP32)
    if (kernel == 0 && (probe || ebeg) && (DEFAULT_KERNEL == 1 || DEFAULT_KERNEL == 3))
      kernel = (Pipe2<DIM, Nq, T>::OK || !LEAN_OK) ? 1 : 4;
    else if (kernel == 0 && DEFAULT_KERNEL == 3)
      kernel = 3;
    if (kernel == 2 && !(MMA_OK && aligned2)) return cudaErrorNotSupported;
    if (kernel == 4 && !LEAN_OK) return cudaErrorNotSupported;
    if (kernel == 4 && !aligned2) kernel = 1;  // bulk copies need 16-byte aligned slabs
    if (ebeg < 0 || ebeg > nelem) return cudaErrorInvalidValue;
    const int64_t groups = (nelem - ebeg + C::EPB - 1) / C::EPB;
    if (groups == 0) return cudaSuccess;
    if constexpr (MMA_OK) {
      if ((kernel == 2 || (kernel == 0 && MMA_DEFAULT)) && aligned2) {
        using S = MeshSrc<T, NS, C::EPB>;  // MeshSrc<T, 5, 1> here
        using PM = PipeMT<T>;
        static int per_sm[MAX_DEVICES] = {0};
        int bps = 0;
        cudaError_t err = blocks_per_sm(k_stage_mma<S, PM::MINB>, PM::THREADS, PM::smem(), per_sm, &bps);
        if (err != cudaSuccess) return err;
        int64_t g = (int64_t)num_sms() * bps;
        if (g > groups) g = groups;
        const S src{Qin, Qout, rhs, vgeo, sgeo, nbr, D, nelem, qref, rkbdt, status, probe, ebeg};
        k_stage_mma<S, PM::MINB><<<(int)g, PM::THREADS, PM::smem(), st>>>(src, p, rka);
        return cudaGetLastError();
      }
    }
    if constexpr (LEAN_OK) {
      if (kernel == 4 || (kernel == 0 && LEAN_DEFAULT && aligned2)) {
        using S = MeshSrc<T, NS, C::EPB>;
        using PL = Lean<DIM, Nq, T>;
        static int per_sm[MAX_DEVICES] = {0};
        int bps = 0;
        cudaError_t err = blocks_per_sm(k_stage_lean<DIM, Nq, T, S>, C::THREADS, PL::smem(), per_sm, &bps);
        if (err != cudaSuccess) return err;
        int64_t g = (int64_t)num_sms() * bps;
        if (g > groups) g = groups;
        const S src{Qin, Qout, rhs, vgeo, sgeo, nbr, D, nelem, qref, rkbdt, status, probe, ebeg};
        k_stage_lean<DIM, Nq, T, S><<<(int)g, C::THREADS, PL::smem(), st>>>(src, p, rka);
        return cudaGetLastError();
      }
    }
    if (Pipe2<DIM, Nq, T>::OK && aligned2 && kernel != 3) {
      using PP = Pipe2<DIM, Nq, T>;
      using S = MeshSrc<T, NS, C::EPB>;
      const size_t sm = PP::smem();
      static int per_sm[MAX_DEVICES] = {0};
      int bps = 0;
      cudaError_t err = blocks_per_sm(k_stage_pipe2<DIM, Nq, T, S>, C::THREADS, sm, per_sm, &bps);
      if (err != cudaSuccess) return err;
      int64_t g = (int64_t)num_sms() * bps;
      if (g > groups) g = groups;
      const S src{Qin, Qout, rhs, vgeo, sgeo, nbr, D, nelem, qref, rkbdt, status, probe, ebeg};
      k_stage_pipe2<DIM, Nq, T, S><<<(int)g, C::THREADS, sm, st>>>(src, p, rka);
      return cudaGetLastError();
    } else if (probe || ebeg) {
      return cudaErrorNotSupported;
    } else if (pipe_ok && aligned && kernel != 3) {
      using PP = Pipe<DIM, Nq, T>;
      size_t sm = PP::smem();
      cudaError_t err = prep(k_stage_pipe<DIM, Nq, T>, sm);
      if (err != cudaSuccess) return err;
      int g = num_sms();
      if ((int64_t)g > groups) g = (int)groups;
      k_stage_pipe<DIM, Nq, T><<<g, C::THREADS, sm, st>>>(Qin, Qout, rhs, vgeo, sgeo, nbr, D, nelem,
                                                          p, qref, rka, rkbdt, status);
      return cudaGetLastError();
    } else {
      size_t sm = smem_stage();
      cudaError_t err = prep(k_stage<DIM, Nq, T>, sm);
      if (err != cudaSuccess) return err;
      k_stage<DIM, Nq, T><<<grid(nelem), C::THREADS, sm, st>>>(Qin, Qout, rhs, vgeo, sgeo, nbr, D,
                                                                nelem, p, qref, rka, rkbdt, status);
      return cudaGetLastError();
    }
  }
  // Whether stage() takes an element range (ebeg > 0) for arrays aligned
  // like these.
  static bool ranged(const void *Qin, const void *rhs, const void *vgeo, const void *sgeo) {
    const bool a = ((reinterpret_cast<uintptr_t>(Qin) | reinterpret_cast<uintptr_t>(rhs) |
                     reinterpret_cast<uintptr_t>(vgeo) | reinterpret_cast<uintptr_t>(sgeo)) & 15) == 0;
    return a && (Pipe2<DIM, Nq, T>::OK || MMA_OK || LEAN_OK);
  }
  static cudaError_t build_nbr(int32_t *nbr, const int64_t *vmapM, const int64_t *vmapP,
                               const int64_t *bnd, int64_t nelem, unsigned *status,
                               cudaStream_t st) {
    const int64_t n = nelem * C::NFACE;
    k_build_nbr<DIM, Nq><<<(int)((n + 255) / 256), 256, 0, st>>>(nbr, vmapM, vmapP, bnd, nelem, nelem, status);
    return cudaGetLastError();
  }
  static cudaError_t build_nbr_ghost(int32_t *nbr, const int64_t *vmapM, const int64_t *vmapP,
                                     const int64_t *bnd, int64_t nelem, int64_t nall, unsigned *status,
                                     cudaStream_t st) {
    const int64_t n = nelem * C::NFACE;
    k_build_nbr<DIM, Nq><<<(int)((n + 255) / 256), 256, 0, st>>>(nbr, vmapM, vmapP, bnd, nelem, nall, status);
    return cudaGetLastError();
  }
  static cudaError_t volume_grad(T *rhs, const T *Q, const T *vgeo, const T *D, int64_t nelem,
                                 const PhysT<T> &p, cudaStream_t st) {
    size_t sm = smem_volume();
    cudaError_t err = prep(k_volume_grad<DIM, Nq, T>, sm);
    if (err != cudaSuccess) return err;
    k_volume_grad<DIM, Nq, T><<<grid(nelem), C::THREADS, sm, st>>>(rhs, Q, vgeo, D, nelem, p);
    return cudaGetLastError();
  }
  static cudaError_t flux_grad(T *rhs, const T *Q, const T *sgeo, const T *vgeo, int64_t nelem,
                               const int64_t *vmapM, const int64_t *vmapP, const int64_t *bnd,
                               const PhysT<T> &p, unsigned *status, cudaStream_t st) {
    size_t sm = smem_face_grad();
    cudaError_t err = prep(k_flux_grad<DIM, Nq, T>, sm);
    if (err != cudaSuccess) return err;
    k_flux_grad<DIM, Nq, T><<<grid(nelem), C::THREADS, sm, st>>>(rhs, Q, sgeo, vgeo, nelem, vmapM,
                                                                  vmapP, bnd, p, status);
    return cudaGetLastError();
  }
  static cudaError_t volume_div(T *rhs, const T *gradQ, const T *Q, const T *vgeo, const T *D,
                                int64_t nelem, const PhysT<T> &p, cudaStream_t st) {
    size_t sm = smem_volume();
    cudaError_t err = prep(k_volume_div<DIM, Nq, T>, sm);
    if (err != cudaSuccess) return err;
    k_volume_div<DIM, Nq, T><<<grid(nelem), C::THREADS, sm, st>>>(rhs, gradQ, Q, vgeo, D, nelem, p);
    return cudaGetLastError();
  }
  static cudaError_t flux_div(T *rhs, const T *gradQ, const T *Q, const T *sgeo, int64_t nelem,
                              const int64_t *vmapM, const int64_t *vmapP, const int64_t *bnd,
                              const PhysT<T> &p, unsigned *status, cudaStream_t st) {
    size_t sm = smem_face();
    cudaError_t err = prep(k_flux_div<DIM, Nq, T>, sm);
    if (err != cudaSuccess) return err;
    k_flux_div<DIM, Nq, T><<<grid(nelem), C::THREADS, sm, st>>>(rhs, gradQ, Q, sgeo, nelem, vmapM,
                                                                 vmapP, bnd, p, status);
    return cudaGetLastError();
  }
};

}  // namespace cb
