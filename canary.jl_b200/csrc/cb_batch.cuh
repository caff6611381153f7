// Kernels and device-side types of the batched LSRK driver (cb_batch.cu).
// The stage kernels of each (dim, precision) are instantiated in their own
// translation unit (cb_batch_<dim>d_<prec>.cu) through b_fill_dim.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

#include "cb_kernels.cuh"

namespace cb {

constexpr int BT = 256;                // threads per block of the grouped stage
constexpr int BMAXN2 = 8, BMAXN3 = 7;  // orders compiled into the batched stage

// Shape of the grouped (non-pipelined) stage for (dim, Nq) at BT threads:
// groups of about 256 (G = 0) or 512 (G = 1) nodes.
template <int DIM, int Nq, int G>
struct BCfg {
  static constexpr int Np = ipow(Nq, DIM), Nfp = ipow(Nq, DIM - 1), NFACE = 2 * DIM;
  static constexpr int BASE = Np >= BT ? 1 : BT / Np;
  static constexpr int EPB = BASE * (G + 1);
  static constexpr int SLOTS = EPB * Np;
  static constexpr int NPT = cdiv(SLOTS, BT);
  static constexpr int FSLOTS = EPB * NFACE * Nfp;
  static constexpr int FPT = cdiv(FSLOTS, BT);
  static constexpr bool OK = NPT <= 2;  // variants with more nodes per thread are not built
};

// Descriptor of one admitted instance (one per slot; the table is small and
// stays in cache).  At batch step k the instance has taken k - start steps; it
// is advanced while that is below `target`, and its current state is
// Q[(k - start + stage) mod 2] at stage `stage`.
template <typename T>
struct alignas(16) BDesc {
  T *Q[2];  // Q[0]: the caller's state, Q[1]: the batch-owned twin
  T *rhs;   // residual carry (caller's)
  const T *vgeo, *sgeo, *D;
  const int32_t *nbr;
  unsigned *status;  // the instance's status word
  T *gq;             // gradient buffer (viscous batches)
  int64_t start, target;
  double dt;
  T qref[5];
};
// One work item: a group of `nv` consecutive elements (from e0) of the
// instance in `slot`; written when the instance is admitted (valid = 1, or 3
// for the instance's last group) and invalidated (valid = 0) when it is
// released.
struct alignas(16) BWork {
  int32_t slot, e0, nv, valid;
};

// Stage variants per (dim, N): 0 pipelined (k_stage_pipe2, groups of
// Cfg::EPB elements staged one group ahead, default occupancy), 1 / 2
// grouped (~256 / ~512 nodes), 3 / 4 pipelined at other occupancies,
// VAR_DEEP pipelined with copies two groups ahead, VAR_WIDE pipelined with
// twice the elements per group on 512-thread blocks, VAR_NPT2 pipelined with
// two nodes per thread (half the threads), and the affine-element stages
// (affine-element geometry, copies two groups ahead) VAR_AFFINE and
// VAR_AFFINE_NPT2 (two nodes per thread).  Affine variants run only on
// meshes whose elements are all affine (gravity off); when no variant was
// chosen for a shape the batch uses VAR_AFFINE in place of its default
// pipelined variant for such meshes.  VAR_MMA
// is the tensor-core stage (k_stage_mma, 3-D N = 7), VAR_LEAN the lean
// pipelined stage (k_stage_lean: only the state staged in shared memory).
constexpr int VAR_AFFINE = 5, VAR_DEEP = 6, VAR_WIDE = 7, VAR_NPT2 = 8, VAR_AFFINE_NPT2 = 9, VAR_MMA = 10,
              VAR_LEAN = 11, NVAR = 12;
__host__ __device__ constexpr bool var_affine(int var) { return var == VAR_AFFINE || var == VAR_AFFINE_NPT2; }
// Shape id of (dim, N, variant); ids of shapes that are not built stay
// unused.
constexpr int NSHAPE = 2 * NVAR * (BMAXN2 + 1);
__host__ __device__ constexpr int shape_id(int dim, int N, int var) {
  return (dim - 2) * NVAR * (BMAXN2 + 1) + NVAR * N + var;
}
// Device header: the instance table (BDesc<T>[slots]), the work list of
// every shape and the batch step counter.
struct BHdr {
  void *desc;
  BWork *work[NSHAPE];
  int32_t nwork[NSHAPE];
  int64_t step;
  void *gq;  // viscous batches: per slot the instance's gradient buffer (T *)
};

// One group of the fused stage (volume + face + LSRK update) of one instance.
template <int DIM, int Nq, int G, typename T>
__device__ __forceinline__ void stage_group(const BDesc<T> &I, int64_t e0, int nv, int par, const PhysT<T> &p,
                                            T rka, T rkbdt, unsigned char *smem) {
  using C = BCfg<DIM, Nq, G>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, SP = C::SLOTS, FS = C::EPB * Nfp;
  constexpr int MJI = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  const T *__restrict__ Qin = I.Q[par];
  T *__restrict__ Qout = I.Q[par ^ 1];
  T *__restrict__ rhs = I.rhs;
  const T *__restrict__ vgeo = I.vgeo;
  T *Ds = reinterpret_cast<T *>(smem);
  T *sQ = Ds + ((Nq * Nq + 1) & ~1);  // [NS][SP]
  T *sF = sQ + NS * SP;               // [DIM][NS][SP], reused as the face buffer
  for (int t = threadIdx.x; t < Nq * Nq; t += BT) Ds[t] = I.D[t];
  T R[C::NPT][NS];
  // ---- pointwise contravariant fluxes
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * BT;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < SP && el < nv) {
      T q[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const T d = Qin[n + Np * (s + NS * e)];
        sQ[s * SP + slot] = d;
        q[s] = d + I.qref[s];
        R[u][s] = rhs[n + Np * (s + NS * e)];
      }
      const T *vg = vgeo + (int64_t)Np * NVG * e;
      T met[DIM][DIM], MJ;
      load_metric<DIM, T>(vg, n, Np, met, MJ);
      const T gc = p.grav != T(0) ? vg[n + Np * GC] : T(0);
      const T ri = T(1) / q[IR];
      const T P = pressure_ri<DIM, T>(q, ri, gc, p);
      T f[NS][DIM];
      euler_flux_ri<DIM, T>(q, ri, P, f);
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          T a = met[r][0] * f[s][0] + met[r][1] * f[s][1];
          if (DIM == 3) a = a + met[r][2] * f[s][2];
          sF[(r * NS + s) * SP + el * Np + n] = MJ * a;
        }
      R[u][DIM - 1] -= MJ * q[IR] * p.grav;
    }
  }
  __syncthreads();
  // ---- volume contraction
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * BT;
    const int el = slot / Np, n = slot % Np;
    if (slot < SP && el < nv) contract<DIM, Nq, C::EPB, T>(sF, Ds, el, n, R[u]);
  }
  __syncthreads();
  // ---- face fluxes into FF[NF][NS][EPB*Nfp] (aliases sF)
  T *FF = sF;
#pragma unroll
  for (int u = 0; u < C::FPT; ++u) {
    const int fs = threadIdx.x + u * BT;
    if (fs >= C::FSLOTS) break;
    const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
    const int64_t e = e0 + el;
    if (el >= nv) continue;
    const int vM = face_node<DIM, Nq>(f, fn);
    const T *sg = I.sgeo + (int64_t)NSG * (fn + (int64_t)Nfp * (f + NF * e));
    T nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
    const T smj = sg[DIM];
    T qM[NS], qP[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qM[s] = sQ[s * SP + el * Np + vM] + I.qref[s];
    const T gM = p.grav != T(0) ? vgeo[vM + Np * (GC + NVG * e)] : T(0);
    const T riM = T(1) / qM[IR];
    const T PM = pressure_ri<DIM, T>(qM, riM, gM, p);
    const int32_t nb = I.nbr[f + NF * e];
    T PP, riP;
    if (nb >= 0) {
      const int64_t e2 = nb >> 3;
      const int vP = face_node<DIM, Nq>(nb & 7, fn);
#pragma unroll
      for (int s = 0; s < NS; ++s) qP[s] = Qin[vP + Np * (s + NS * e2)] + I.qref[s];
      const T gP = p.grav != T(0) ? vgeo[vP + Np * (GC + NVG * e2)] : T(0);
      riP = T(1) / qP[IR];
      PP = pressure_ri<DIM, T>(qP, riP, gP, p);
    } else {
      wall_state<DIM, T>(qM, nrm, qP);
      riP = riM;
      PP = PM;
    }
    T out[NS];
    rusanov_n<DIM, T>(qM, riM, PM, qP, riP, PP, nrm, p, out);
#pragma unroll
    for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = smj * out[s];
  }
  __syncthreads();
  // ---- face accumulation and LSRK update
  bool bad = false;
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * BT;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < SP && el < nv) {
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
  if (bad) atomicOr(I.status, ST_NONFINITE);
  __syncthreads();  // shared memory is reused by the block's next item
}

// Persistent grouped stage kernel of one shape: the blocks stride over the
// shape's work list.
template <int DIM, int Nq, int G, typename T>
__global__ void __launch_bounds__(BT, 2)
k_stage_batch(const BHdr *__restrict__ hdr, int stage, PhysT<T> p, T rka, double rkb) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int SID = shape_id(DIM, Nq - 1, 1 + G);
  const int nwork = hdr->nwork[SID];
  const int64_t step = hdr->step;
  const BWork *__restrict__ work = hdr->work[SID];
  const BDesc<T> *__restrict__ desc = static_cast<const BDesc<T> *>(hdr->desc);
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const BWork it = work[w];
    if (!it.valid) continue;  // uniform over the block
    const BDesc<T> &I = desc[it.slot];
    const int64_t k = step - I.start;
    if (k >= I.target) continue;
    stage_group<DIM, Nq, G, T>(I, it.e0, it.nv, (int)((k + stage) & 1), p, rka, T(rkb * I.dt), smem_raw);
  }
}

// ---------------------------------------------------------------- viscous
// LDG Navier–Stokes stage of a viscous batch, in two grouped passes per RK
// stage instead of the reference's six (volume_grad!, flux_grad!,
// update_gradQ!, volume_div!, flux_div!, updatesolution! with the inviscid
// volumerhs!/fluxrhs!: nse3d.jl:475-955, nse2d.jl:396-778, nse2d.jl:1826-1849):
//   grad:  gQ[:, s, c, e] = MJI (-Σ Dᵀ (MJ ξ_c prim_s) + Σ_f sMJ n_c avg_f prim_s)
//          for the primitives (u, v, [w], ρ, T), written to the instance's
//          gradient buffer (Np, nstate, dim, nelem);
//   stage: the fused inviscid stage with the viscous flux folded in — flux
//          rows MJ ξ·F_inv - μ MJ ξ·F_visc(gQ), face terms sMJ (Rusanov -
//          μ n·(F_visc⁻ + F_visc⁺)/2) — then the LSRK update.
// The viscous contributions are summed with the inviscid ones instead of in
// a separate residual (the reference adds μ·rhs_gradQ at the update): the
// same terms, rounded in another order.

// Gradient pass of one group: gq of elements e0 .. e0 + nv - 1.
template <int DIM, int Nq, typename T>
__device__ __forceinline__ void ns_grad_group(const BDesc<T> &I, T *__restrict__ gq, int64_t e0, int nv, int par,
                                              const PhysT<T> &p, unsigned char *smem) {
  using C = BCfg<DIM, Nq, 0>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, SP = C::SLOTS, FS = C::EPB * Nfp, ND = NS * DIM;
  constexpr int MJI = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  const T *__restrict__ Qin = I.Q[par];
  const T *__restrict__ vgeo = I.vgeo;
  T *Ds = reinterpret_cast<T *>(smem);
  T *sQ = Ds + ((Nq * Nq + 1) & ~1);  // [NS][SP] state (offsets added)
  T *sF = sQ + NS * SP;               // [DIM][NS][SP] rows of one gradient component
  T *FF = sF + DIM * NS * SP;         // [NF][NS*DIM][FS] face terms sMJ n_c (prim⁻ + prim⁺)/2
  for (int t = threadIdx.x; t < Nq * Nq; t += BT) Ds[t] = I.D[t];
  T prim[C::NPT][NS], met[C::NPT][DIM][DIM], MJ[C::NPT];
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * BT;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < SP && el < nv) {
      T q[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        q[s] = Qin[n + Np * (s + NS * e)] + I.qref[s];
        sQ[s * SP + slot] = q[s];
      }
      const T *vg = vgeo + (int64_t)Np * NVG * e;
      load_metric<DIM, T>(vg, n, Np, met[u], MJ[u]);
      const T gc = p.grav != T(0) ? vg[n + Np * GC] : T(0);
      primitives<DIM, T>(q, gc, p, prim[u]);
    }
  }
  __syncthreads();
  // ---- face averages of the primitives (flux_grad!)
  for (int fs = threadIdx.x; fs < C::FSLOTS; fs += BT) {
    const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
    if (el >= nv) continue;
    const int64_t e = e0 + el;
    const int vM = face_node<DIM, Nq>(f, fn);
    const T *sg = I.sgeo + (int64_t)NSG * (fn + (int64_t)Nfp * (f + NF * e));
    T nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
    const T sMJ = sg[DIM];
    T qM[NS], pM[NS], pP[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qM[s] = sQ[s * SP + el * Np + vM];
    const T gM = p.grav != T(0) ? vgeo[vM + Np * (GC + NVG * e)] : T(0);
    primitives<DIM, T>(qM, gM, p, pM);
    const int32_t nb = I.nbr[f + NF * e];
    if (nb >= 0) {
      const int64_t e2 = nb >> 3;
      const int vP = face_node<DIM, Nq>(nb & 7, fn);
      T qP[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) qP[s] = Qin[vP + Np * (s + NS * e2)] + I.qref[s];
      const T gP = p.grav != T(0) ? vgeo[vP + Np * (GC + NVG * e2)] : T(0);
      primitives<DIM, T>(qP, gP, p, pP);
    } else {  // reflective wall: mirrored velocity, same density and temperature
      T qP[NS];
      wall_state<DIM, T>(qM, nrm, qP);
#pragma unroll
      for (int c = 0; c < DIM; ++c) pP[c] = qP[c] / qM[IR];
      pP[IR] = qM[IR];
      pP[IE] = pM[IE];
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const T fsv = T(0.5) * (pM[s] + pP[s]);
#pragma unroll
      for (int c = 0; c < DIM; ++c) FF[(f * ND + s * DIM + c) * FS + el * Nfp + fn] = sMJ * nrm[c] * fsv;
    }
  }
  // ---- per gradient component: volume term, face terms in face order, × MJI
  for (int c = 0; c < DIM; ++c) {
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = threadIdx.x + u * BT;
      const int el = slot / Np, n = slot % Np;
      if (slot < SP && el < nv)
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int s = 0; s < NS; ++s) sF[(r * NS + s) * SP + el * Np + n] = MJ[u] * (met[u][r][c] * prim[u][s]);
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = threadIdx.x + u * BT;
      const int el = slot / Np, n = slot % Np;
      const int64_t e = e0 + el;
      if (slot < SP && el < nv) {
        T R[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) R[s] = T(0);
        contract_sub<DIM, Nq, C::EPB, T>(sF, Ds, el, n, R);
        const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
        auto add = [&](int f, int fn) {
#pragma unroll
          for (int s = 0; s < NS; ++s) R[s] += FF[(f * ND + s * DIM + c) * FS + el * Nfp + fn];
        };
        if (i == 0) add(0, DIM == 3 ? j + Nq * k : j);
        if (i == Nq - 1) add(1, DIM == 3 ? j + Nq * k : j);
        if (j == 0) add(2, DIM == 3 ? i + Nq * k : i);
        if (j == Nq - 1) add(3, DIM == 3 ? i + Nq * k : i);
        if (DIM == 3 && k == 0) add(4, i + Nq * j);
        if (DIM == 3 && k == Nq - 1) add(5, i + Nq * j);
        const T mji = vgeo[n + Np * (MJI + (int64_t)NVG * e)];
#pragma unroll
        for (int s = 0; s < NS; ++s) gq[n + Np * (s + NS * (c + (int64_t)DIM * e))] = R[s] * mji;
      }
    }
    __syncthreads();  // sF is rewritten for the next component; the last one frees shared memory
  }
}

// Stage pass of one group: inviscid + viscous residual and the LSRK update.
template <int DIM, int Nq, typename T>
__device__ __forceinline__ void ns_stage_group(const BDesc<T> &I, const T *__restrict__ gq, int64_t e0, int nv,
                                               int par, const PhysT<T> &p, T rka, T rkbdt, unsigned char *smem) {
  using C = BCfg<DIM, Nq, 0>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, SP = C::SLOTS, FS = C::EPB * Nfp;
  constexpr int MJI = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  const T *__restrict__ Qin = I.Q[par];
  T *__restrict__ Qout = I.Q[par ^ 1];
  T *__restrict__ rhs = I.rhs;
  const T *__restrict__ vgeo = I.vgeo;
  T *Ds = reinterpret_cast<T *>(smem);
  T *sQ = Ds + ((Nq * Nq + 1) & ~1);  // [NS][SP] stored state (without offsets)
  T *sF = sQ + NS * SP;               // [DIM][NS][SP], reused as the face buffer
  for (int t = threadIdx.x; t < Nq * Nq; t += BT) Ds[t] = I.D[t];
  T R[C::NPT][NS];
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * BT;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < SP && el < nv) {
      T q[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        const T d = Qin[n + Np * (s + NS * e)];
        sQ[s * SP + slot] = d;
        q[s] = d + I.qref[s];
        R[u][s] = rhs[n + Np * (s + NS * e)];
      }
      const T *vg = vgeo + (int64_t)Np * NVG * e;
      T met[DIM][DIM], MJ;
      load_metric<DIM, T>(vg, n, Np, met, MJ);
      const T gc = p.grav != T(0) ? vg[n + Np * GC] : T(0);
      const T ri = T(1) / q[IR];
      const T P = pressure_ri<DIM, T>(q, ri, gc, p);
      T f[NS][DIM];
      euler_flux_ri<DIM, T>(q, ri, P, f);
      T g[NS][DIM], vel[DIM], fv[NS][DIM];
#pragma unroll
      for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int c = 0; c < DIM; ++c) g[s][c] = gq[n + Np * (s + NS * (c + (int64_t)DIM * e))];
#pragma unroll
      for (int c = 0; c < DIM; ++c) vel[c] = q[c] / q[IR];
      visc_flux<DIM, T>(g, vel, p, fv);
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          T a = met[r][0] * f[s][0] + met[r][1] * f[s][1];
          T b = met[r][0] * fv[s][0] + met[r][1] * fv[s][1];
          if (DIM == 3) {
            a = a + met[r][2] * f[s][2];
            b = b + met[r][2] * fv[s][2];
          }
          sF[(r * NS + s) * SP + el * Np + n] = MJ * a - p.visc * (MJ * b);
        }
      R[u][DIM - 1] -= MJ * q[IR] * p.grav;
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * BT;
    const int el = slot / Np, n = slot % Np;
    if (slot < SP && el < nv) contract<DIM, Nq, C::EPB, T>(sF, Ds, el, n, R[u]);
  }
  __syncthreads();
  // ---- face terms into FF[NF][NS][EPB*Nfp] (aliases sF): Rusanov - μ viscous average
  T *FF = sF;
  for (int fs = threadIdx.x; fs < C::FSLOTS; fs += BT) {
    const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
    if (el >= nv) continue;
    const int64_t e = e0 + el;
    const int vM = face_node<DIM, Nq>(f, fn);
    const T *sg = I.sgeo + (int64_t)NSG * (fn + (int64_t)Nfp * (f + NF * e));
    T nrm[DIM];
#pragma unroll
    for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
    const T smj = sg[DIM];
    T qM[NS], qP[NS], vM_[DIM], vP_[DIM];
#pragma unroll
    for (int s = 0; s < NS; ++s) qM[s] = sQ[s * SP + el * Np + vM] + I.qref[s];
    const T gM = p.grav != T(0) ? vgeo[vM + Np * (GC + NVG * e)] : T(0);
    const T riM = T(1) / qM[IR];
    const T PM = pressure_ri<DIM, T>(qM, riM, gM, p);
#pragma unroll
    for (int c = 0; c < DIM; ++c) vM_[c] = qM[c] / qM[IR];
    const int32_t nb = I.nbr[f + NF * e];
    const int64_t e2 = nb >= 0 ? (int64_t)(nb >> 3) : e;
    const int vP = nb >= 0 ? face_node<DIM, Nq>(nb & 7, fn) : vM;
    T PP, riP;
    if (nb >= 0) {
#pragma unroll
      for (int s = 0; s < NS; ++s) qP[s] = Qin[vP + Np * (s + NS * e2)] + I.qref[s];
      const T gP = p.grav != T(0) ? vgeo[vP + Np * (GC + NVG * e2)] : T(0);
      riP = T(1) / qP[IR];
      PP = pressure_ri<DIM, T>(qP, riP, gP, p);
#pragma unroll
      for (int c = 0; c < DIM; ++c) vP_[c] = qP[c] / qP[IR];
    } else {  // reflective wall (nse3d.jl:880-900): mirrored state and velocity
      wall_state<DIM, T>(qM, nrm, qP);
      riP = riM;
      PP = PM;
      T un = nrm[0] * vM_[0] + nrm[1] * vM_[1];
      if (DIM == 3) un = un + nrm[2] * vM_[2];
#pragma unroll
      for (int c = 0; c < DIM; ++c) vP_[c] = vM_[c] - T(2) * un * nrm[c];
    }
    T out[NS];
    rusanov_n<DIM, T>(qM, riM, PM, qP, riP, PP, nrm, p, out);
    // n · (F_visc⁻ + F_visc⁺), one side at a time (fewer live registers)
    T av[NS];
    {
      T g[NS][DIM], fv[NS][DIM];
#pragma unroll
      for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int c = 0; c < DIM; ++c) g[s][c] = gq[vM + Np * (s + NS * (c + (int64_t)DIM * e))];
      visc_flux<DIM, T>(g, vM_, p, fv);
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        av[s] = nrm[0] * fv[s][0] + nrm[1] * fv[s][1];
        if (DIM == 3) av[s] = av[s] + nrm[2] * fv[s][2];
      }
      if (nb >= 0) {
#pragma unroll
        for (int s = 0; s < NS; ++s)
#pragma unroll
          for (int c = 0; c < DIM; ++c) g[s][c] = gq[vP + Np * (s + NS * (c + (int64_t)DIM * e2))];
      } else {  // mirrored gradients, the temperature gradient copied from the interior
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          if (s == IE) continue;
          T sn = nrm[0] * g[s][0] + nrm[1] * g[s][1];
          if (DIM == 3) sn = sn + nrm[2] * g[s][2];
#pragma unroll
          for (int c = 0; c < DIM; ++c) g[s][c] = g[s][c] - T(2) * sn * nrm[c];
        }
      }
      visc_flux<DIM, T>(g, vP_, p, fv);
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        T b = nrm[0] * fv[s][0] + nrm[1] * fv[s][1];
        if (DIM == 3) b = b + nrm[2] * fv[s][2];
        av[s] = av[s] + b;
      }
    }
#pragma unroll
    for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = smj * out[s] - p.visc * (smj * (T(0.5) * av[s]));
  }
  __syncthreads();
  bool bad = false;
#pragma unroll
  for (int u = 0; u < C::NPT; ++u) {
    const int slot = threadIdx.x + u * BT;
    const int el = slot / Np, n = slot % Np;
    const int64_t e = e0 + el;
    if (slot < SP && el < nv) {
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
  if (bad) atomicOr(I.status, ST_NONFINITE);
  __syncthreads();  // shared memory is reused by the block's next item
}

// Persistent viscous passes of one shape (the grouped variant's work list).
template <int DIM, int Nq, typename T, bool GRAD>
__global__ void __launch_bounds__(BT, 2)
k_ns_batch(const BHdr *__restrict__ hdr, int stage, PhysT<T> p, T rka, double rkb) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int SID = shape_id(DIM, Nq - 1, 1);
  const int nwork = hdr->nwork[SID];
  const int64_t step = hdr->step;
  const BWork *__restrict__ work = hdr->work[SID];
  const BDesc<T> *__restrict__ desc = static_cast<const BDesc<T> *>(hdr->desc);
  T *const *gqt = static_cast<T *const *>(hdr->gq);
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const BWork it = work[w];
    if (!it.valid) continue;  // uniform over the block
    const BDesc<T> &I = desc[it.slot];
    const int64_t k = step - I.start;
    if (k >= I.target) continue;
    const int par = (int)((k + stage) & 1);
    if constexpr (GRAD)
      ns_grad_group<DIM, Nq, T>(I, gqt[it.slot], it.e0, it.nv, par, p, smem_raw);
    else
      ns_stage_group<DIM, Nq, T>(I, gqt[it.slot], it.e0, it.nv, par, p, rka, T(rkb * I.dt), smem_raw);
  }
}

// The two viscous passes over one mesh (cb_lsrk_run with visc > 0): groups
// of BCfg<DIM, Nq, 0>::EPB consecutive elements, blocks striding over them;
// the state is read from I.Q[0] and written to I.Q[1].
// Block-wide L2 prefetch of `bytes` bytes from p (one request per 128-byte line).
__device__ __forceinline__ void prefetch_l2(const void *p, size_t bytes) {
  const char *c = static_cast<const char *>(p);
  for (size_t off = (size_t)threadIdx.x * 128; off < bytes; off += (size_t)blockDim.x * 128)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(c + off));
}

template <int DIM, int Nq, typename T, bool GRAD>
__global__ void __launch_bounds__(BT, 2)
k_ns_mesh(BDesc<T> I, T *gq, int64_t nelem, PhysT<T> p, T rka, T rkbdt) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  using C = BCfg<DIM, Nq, 0>;
  constexpr int EPB = C::EPB, NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG;
  constexpr size_t QE = (size_t)C::Np * NS, VE = (size_t)C::Np * NVG, SE = (size_t)NSG * C::Nfp * C::NFACE;
  for (int64_t g = blockIdx.x; g * EPB < nelem; g += gridDim.x) {
    const int64_t e0 = g * EPB;
    const int nv = nelem - e0 < EPB ? (int)(nelem - e0) : EPB;
    // the block's next group: bring its slabs into L2 while this one runs
    const int64_t n0 = e0 + (int64_t)gridDim.x * EPB;
    if (n0 < nelem) {
      const size_t nn = (size_t)(nelem - n0 < EPB ? nelem - n0 : EPB);
      prefetch_l2(I.Q[0] + n0 * QE, sizeof(T) * nn * QE);
      prefetch_l2(I.vgeo + n0 * VE, sizeof(T) * nn * VE);
      prefetch_l2(I.sgeo + n0 * SE, sizeof(T) * nn * SE);
      if constexpr (!GRAD) {
        prefetch_l2(I.rhs + n0 * QE, sizeof(T) * nn * QE);
        prefetch_l2(gq + n0 * QE * DIM, sizeof(T) * nn * QE * DIM);
      }
    }
    if constexpr (GRAD)
      ns_grad_group<DIM, Nq, T>(I, gq, e0, nv, 0, p, smem_raw);
    else
      ns_stage_group<DIM, Nq, T>(I, gq, e0, nv, 0, p, rka, rkbdt, smem_raw);
  }
}
// Shared memory of the gradient (pass 0) and stage (pass 1) passes.
template <int DIM, int Nq, typename T>
constexpr size_t ns_smem(int pass) {
  using C = BCfg<DIM, Nq, 0>;
  return sizeof(T) * (((Nq * Nq + 1) & ~1) + (size_t)Lay<DIM>::NS * C::SLOTS + (size_t)DIM * Lay<DIM>::NS * C::SLOTS +
                      (pass == 0 ? (size_t)C::NFACE * Lay<DIM>::NS * DIM * C::EPB * C::Nfp : 0));
}

// Item source of the pipelined stage over a work list of many instances
// (see k_stage_pipe2).  The second warp of the block (the first issues the
// bulk copies) finds the block's next live item and publishes it into a
// shared-memory ring (the current item, the ones whose copies are in flight,
// and the one being published; three entries, four for the DEEP stage):
// each lane copies one 8-byte word of the instance descriptor, so a publish
// costs two parallel round trips (work item, descriptor).  The shape's list,
// the descriptor table and the batch step are cached at the head of the ring.
template <typename T>
struct BItem {
  BDesc<T> d;  // word-for-word copy of the instance descriptor
  int64_t e0;
  int32_t nv, valid, par, last;  // last: the group ends the instance's arrays
};
struct alignas(16) BRingHdr {
  const BWork *work;
  const void *desc;
  int64_t step;
  int32_t nwork, pad;
};
// RING: ring entries; items it .. it + RING - 2 are published at the top of
// iteration it (the group in work and RING - 2 ahead of it), and publish(it)
// writes item it + RING - 1.
template <typename T, int NS, int EPB, int RING = 3>
struct BatchSrc {
  using Real = T;
  static constexpr int WORDS = (int)(sizeof(BDesc<T>) / 8);
  static_assert(sizeof(BDesc<T>) % 8 == 0 && WORDS <= 32, "descriptor words");
  static constexpr int START_WORD = (int)(offsetof(BDesc<T>, start) / 8);
  static constexpr int TARGET_WORD = (int)(offsetof(BDesc<T>, target) / 8);
  static constexpr int AHEAD = RING - 2;
  static constexpr size_t RING_BYTES = sizeof(BRingHdr) + RING * sizeof(BItem<T>);
  static constexpr int PUBLISHER = 32;  // first thread of the publishing warp
  const BHdr *hdr;
  int sid, stage;
  double rkb;
  BRingHdr *rh;
  BItem<T> *ring;
  int wpos;  // publishing warp: work index of the last published item (-1: none)

  // whole publishing warp: publish the first live item at or after w on this
  // block's stride into dst; returns its index (-1: none)
  __device__ int publish_from(int w, BItem<T> &dst) const {
    const int lane = threadIdx.x & 31;
    const BWork *work = rh->work;
    const int nwork = rh->nwork;
    const int64_t step = rh->step;
    const unsigned long long *dw = static_cast<const unsigned long long *>(rh->desc);
    for (; w >= 0 && w < nwork; w += gridDim.x) {
      const BWork wk = work[w];
      if (!wk.valid) continue;
      const unsigned long long v = lane < WORDS ? dw[(size_t)wk.slot * WORDS + lane] : 0ull;
      const int64_t start = (int64_t)__shfl_sync(0xffffffffu, v, START_WORD);
      const int64_t target = (int64_t)__shfl_sync(0xffffffffu, v, TARGET_WORD);
      if (step - start >= target) continue;
      if (lane < WORDS) reinterpret_cast<unsigned long long *>(&dst.d)[lane] = v;
      if (lane == 0) {
        dst.e0 = wk.e0;
        dst.nv = wk.nv;
        dst.last = wk.valid >> 1;
        dst.par = (int)((step - start + stage) & 1);
        dst.valid = 1;
      }
      return w;
    }
    if (lane == 0) dst.valid = 0;
    return -1;
  }
  __device__ void begin(unsigned char *mem) {
    rh = reinterpret_cast<BRingHdr *>(mem);
    ring = reinterpret_cast<BItem<T> *>(mem + sizeof(BRingHdr));
    if ((threadIdx.x >> 5) == (PUBLISHER >> 5)) {
      if ((threadIdx.x & 31) == 0) {
        rh->work = hdr->work[sid];
        rh->desc = hdr->desc;
        rh->step = hdr->step;
        rh->nwork = hdr->nwork[sid];
      }
      __syncwarp();
      int w = publish_from(blockIdx.x, ring[0]);
      for (int j = 1; j < RING - 1; ++j) {
        if (w >= 0) w = publish_from(w + gridDim.x, ring[j]);
        else if ((threadIdx.x & 31) == 0) ring[j].valid = 0;
      }
      wpos = w;
    }
  }
  // start fetching the work item that publish() will most likely read (the
  // next one on this block's stride), so that its cache miss overlaps the wait
  // for the current group's bulk copies
  __device__ void prefetch() const {
    const int w = wpos < 0 ? -1 : wpos + (int)gridDim.x;
    if (w < 0 || w >= rh->nwork) return;
    asm volatile("prefetch.global.L1 [%0];" ::"l"(rh->work + w));
  }
  __device__ void publish(int it) {
    wpos = wpos < 0 ? -1 : publish_from(wpos + gridDim.x, ring[(it + RING - 1) % RING]);
    if (wpos < 0 && (threadIdx.x & 31) == 0) ring[(it + RING - 1) % RING].valid = 0;
  }
  __device__ bool skip_copy(int) const { return false; }
  __device__ uint32_t wait_limit() const { return WAIT_LIMIT; }
  __device__ const BItem<T> &at(int it) const { return ring[it % RING]; }
  __device__ bool valid(int it) const { return at(it).valid != 0; }
  __device__ bool last(int it) const { return at(it).last != 0; }
  __device__ int64_t e0(int it) const { return at(it).e0; }
  __device__ int nv(int it) const { return at(it).nv; }
  // (par & 1: an entry that holds no item leaves par unset; the index stays
  // inside the descriptor even if such an entry is asked)
  __device__ const T *Qin(int it) const { return at(it).d.Q[at(it).par & 1]; }
  __device__ T *Qout(int it) const { return at(it).d.Q[(at(it).par & 1) ^ 1]; }
  __device__ T *rhs(int it) const { return at(it).d.rhs; }
  __device__ const T *vgeo(int it) const { return at(it).d.vgeo; }
  __device__ const T *sgeo(int it) const { return at(it).d.sgeo; }
  __device__ const int32_t *nbr(int it) const { return at(it).d.nbr; }
  __device__ const T *D(int it) const { return at(it).d.D; }
  __device__ const T *gq(int it) const { return at(it).d.gq; }
  __device__ T qref(int it, int s) const { return at(it).d.qref[s]; }
  __device__ T rkbdt(int it) const { return T(rkb * at(it).d.dt); }
  __device__ unsigned *status(int it) const { return at(it).d.status; }
};
template <int DIM, int Nq, typename T, int RING = 3, int X = 1>
using BPipeSrc = BatchSrc<T, Lay<DIM>::NS, CfgX<DIM, Nq, X>::EPB, RING>;  // EPB does not depend on Y

inline bool b_order_ok(int dim, int N) { return N >= 1 && N <= (dim == 2 ? BMAXN2 : BMAXN3); }

// Host table of the stage kernels of one precision, indexed by shape id:
// kernel, elements per group, threads, dynamic shared memory, whether the
// kernel is the pipelined one, and its persistent grid once prepared.
template <typename T>
struct BKernels {
  const void *fn[NSHAPE] = {};
  int epb[NSHAPE] = {}, threads[NSHAPE] = {}, grid[NSHAPE] = {};
  int ahead[NSHAPE] = {};  // element groups whose copies are in flight ahead of the work (0: grouped)
  size_t smem[NSHAPE] = {};
  bool pipelined[NSHAPE] = {}, ready[NSHAPE] = {};
  // viscous batches (variant 1 shapes only): gradient and stage passes
  const void *vfn[2][NSHAPE] = {};
  int vgrid[2][NSHAPE] = {}, vthreads[2][NSHAPE] = {};
  size_t vsmem[2][NSHAPE] = {};
  bool vpipelined[2][NSHAPE] = {};  // the pass takes a BatchSrc (k_ns_stage_pipe)
  bool vready[NSHAPE] = {};
};
template <int DIM, int Nq, int G, typename T>
constexpr size_t b_group_smem() {
  using C = BCfg<DIM, Nq, G>;
  return sizeof(T) * (((Nq * Nq + 1) & ~1) + (size_t)Lay<DIM>::NS * C::SLOTS +
                      (size_t)DIM * Lay<DIM>::NS * C::SLOTS);
}
template <int DIM, int Nq, typename T, int MINB, bool AFF = false, bool DEEP = false, int X = 1, int Y = 1>
void b_fill_pipe(BKernels<T> &k, int var) {
  using Src = BPipeSrc<DIM, Nq, T, DEEP ? 4 : 3, X>;
  const int id = shape_id(DIM, Nq - 1, var);
  k.fn[id] = (const void *)k_stage_pipe2<DIM, Nq, T, Src, MINB, AFF, DEEP, X, Y>;
  k.epb[id] = CfgX<DIM, Nq, X, Y>::EPB;
  k.threads[id] = CfgX<DIM, Nq, X, Y>::THREADS;
  k.smem[id] = Pipe2<DIM, Nq, T, AFF, DEEP, X, Y>::smem() + Src::RING_BYTES;
  k.pipelined[id] = true;
  k.ahead[id] = DEEP ? 2 : 1;
}
template <int DIM, int Nq, typename T>
void b_fill(BKernels<T> &k) {
  constexpr int N = Nq - 1;
  if constexpr (Pipe2<DIM, Nq, T>::OK) {
    constexpr int M0 = Pipe2<DIM, Nq, T>::MINB;
    b_fill_pipe<DIM, Nq, T, M0>(k, 0);
    // blocks of up to 256 threads: also sized for three and four per SM
    if constexpr (Cfg<DIM, Nq>::THREADS <= 256) {
      b_fill_pipe<DIM, Nq, T, M0 == 3 ? 2 : 3>(k, 3);
      b_fill_pipe<DIM, Nq, T, M0 == 4 ? 2 : 4>(k, 4);
    }
    // the per-node stage with copies two groups ahead (staging depth 2), at
    // the default occupancy where that fits
    using PN = Pipe2<DIM, Nq, T, false, true>;
    if constexpr (PN::OK && PN::fits(M0)) b_fill_pipe<DIM, Nq, T, M0, false, true>(k, VAR_DEEP);
    // twice the elements per group on twice the threads (blocks of 512)
    if constexpr (Cfg<DIM, Nq>::THREADS <= 256) {
      using PW = Pipe2<DIM, Nq, T, false, false, 2>;
      if constexpr (PW::OK && PW::fits(PW::MINB)) b_fill_pipe<DIM, Nq, T, PW::MINB, false, false, 2>(k, VAR_WIDE);
    }
    // the affine stage copies two groups ahead where that fits M0 blocks per SM
    using PD = Pipe2<DIM, Nq, T, true, true>;
    if constexpr (PD::OK && PD::fits(M0)) b_fill_pipe<DIM, Nq, T, M0, true, true>(k, VAR_AFFINE);
    else if constexpr (Pipe2<DIM, Nq, T, true>::OK) b_fill_pipe<DIM, Nq, T, M0, true>(k, VAR_AFFINE);
    // the lean pipelined stage (state-only staging)
    if constexpr (Lean<DIM, Nq, T>::OK) {
      using Src = BatchSrc<T, Lay<DIM>::NS, Cfg<DIM, Nq>::EPB, 3>;
      const int id = shape_id(DIM, N, VAR_LEAN);
      k.fn[id] = (const void *)k_stage_lean<DIM, Nq, T, Src>;
      k.epb[id] = Cfg<DIM, Nq>::EPB;
      k.threads[id] = Cfg<DIM, Nq>::THREADS;
      k.smem[id] = Lean<DIM, Nq, T>::smem() + Src::RING_BYTES;
      k.pipelined[id] = true;
      k.ahead[id] = 1;
    }
    // the tensor-core stage (3-D N = 7, one element per group)
    if constexpr (DIM == 3 && Nq == 8) {
      using PM = PipeMT<T>;
      using Src = BatchSrc<T, 5, 1, 3>;
      const int id = shape_id(DIM, N, VAR_MMA);
      k.fn[id] = (const void *)k_stage_mma<Src, PM::MINB>;
      k.epb[id] = 1;
      k.threads[id] = PM::THREADS;
      k.smem[id] = PM::smem() + Src::RING_BYTES;
      k.pipelined[id] = true;
      k.ahead[id] = 1;
    }
    // two nodes per thread on half the threads (blocks of 128 or more), per-node
    // and affine geometry, as many blocks per SM as shared memory holds
    if constexpr (Cfg<DIM, Nq>::THREADS >= 256) {
      using PY = Pipe2<DIM, Nq, T, false, false, 1, 2>;
      if constexpr (PY::OK && PY::fits(PY::MINB)) b_fill_pipe<DIM, Nq, T, PY::MINB, false, false, 1, 2>(k, VAR_NPT2);
      using PA = Pipe2<DIM, Nq, T, true, true, 1, 2>;
      if constexpr (PA::OK && PA::fits(PA::MINB)) b_fill_pipe<DIM, Nq, T, PA::MINB, true, true, 1, 2>(k, VAR_AFFINE_NPT2);
    }
  }
  {
    const int id = shape_id(DIM, N, 1);
    k.fn[id] = (const void *)k_stage_batch<DIM, Nq, 0, T>;
    k.epb[id] = BCfg<DIM, Nq, 0>::EPB;
    k.threads[id] = BT;
    k.smem[id] = b_group_smem<DIM, Nq, 0, T>();
  }
  if constexpr (BCfg<DIM, Nq, 1>::OK) {
    const int id = shape_id(DIM, N, 2);
    k.fn[id] = (const void *)k_stage_batch<DIM, Nq, 1, T>;
    k.epb[id] = BCfg<DIM, Nq, 1>::EPB;
    k.threads[id] = BT;
    k.smem[id] = b_group_smem<DIM, Nq, 1, T>();
  }
  {
    const int id = shape_id(DIM, N, 1);
    k.vfn[0][id] = (const void *)k_ns_batch<DIM, Nq, T, true>;
    k.vfn[1][id] = (const void *)k_ns_batch<DIM, Nq, T, false>;
    k.vsmem[0][id] = ns_smem<DIM, Nq, T>(0);
    k.vsmem[1][id] = ns_smem<DIM, Nq, T>(1);
    k.vthreads[0][id] = k.vthreads[1][id] = BT;
    // the pipelined passes where their plans fit (their groups have the
    // element count of the grouped passes: one work list serves all)
    static_assert(Cfg<DIM, Nq>::EPB == BCfg<DIM, Nq, 0>::EPB, "one work list for both viscous passes");
    using VSrc = BatchSrc<T, Lay<DIM>::NS, Cfg<DIM, Nq>::EPB, 3>;
    if constexpr (NsGradPipe<DIM, Nq, T>::OK) {
      k.vfn[0][id] = (const void *)k_ns_grad_pipe<DIM, Nq, T, VSrc>;
      k.vsmem[0][id] = NsGradPipe<DIM, Nq, T>::smem() + VSrc::RING_BYTES;
      k.vthreads[0][id] = Cfg<DIM, Nq>::THREADS;
      k.vpipelined[0][id] = true;
    }
    if constexpr (NsPipe<DIM, Nq, T>::OK) {
      k.vfn[1][id] = (const void *)k_ns_stage_pipe<DIM, Nq, T, VSrc>;
      k.vsmem[1][id] = NsPipe<DIM, Nq, T>::smem() + VSrc::RING_BYTES;
      k.vthreads[1][id] = Cfg<DIM, Nq>::THREADS;
      k.vpipelined[1][id] = true;
    }
  }
}
// Fill the table entries of one dimension (one translation unit per
// dimension and precision instantiates the kernels).
template <int DIM, typename T>
void b_fill_dim(BKernels<T> &k);

}  // namespace cb
