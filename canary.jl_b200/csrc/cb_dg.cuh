// Device code of the nodal-DG hot path for sm_100a.
//
// Layouts are the reference's (column-major Julia arrays):
//   Q, rhs   [Np, NS, nelem]            vgeo [Np, NVG, nelem]
//   gradQ    [Np, NS, DIM, nelem]       sgeo [NSG, Nfp, nface, nelem]
// with node index n = i + Nq*(j + Nq*k).  One thread block processes EPB
// consecutive elements; a thread owns nodes t, t+THREADS, ... of that group.
// The element-local stage is: pointwise fluxes -> shared memory ->
// tensor-product contraction with D -> face fluxes into a shared face buffer
// -> per-node accumulation in face order -> update.  All sums run in the
// same order as the reference CPU loops so that FP64 results agree to
// round-off.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cb {

// Mirror of the public cb_phys.
struct Phys {
  double gamma, R_gas, c_p, c_v, gravity, Pr, lambda, visc;
};

// Device-side sticky status bits (see cb_device_status).
enum : unsigned { ST_BC = 1u, ST_NONFINITE = 2u, ST_MESH = 4u, ST_TIMEOUT = 8u };

template <int DIM>
struct Lay;
// euler3d_set3c.jl:96-111
template <>
struct Lay<3> {
  static constexpr int NS = 5, NVG = 14, NSG = 5, IR = 3, IE = 4, NFACE = 6;
};
// euler2d_set3c.jl:96-110
template <>
struct Lay<2> {
  static constexpr int NS = 4, NVG = 8, NSG = 4, IR = 2, IE = 3, NFACE = 4;
};
// vgeo field of metric term d(r-th reference coordinate)/d(x_c): r + DIM*c;
// MJ = DIM*DIM, MJI = DIM*DIM+1, coordinates from DIM*DIM+2.

// Per-field constants subtracted from the stored state (Q = qref + q').  The
// FP32 form keeps q' so that each stage's rounding is relative to the
// deviation instead of the full state; the FP64 form uses qref = 0.
template <typename T, int NS>
struct Offs {
  T v[NS];
};

template <typename T>
struct PhysT {
  T gamma, eos, grav, R, cpPr, lambda, visc;
  __host__ __device__ PhysT() {}
  __host__ PhysT(const Phys &p)
      : gamma(T(p.gamma)), eos(T(p.R_gas) / T(p.c_v)), grav(T(p.gravity)),
        R(T(p.R_gas)), cpPr(T(p.c_p) / T(p.Pr)), lambda(T(p.lambda)),
        visc(T(p.visc)) {}
};

__host__ __device__ constexpr int ipow(int b, int e) {
  return e == 0 ? 1 : b * ipow(b, e - 1);
}
__host__ __device__ constexpr int cdiv(int a, int b) { return (a + b - 1) / b; }

// Launch shape per (dim, Nq): elements per block and threads per block.
template <int DIM, int Nq>
struct Cfg {
  static constexpr int Np = ipow(Nq, DIM);
  static constexpr int Nfp = ipow(Nq, DIM - 1);
  static constexpr int NFACE = 2 * DIM;
  static constexpr int EPB = Np >= 200 ? 1 : (256 / Np > 0 ? 256 / Np : 1);
  static constexpr int SLOTS = EPB * Np;
  static constexpr int THREADS =
      SLOTS >= 512 ? 512 : (cdiv(SLOTS, 32) * 32 < 64 ? 64 : cdiv(SLOTS, 32) * 32);
  static constexpr int NPT = cdiv(SLOTS, THREADS);  // nodes per thread
  static constexpr int FSLOTS = EPB * NFACE * Nfp;  // face-node slots
  static constexpr int FPT = cdiv(FSLOTS, THREADS);
};

// The same with X times the elements per group on X / Y times the threads:
// X > 1 shares each block barrier among more nodes, Y > 1 gives each thread
// Y times the nodes (more independent work per thread, the per-group
// bookkeeping spread over more nodes).  X = Y = 1 is Cfg.
template <int DIM, int Nq, int X, int Y = 1>
struct CfgX : Cfg<DIM, Nq> {
  using B = Cfg<DIM, Nq>;
  static constexpr int EPB = B::EPB * X;
  static constexpr int SLOTS = EPB * B::Np;
  static constexpr int THREADS =
      Y == 1 ? B::THREADS * X : (cdiv(B::THREADS * X / Y, 32) * 32 < 64 ? 64 : cdiv(B::THREADS * X / Y, 32) * 32);
  static constexpr int NPT = cdiv(SLOTS, THREADS);
  static constexpr int FSLOTS = EPB * B::NFACE * B::Nfp;
  static constexpr int FPT = cdiv(FSLOTS, THREADS);
};

// ---------------------------------------------------------------- physics
template <int DIM, typename T>
__device__ __forceinline__ T pressure(const T *q, T gc, const PhysT<T> &p) {
  constexpr int IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  T ke = q[0] * q[0] + q[1] * q[1];
  if (DIM == 3) ke = ke + q[2] * q[2];
  const T rho = q[IR];
  return p.eos * ((q[IE] - ke / (T(2) * rho)) - rho * p.grav * gc);
}

// Euler flux f[s][c] (state s in reference order, direction c).
template <int DIM, typename T>
__device__ __forceinline__ void euler_flux(const T *q, T P, T (*f)[DIM]) {
  constexpr int IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  const T ri = T(1) / q[IR];
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      T v = ri * q[a] * q[c];
      if (a == c) v = v + P;
      f[a][c] = v;
    }
    f[IR][a] = q[a];
    f[IE][a] = ri * q[a] * (q[IE] + P);
  }
}

// Variants for the fused stage: 1/ρ is formed once per state and reused by the
// pressure, the fluxes and the wave speed (one FP64 division per state
// instead of two; rounding differs from the reference's `/(2ρ)` by <= 1 ulp).
template <int DIM, typename T>
__device__ __forceinline__ T pressure_ri(const T *q, T ri, T gc, const PhysT<T> &p) {
  constexpr int IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  T ke = q[0] * q[0] + q[1] * q[1];
  if (DIM == 3) ke = ke + q[2] * q[2];
  return p.eos * ((q[IE] - T(0.5) * ke * ri) - q[IR] * p.grav * gc);
}
template <int DIM, typename T>
__device__ __forceinline__ void euler_flux_ri(const T *q, T ri, T P, T (*f)[DIM]) {
  constexpr int IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
#pragma unroll
  for (int a = 0; a < DIM; ++a) {
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
      T v = ri * q[a] * q[c];
      if (a == c) v = v + P;
      f[a][c] = v;
    }
    f[IR][a] = q[a];
    f[IE][a] = ri * q[a] * (q[IE] + P);
  }
}
template <int DIM, typename T>
__device__ __forceinline__ void rusanov_ri(const T *qM, T rMi, T PM, const T *qP, T rPi, T PP,
                                           const T *nrm, const PhysT<T> &p, T *out) {
  constexpr int NS = Lay<DIM>::NS;
  T fM[NS][DIM], fP[NS][DIM];
  euler_flux_ri<DIM, T>(qM, rMi, PM, fM);
  euler_flux_ri<DIM, T>(qP, rPi, PP, fP);
  T unM = nrm[0] * qM[0] + nrm[1] * qM[1];
  T unP = nrm[0] * qP[0] + nrm[1] * qP[1];
  if (DIM == 3) {
    unM = unM + nrm[2] * qM[2];
    unP = unP + nrm[2] * qP[2];
  }
  const T lM = rMi * fabs(unM) + sqrt(rMi * p.gamma * PM);
  const T lP = rPi * fabs(unP) + sqrt(rPi * p.gamma * PP);
  T lam = lM > lP ? lM : lP;
  if (lM != lM || lP != lP) lam = lM + lP;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    T a = nrm[0] * (fM[s][0] + fP[s][0]) + nrm[1] * (fM[s][1] + fP[s][1]);
    if (DIM == 3) a = a + nrm[2] * (fM[s][2] + fP[s][2]);
    out[s] = (a - lam * (qP[s] - qM[s])) * T(0.5);
  }
}

// Normal Euler flux n·F of one state (5 values) given 1/ρ and P: the
// fused stage uses it instead of forming both 3x5 flux tensors and dotting
// them with n (same mathematics, about a third of the operations).
template <int DIM, typename T>
__device__ __forceinline__ void normal_flux(const T *q, T ri, T P, const T *nrm, T &un, T *fn) {
  constexpr int IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  un = nrm[0] * q[0] + nrm[1] * q[1];
  if (DIM == 3) un = un + nrm[2] * q[2];
  const T riun = ri * un;
#pragma unroll
  for (int a = 0; a < DIM; ++a) fn[a] = riun * q[a] + P * nrm[a];
  fn[IR] = un;
  fn[IE] = riun * (q[IE] + P);
}
template <int DIM, typename T>
__device__ __forceinline__ void rusanov_n(const T *qM, T rMi, T PM, const T *qP, T rPi, T PP,
                                          const T *nrm, const PhysT<T> &p, T *out) {
  constexpr int NS = Lay<DIM>::NS;
  T fM[NS], fP[NS], unM, unP;
  normal_flux<DIM, T>(qM, rMi, PM, nrm, unM, fM);
  normal_flux<DIM, T>(qP, rPi, PP, nrm, unP, fP);
  const T lM = rMi * fabs(unM) + sqrt(rMi * p.gamma * PM);
  const T lP = rPi * fabs(unP) + sqrt(rPi * p.gamma * PP);
  T lam = lM > lP ? lM : lP;
  if (lM != lM || lP != lP) lam = lM + lP;
#pragma unroll
  for (int s = 0; s < NS; ++s) out[s] = ((fM[s] + fP[s]) - lam * (qP[s] - qM[s])) * T(0.5);
}

// Rusanov numerical flux (euler3d_set3c.jl:394-446): out[s] = n·(F⁻+F⁺)/2 - λ(q⁺-q⁻)/2
template <int DIM, typename T>
__device__ __forceinline__ void rusanov(const T *qM, T PM, const T *qP, T PP,
                                        const T *nrm, const PhysT<T> &p,
                                        T *out) {
  constexpr int NS = Lay<DIM>::NS, IR = Lay<DIM>::IR;
  T fM[NS][DIM], fP[NS][DIM];
  euler_flux<DIM, T>(qM, PM, fM);
  euler_flux<DIM, T>(qP, PP, fP);
  const T rMi = T(1) / qM[IR], rPi = T(1) / qP[IR];
  T unM = nrm[0] * qM[0] + nrm[1] * qM[1];
  T unP = nrm[0] * qP[0] + nrm[1] * qP[1];
  if (DIM == 3) {
    unM = unM + nrm[2] * qM[2];
    unP = unP + nrm[2] * qP[2];
  }
  const T lM = rMi * fabs(unM) + sqrt(rMi * p.gamma * PM);
  const T lP = rPi * fabs(unP) + sqrt(rPi * p.gamma * PP);
  T lam = lM > lP ? lM : lP;
  if (lM != lM || lP != lP) lam = lM + lP;  // propagate NaN like Julia max
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    T a = nrm[0] * (fM[s][0] + fP[s][0]) + nrm[1] * (fM[s][1] + fP[s][1]);
    if (DIM == 3) a = a + nrm[2] * (fM[s][2] + fP[s][2]);
    out[s] = (a - lam * (qP[s] - qM[s])) / T(2);
  }
}

// --------------------------------------------------------------- indexing
// Local volume node of face node fn on face f (mesh.jl:979-983).
template <int DIM, int Nq>
__device__ __forceinline__ int face_node(int f, int fn) {
  const int d0 = f >> 1, side = (f & 1) * (Nq - 1);
  if (DIM == 2) return d0 == 0 ? side + Nq * fn : fn + Nq * side;
  const int a = fn % Nq, b = fn / Nq;
  if (d0 == 0) return side + Nq * (a + Nq * b);
  if (d0 == 1) return a + Nq * (side + Nq * b);
  return a + Nq * (b + Nq * side);
}

// The same with the order as a run-time value.
template <int DIM>
__device__ __forceinline__ int face_node_rt(int Nq, int f, int fn) {
  const int d0 = f >> 1, side = (f & 1) * (Nq - 1);
  if (DIM == 2) return d0 == 0 ? side + Nq * fn : fn + Nq * side;
  const int a = fn % Nq, b = fn / Nq;
  if (d0 == 0) return side + Nq * (a + Nq * b);
  if (d0 == 1) return a + Nq * (side + Nq * b);
  return a + Nq * (b + Nq * side);
}

// Subtract the face contributions of a node in face order f = 1..nface.
// FF is [NFACE][NS][EPB*Nfp] (already multiplied by sMJ).
template <int DIM, int Nq, int EPB, typename T>
__device__ __forceinline__ void gather_face_terms(const T *FF, int el, int n,
                                                  T *R) {
  constexpr int NS = Lay<DIM>::NS, Nfp = ipow(Nq, DIM - 1);
  constexpr int FS = EPB * Nfp;
  const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
  auto sub = [&](int f, int fn) {
#pragma unroll
    for (int s = 0; s < NS; ++s) R[s] -= FF[(f * NS + s) * FS + el * Nfp + fn];
  };
  if (DIM == 3) {
    if (i == 0) sub(0, j + Nq * k);
    if (i == Nq - 1) sub(1, j + Nq * k);
    if (j == 0) sub(2, i + Nq * k);
    if (j == Nq - 1) sub(3, i + Nq * k);
    if (k == 0) sub(4, i + Nq * j);
    if (k == Nq - 1) sub(5, i + Nq * j);
  } else {
    if (i == 0) sub(0, j);
    if (i == Nq - 1) sub(1, j);
    if (j == 0) sub(2, i);
    if (j == Nq - 1) sub(3, i);
  }
}

// Contraction of one node: R[s] += Σ_m D[m,i] F0[m,j,k,s] (+ η, ζ terms),
// each direction summed completely before the next (euler3d_set3c.jl:326-337).
// sF is [DIM][NS][EPB*Np]; Ds is Nq*Nq column-major.
template <int DIM, int Nq, int EPB, typename T>
__device__ __forceinline__ void contract(const T *sF, const T *Ds, int el,
                                         int n, T *R) {
  constexpr int NS = Lay<DIM>::NS, Np = ipow(Nq, DIM);
  constexpr int SP = EPB * Np;
  const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
  const T *base = sF + el * Np;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const T *F = base + (0 * NS + s) * SP;
    T acc = R[s];
#pragma unroll
    for (int m = 0; m < Nq; ++m) acc += Ds[m + Nq * i] * F[m + Nq * (j + Nq * k)];
    const T *G = base + (1 * NS + s) * SP;
#pragma unroll
    for (int m = 0; m < Nq; ++m) acc += Ds[m + Nq * j] * G[i + Nq * (m + Nq * k)];
    if (DIM == 3) {
      const T *H = base + (2 * NS + s) * SP;
#pragma unroll
      for (int m = 0; m < Nq; ++m) acc += Ds[m + Nq * k] * H[i + Nq * (j + Nq * m)];
    }
    R[s] = acc;
  }
}

// Same contraction with a sign (for the LDG passes, which subtract).
template <int DIM, int Nq, int EPB, typename T>
__device__ __forceinline__ void contract_sub(const T *sF, const T *Ds, int el,
                                             int n, T *R) {
  constexpr int NS = Lay<DIM>::NS, Np = ipow(Nq, DIM);
  constexpr int SP = EPB * Np;
  const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
  const T *base = sF + el * Np;
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const T *F = base + (0 * NS + s) * SP;
    T acc = R[s];
#pragma unroll
    for (int m = 0; m < Nq; ++m) acc -= Ds[m + Nq * i] * F[m + Nq * (j + Nq * k)];
    const T *G = base + (1 * NS + s) * SP;
#pragma unroll
    for (int m = 0; m < Nq; ++m) acc -= Ds[m + Nq * j] * G[i + Nq * (m + Nq * k)];
    if (DIM == 3) {
      const T *H = base + (2 * NS + s) * SP;
#pragma unroll
      for (int m = 0; m < Nq; ++m) acc -= Ds[m + Nq * k] * H[i + Nq * (j + Nq * m)];
    }
    R[s] = acc;
  }
}

// Load one node's metric: met[r][c] and MJ.
template <int DIM, typename T>
__device__ __forceinline__ void load_metric(const T *__restrict__ vg, int n,
                                            int Np, T (*met)[DIM], T &MJ) {
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int c = 0; c < DIM; ++c) met[r][c] = vg[n + Np * (r + DIM * c)];
  MJ = vg[n + Np * (DIM * DIM)];
}

// Pointwise inviscid phase: contravariant fluxes of one node into sF and the
// buoyancy source into R (euler3d_set3c.jl:274-324).
template <int DIM, int Nq, int EPB, typename T>
__device__ __forceinline__ void pointwise_euler(const T *q, const T *__restrict__ vg,
                                                int n, int el, T *sF,
                                                const PhysT<T> &p, T *R) {
  constexpr int NS = Lay<DIM>::NS, Np = ipow(Nq, DIM), SP = EPB * Np;
  constexpr int IR = Lay<DIM>::IR;
  T met[DIM][DIM], MJ;
  load_metric<DIM, T>(vg, n, Np, met, MJ);
  const T gc = p.grav != T(0) ? vg[n + Np * (DIM * DIM + 2 + DIM - 1)] : T(0);
  const T P = pressure<DIM, T>(q, gc, p);
  T f[NS][DIM];
  euler_flux<DIM, T>(q, P, f);
#pragma unroll
  for (int r = 0; r < DIM; ++r)
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      T a = met[r][0] * f[s][0] + met[r][1] * f[s][1];
      if (DIM == 3) a = a + met[r][2] * f[s][2];
      sF[(r * NS + s) * SP + el * Np + n] = MJ * a;
    }
  R[DIM - 1] -= MJ * q[IR] * p.grav;
}

}  // namespace cb
