// Device-side FP64 grid and geometry of the set3c drivers: creategrid
// (src/metric.jl:11-107), the optional sinusoidal mesh warp, computemetric
// (src/metric.jl:155-208 in 2-D, the curl-invariant form of
// src/metric.jl:230-400 in 3-D) and computegeometry's assembly of vgeo / sgeo
// (examples/3d_kernels/euler3d_set3c.jl:210-248,
// examples/2d_kernels/euler2d_set3c.jl:171-208).
//
// One block per element; the element's coordinates, their derivatives, the
// curl products and the metric live in shared memory.  Sums over the 1-D
// index run in the reference's order, and this file is compiled without
// multiply-add contraction, so the results follow the reference's
// arithmetic up to the last bits of the libm functions (sin, hypot).
#include <cuda_runtime.h>

#include "../../include/canary_b200.h"
#include "cb_dg.cuh"

namespace cb {
int solver_fail(int code, const char *fmt, ...);

namespace {

constexpr int GT = 256;  // threads per block

// Julia's n-argument hypot: maxabs * sqrt(sum((v / maxabs)^2)).
__device__ __forceinline__ double hypot3(double a, double b, double c) {
  const double m = fmax(fmax(fabs(a), fabs(b)), fabs(c));
  if (m == 0.0 || isinf(m)) return m;
  const double p = a / m, q = b / m, s = c / m;
  return m * sqrt((p * p + q * q) + s * s);
}

template <int DIM, int Nq>
struct GeoPlan {
  static constexpr int Np = ipow(Nq, DIM), Nfp = ipow(Nq, DIM - 1), NF = 2 * DIM, NV = 1 << DIM;
  static constexpr int NX = DIM, ND = DIM * DIM, NP = DIM == 3 ? 9 : 0;
  static constexpr size_t smem() { return sizeof(double) * ((size_t)(Nq * Nq + 2 * Nq) + (size_t)(NX + ND + NP) * Np); }
};

// e2c: elemtocoord (DIM, 2^DIM, nelem); r, w: LGL points and weights; D: (Nq, Nq).
template <int DIM, int Nq>
__global__ void __launch_bounds__(GT) k_geometry(const double *__restrict__ e2c, int64_t nelem, double amp,
                                                 const double *__restrict__ r_, const double *__restrict__ w_,
                                                 const double *__restrict__ D_, double *__restrict__ vgeo,
                                                 double *__restrict__ sgeo) {
  using G = GeoPlan<DIM, Nq>;
  constexpr int Np = G::Np, Nfp = G::Nfp, NF = G::NF, NV = G::NV;
  constexpr int NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, NM = DIM * DIM;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double *Ds = reinterpret_cast<double *>(smem_raw);  // D[i + Nq n]
  double *rs = Ds + Nq * Nq, *ws = rs + Nq;
  double *X = ws + Nq;        // [DIM][Np] coordinates; X[0] later holds J
  double *dX = X + DIM * Np;  // [DIM*DIM][Np] dx_c/dr_a at c*DIM + a; later the metric
  double *P = dX + NM * Np;   // 3-D: [9][Np] curl products
  const int64_t e = blockIdx.x;
  if (e >= nelem) return;
  for (int t = threadIdx.x; t < Nq * Nq; t += GT) Ds[t] = D_[t];
  for (int t = threadIdx.x; t < Nq; t += GT) {
    rs[t] = r_[t];
    ws[t] = w_[t];
  }
  __syncthreads();
  const double *ec = e2c + (int64_t)DIM * NV * e;
  double *vg = vgeo + (int64_t)Np * NVG * e;
  // ---- creategrid (+ warp), coordinates into vgeo
  for (int p = threadIdx.x; p < Np; p += GT) {
    const int i = p % Nq, j = (p / Nq) % Nq, k = DIM == 3 ? p / (Nq * Nq) : 0;
    const double ai = 1.0 - rs[i], bi = 1.0 + rs[i], aj = 1.0 - rs[j], bj = 1.0 + rs[j];
    double c[DIM];
    if (DIM == 2) {
      const double wv[4] = {ai * aj, bi * aj, ai * bj, bi * bj};
#pragma unroll
      for (int n = 0; n < DIM; ++n) {
        double t = wv[0] * ec[n + DIM * 0];
#pragma unroll
        for (int v = 1; v < 4; ++v) t = t + wv[v] * ec[n + DIM * v];
        c[n] = t / 4.0;
      }
    } else {
      const double ak = 1.0 - rs[k], bk = 1.0 + rs[k];
      const double wv[8] = {ai * aj * ak, bi * aj * ak, ai * bj * ak, bi * bj * ak,
                            ai * aj * bk, bi * aj * bk, ai * bj * bk, bi * bj * bk};
#pragma unroll
      for (int n = 0; n < DIM; ++n) {
        double t = wv[0] * ec[n + DIM * 0];
#pragma unroll
        for (int v = 1; v < 8; ++v) t = t + wv[v] * ec[n + DIM * v];
        c[n] = t / 8.0;
      }
    }
    if (amp != 0.0) {  // x_c += amp * prod_d sin(x_d)
      double s = sin(c[0]);
#pragma unroll
      for (int n = 1; n < DIM; ++n) s = s * sin(c[n]);
      const double dx = amp * s;
#pragma unroll
      for (int n = 0; n < DIM; ++n) c[n] = c[n] + dx;
    }
#pragma unroll
    for (int n = 0; n < DIM; ++n) {
      X[n * Np + p] = c[n];
      vg[p + Np * (NM + 2 + n)] = c[n];
    }
  }
  __syncthreads();
  // ---- derivatives of the coordinates along each reference direction
  for (int p = threadIdx.x; p < Np; p += GT) {
    const int idx[3] = {p % Nq, (p / Nq) % Nq, DIM == 3 ? p / (Nq * Nq) : 0};
    const int str[3] = {1, Nq, Nq * Nq};
#pragma unroll
    for (int a = 0; a < DIM; ++a) {
      const int base = p - idx[a] * str[a];
#pragma unroll
      for (int cc = 0; cc < DIM; ++cc) {
        const double *x = X + cc * Np;
        double acc = 0.0;
        for (int n = 0; n < Nq; ++n) acc = acc + Ds[idx[a] + Nq * n] * x[base + n * str[a]];
        dX[(cc * DIM + a) * Np + p] = acc;
      }
    }
  }
  __syncthreads();
  if (DIM == 2) {
    // ---- 2-D metric (metric.jl:155-208) into dX, J into X[0]
    for (int p = threadIdx.x; p < Np; p += GT) {
      const double xr = dX[0 * Np + p], xs = dX[1 * Np + p], yr = dX[2 * Np + p], ys = dX[3 * Np + p];
      const double J = xr * ys - yr * xs;
      const double m[4] = {ys / J, -yr / J, -xs / J, xr / J};  // xix, etax, xiy, etay
      const int i = p % Nq, j = p / Nq;
      const double MJ = ws[j] * ws[i] * J;
#pragma unroll
      for (int f = 0; f < 4; ++f) vg[p + Np * f] = m[f];
      vg[p + Np * 4] = MJ;
      vg[p + Np * 5] = 1.0 / MJ;
      X[p] = J;  // only this thread reads or writes node p in this pass
#pragma unroll
      for (int f = 0; f < 4; ++f) dX[f * Np + p] = m[f];
    }
  } else {
    // ---- 3-D: J and the curl products (metric.jl:230-300), pointwise
    for (int p = threadIdx.x; p < Np; p += GT) {
      const double x = X[p], y = X[Np + p], z = X[2 * Np + p];
      const double xr = dX[0 * Np + p], xs = dX[1 * Np + p], xt = dX[2 * Np + p];
      const double yr = dX[3 * Np + p], ys = dX[4 * Np + p], yt = dX[5 * Np + p];
      const double zr = dX[6 * Np + p], zs = dX[7 * Np + p], zt = dX[8 * Np + p];
      const double J = (xr * (ys * zt - zs * yt) + yr * (zs * xt - xs * zt)) + zr * (xs * yt - ys * xt);
      // P: yz r,s,t | zx r,s,t | xy r,s,t
      P[0 * Np + p] = y * zr - z * yr;
      P[1 * Np + p] = y * zs - z * ys;
      P[2 * Np + p] = y * zt - z * yt;
      P[3 * Np + p] = z * xr - x * zr;
      P[4 * Np + p] = z * xs - x * zs;
      P[5 * Np + p] = z * xt - x * zt;
      P[6 * Np + p] = x * yr - y * xr;
      P[7 * Np + p] = x * ys - y * xs;
      P[8 * Np + p] = x * yt - y * xt;
      X[p] = J;
    }
    __syncthreads();
    // ---- metric terms: curl of the products along two directions, times 1/(2J)
    for (int p = threadIdx.x; p < Np; p += GT) {
      const int idx[3] = {p % Nq, (p / Nq) % Nq, p / (Nq * Nq)};
      const int str[3] = {1, Nq, Nq * Nq};
      const double J = X[p], JI2 = 1.0 / (2.0 * J);
      // for component c (x, y, z -> product family yz, zx, xy) and direction
      // (xi, eta, zeta): pos = (product t, s, r) along (s, t, r) axes etc.
      double m[9];
#pragma unroll
      for (int cc = 0; cc < 3; ++cc) {
        const double *Pr = P + (3 * cc + 0) * Np, *Ps = P + (3 * cc + 1) * Np, *Pt = P + (3 * cc + 2) * Np;
        // xi: curl(Pt, axis 1, Ps, axis 2); eta: curl(Pr, axis 2, Pt, axis 0);
        // zeta: curl(Ps, axis 0, Pr, axis 1)
        const double *pos[3] = {Pt, Pr, Ps}, *neg[3] = {Ps, Pt, Pr};
        const int pax[3] = {1, 2, 0}, nax[3] = {2, 0, 1};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const int pa = pax[d], na = nax[d];
          const int pb = p - idx[pa] * str[pa], nb = p - idx[na] * str[na];
          double acc = 0.0;
          for (int n = 0; n < Nq; ++n) {
            acc = acc + Ds[idx[pa] + Nq * n] * pos[d][pb + n * str[pa]];
            acc = acc - Ds[idx[na] + Nq * n] * neg[d][nb + n * str[na]];
          }
          m[d + 3 * cc] = acc * JI2;  // vgeo order: xix etax zetax xiy ...
        }
      }
      const int i = idx[0], j = idx[1], k = idx[2];
      const double MJ = ((ws[k] * ws[j]) * ws[i]) * J;
#pragma unroll
      for (int f = 0; f < 9; ++f) vg[p + Np * f] = m[f];
      vg[p + Np * 9] = MJ;
      vg[p + Np * 10] = 1.0 / MJ;
#pragma unroll
      for (int f = 0; f < 9; ++f) dX[f * Np + p] = m[f];
    }
  }
  __syncthreads();
  // ---- faces: outward normals J * (grad of the face's direction), sJ, sMJ, vMJI
  double *sg = sgeo + (int64_t)NSG * Nfp * NF * e;
  for (int t = threadIdx.x; t < NF * Nfp; t += GT) {
    const int f = t / Nfp, fn = t % Nfp;
    const int p = face_node<DIM, Nq>(f, fn);
    const double J = X[p];
    const int d = f >> 1;
    const bool neg = (f & 1) == 0;
    double nv[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) {
      const double tv = J * dX[(d + DIM * cc) * Np + p];
      nv[cc] = neg ? -tv : tv;
    }
    const double sJ = DIM == 3 ? hypot3(nv[0], nv[1], nv[2]) : hypot(nv[0], nv[1]);
    double *o = sg + (int64_t)NSG * (fn + Nfp * f);
#pragma unroll
    for (int cc = 0; cc < DIM; ++cc) o[cc] = nv[cc] / sJ;
    const double sM = DIM == 3 ? ws[fn / Nq] * ws[fn % Nq] : ws[fn];
    o[DIM] = sM * sJ;
    o[DIM + 1] = vg[p + Np * (NM + 1)];  // MJI at the face node (vmapM of a conforming mesh)
  }
}

template <int DIM, int Nq>
cudaError_t launch_geometry(const double *e2c, int64_t nelem, double amp, const double *r, const double *w,
                            const double *D, double *vgeo, double *sgeo, cudaStream_t st) {
  const size_t sm = GeoPlan<DIM, Nq>::smem();
  cudaError_t e = cudaFuncSetAttribute(k_geometry<DIM, Nq>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k_geometry<DIM, Nq><<<(unsigned)nelem, GT, sm, st>>>(e2c, nelem, amp, r, w, D, vgeo, sgeo);
  return cudaGetLastError();
}

template <int DIM>
cudaError_t dispatch_geometry(int N, const double *e2c, int64_t nelem, double amp, const double *r,
                              const double *w, const double *D, double *vgeo, double *sgeo, cudaStream_t st) {
  switch (N) {
    case 1: return launch_geometry<DIM, 2>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 2: return launch_geometry<DIM, 3>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 3: return launch_geometry<DIM, 4>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 4: return launch_geometry<DIM, 5>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 5: return launch_geometry<DIM, 6>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 6: return launch_geometry<DIM, 7>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 7: return launch_geometry<DIM, 8>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 8: return launch_geometry<DIM, 9>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 9: return launch_geometry<DIM, 10>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    case 10: return launch_geometry<DIM, 11>(e2c, nelem, amp, r, w, D, vgeo, sgeo, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace
}  // namespace cb

extern "C" int cb_computegeometry(int dim, int N, int64_t nelem, const double *elemtocoord, double warp_amp,
                                  const double *r, const double *w, const double *D, double *vgeo, double *sgeo,
                                  cb_stream_t stream) {
  using namespace cb;
  if (dim != 2 && dim != 3) return solver_fail(CB_ERR_ARG, "dim must be 2 or 3 (got %d)", dim);
  if (N < 1 || N > 10) return solver_fail(CB_ERR_UNSUPPORTED, "cb_computegeometry: N must be 1..10 (got %d)", N);
  if (nelem < 0 || nelem > (1ll << 31) - 1) return solver_fail(CB_ERR_ARG, "cb_computegeometry: bad element count");
  if (nelem == 0) return CB_OK;
  if (!elemtocoord || !r || !w || !D || !vgeo || !sgeo) return solver_fail(CB_ERR_ARG, "cb_computegeometry: null array");
  const cudaStream_t st = (cudaStream_t)stream;
  const cudaError_t e = dim == 2 ? dispatch_geometry<2>(N, elemtocoord, nelem, warp_amp, r, w, D, vgeo, sgeo, st)
                                 : dispatch_geometry<3>(N, elemtocoord, nelem, warp_amp, r, w, D, vgeo, sgeo, st);
  return e == cudaSuccess ? CB_OK
                          : solver_fail(CB_ERR_CUDA, "cb_computegeometry launch: %s", cudaGetErrorString(e));
}
