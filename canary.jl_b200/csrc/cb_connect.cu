// Device-side brick mesh and connectivity: cb_brickmesh in
// include/canary_b200.h.
//
// The single-rank set-up sequence of the reference's drivers for Cartesian
// bricks — brickmesh (src/mesh.jl:259-317), partition by the Hilbert code of
// the element centroids (centroidtocode :107-141, hilbertcode :35-88,
// partition :499-580), connectmesh (:751-956) and mappings (:973-1001) — on
// the device, with the same element order and the same arrays as the host
// path:
//   1. one thread per brick element: centroid (sequential corner sum / 2^d,
//      as centroidtocode), then, after a min/max reduction, the scaled
//      integer coordinates floor((2^64 - 1) c) (exact, in 128-bit
//      arithmetic) and the Hilbert code (Skilling's AxestoTranspose and the
//      bit transpose, d 64-bit words, word 0 most significant);
//   2. a stable radix sort of the element numbers by the code words, least
//      significant word first (the lexicographic order of partition, ties by
//      element number);
//   3. one thread per sorted element: corner coordinates, boundary codes,
//      face neighbours in the brick (with periodic wrap; an unmatched face
//      is its own neighbour, as connectmesh leaves it) and vmapM / vmapP
//      (every brick face matches with orientation 1).
#include <cuda_runtime.h>

#include <algorithm>
#include <cub/device/device_radix_sort.cuh>
#include <utility>

#include "../../include/canary_b200.h"
#include "cb_dg.cuh"

namespace cb {
int solver_fail(int code, const char *fmt, ...);
}

using namespace cb;

namespace {

struct Brick {
  int dim;
  int64_t n[3], nelem;
  const double *x[3];
  int per[3];
  int64_t bnd[2][3];
};

__device__ __forceinline__ void brick_index(const Brick &b, int64_t g, int64_t *ec) {
  for (int d = 0; d < b.dim; ++d) {
    ec[d] = g % b.n[d];
    g /= b.n[d];
  }
}

__global__ void k_centroid(Brick b, double *cen) {
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < b.nelem; g += (int64_t)gridDim.x * blockDim.x) {
    int64_t ec[3] = {0, 0, 0};
    brick_index(b, g, ec);
    const int nvert = 1 << b.dim;
    for (int d = 0; d < b.dim; ++d) {
      double s = 0.0;
      for (int v = 0; v < nvert; ++v) s = s + b.x[d][ec[d] + ((v >> d) & 1)];
      cen[d * b.nelem + g] = s / nvert;
    }
  }
}

// min and max of each coordinate of the centroids (one block)
__global__ void k_minmax(const double *cen, int dim, int64_t nelem, double *mm) {
  __shared__ double lo[256], hi[256];
  for (int d = 0; d < dim; ++d) {
    double a = INFINITY, z = -INFINITY;
    for (int64_t g = threadIdx.x; g < nelem; g += blockDim.x) {
      const double c = cen[d * nelem + g];
      a = fmin(a, c);
      z = fmax(z, c);
    }
    lo[threadIdx.x] = a;
    hi[threadIdx.x] = z;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s) {
        lo[threadIdx.x] = fmin(lo[threadIdx.x], lo[threadIdx.x + s]);
        hi[threadIdx.x] = fmax(hi[threadIdx.x], hi[threadIdx.x + s]);
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      mm[d] = lo[0];
      mm[3 + d] = hi[0];
    }
    __syncthreads();
  }
}

// floor((2^64 - 1) c) for c in [0, 1], exactly: c = mi 2^(ex - 53) with a
// 53-bit integer mi, and (2^64 - 1) mi = mi 2^64 - mi is formed in 128 bits.
__device__ uint64_t scaled_floor(double c) {
  if (!(c > 0.0)) return 0;
  int ex = 0;
  const double m = frexp(c, &ex);  // c = m 2^ex, m in [0.5, 1)
  const uint64_t mi = (uint64_t)ldexp(m, 53);
  const int sh = 53 - ex;
  if (sh <= 0) return ~0ull;
  const uint64_t hi = mi - 1, lo = 0ull - mi;  // (mi 2^64 - mi) as hi:lo
  if (sh >= 128) return 0;
  if (sh >= 64) return hi >> (sh - 64);
  return (hi << (64 - sh)) | (lo >> sh);
}

// Hilbert integer of n <= 3 axes coordinates of `bits` bits (hilbertcode,
// mesh.jl:35-88): the transposed form, then its bits interleaved into n words.
__device__ void hilbert(uint64_t *X, int n, int bits, uint64_t *H) {
  const uint64_t M = 1ull << (bits - 1);
  uint64_t Q = M;
  for (int r = 0; r < bits - 1; ++r) {
    const uint64_t P = Q - 1;
    for (int i = 0; i < n; ++i) {
      if (X[i] & Q) {
        X[0] ^= P;
      } else {
        const uint64_t t = (X[0] ^ X[i]) & P;
        X[0] ^= t;
        if (i != 0) X[i] ^= t;
      }
    }
    Q >>= 1;
  }
  for (int i = 1; i < n; ++i) X[i] ^= X[i - 1];
  uint64_t t = 0;
  Q = M;
  for (int r = 0; r < bits - 1; ++r) {
    if (X[n - 1] & Q) t ^= Q - 1;
    Q >>= 1;
  }
  for (int i = 0; i < n; ++i) X[i] ^= t;
  for (int i = 0; i < n; ++i) H[i] = 0;
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < bits; ++j) {
      const int k = i * bits + j;
      const uint64_t bit = (X[n - 1 - (k % n)] >> (k / n)) & 1ull;
      H[n - 1 - i] |= bit << j;
    }
}

__global__ void k_codes(Brick b, const double *cen, const double *mm, uint64_t *code, int64_t *order) {
  // size = cmax - cmin; all zero -> ones; a zero entry -> the largest one
  double size[3], smax = 0.0;
  bool allzero = true;
  for (int d = 0; d < b.dim; ++d) {
    size[d] = mm[3 + d] - mm[d];
    allzero &= size[d] == 0.0;
    smax = fmax(smax, size[d]);
  }
  for (int d = 0; d < b.dim; ++d) size[d] = allzero ? 1.0 : (size[d] == 0.0 ? smax : size[d]);
  for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < b.nelem; g += (int64_t)gridDim.x * blockDim.x) {
    uint64_t X[3], H[3];
    for (int d = 0; d < b.dim; ++d) X[d] = scaled_floor((cen[d * b.nelem + g] - mm[d]) / size[d]);
    hilbert(X, b.dim, 64, H);
    for (int d = 0; d < b.dim; ++d) code[d * b.nelem + g] = H[d];
    order[g] = g;
  }
}

__global__ void k_gather_keys(const uint64_t *word, const int64_t *order, int64_t nelem, uint64_t *keys) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nelem; p += (int64_t)gridDim.x * blockDim.x)
    keys[p] = word[order[p]];
}

__global__ void k_inverse(const int64_t *order, int64_t nelem, int64_t *inv) {
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < nelem; p += (int64_t)gridDim.x * blockDim.x)
    inv[order[p]] = p;
}

template <int DIM>
__global__ void k_connect(Brick b, int Nq, const int64_t *order, const int64_t *inv, double *etc, int64_t *etb,
                          int64_t *vmapM, int64_t *vmapP) {
  constexpr int NV = 1 << DIM, NF = 2 * DIM;
  int Np = Nq, Nfp = 1;
  for (int d = 1; d < DIM; ++d) {
    Np *= Nq;
    Nfp *= Nq;
  }
  for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < b.nelem; p += (int64_t)gridDim.x * blockDim.x) {
    const int64_t g = order[p];
    int64_t ec[3] = {0, 0, 0};
    brick_index(b, g, ec);
    for (int v = 0; v < NV; ++v)
      for (int d = 0; d < DIM; ++d) etc[d + DIM * (v + (int64_t)NV * p)] = b.x[d][ec[d] + ((v >> d) & 1)];
    for (int f = 0; f < NF; ++f) {
      const int d = f >> 1, side = f & 1;
      const bool edge = side ? ec[d] == b.n[d] - 1 : ec[d] == 0;
      etb[f + NF * p] = (!b.per[d] && edge) ? b.bnd[side][d] : 0;
      int64_t e2 = p;
      int f2 = f;
      if (b.per[d] || !edge) {  // the brick neighbour across face f (periodic wrap)
        int64_t en[3] = {ec[0], ec[1], ec[2]};
        en[d] = side ? (ec[d] + 1 == b.n[d] ? 0 : ec[d] + 1) : (ec[d] == 0 ? b.n[d] - 1 : ec[d] - 1);
        int64_t gn = 0, st = 1;
        for (int q = 0; q < DIM; ++q) {
          gn += en[q] * st;
          st *= b.n[q];
        }
        e2 = inv[gn];
        f2 = f ^ 1;
      }
      for (int fn = 0; fn < Nfp; ++fn) {
        const int64_t slot = fn + (int64_t)Nfp * (f + (int64_t)NF * p);
        vmapM[slot] = (int64_t)Np * p + face_node_rt<DIM>(Nq, f, fn) + 1;
        vmapP[slot] = (int64_t)Np * e2 + face_node_rt<DIM>(Nq, f2, fn) + 1;
      }
    }
  }
}

}  // namespace

extern "C" int cb_brickmesh(int dim, int N, const int64_t *n, const double *const *x, const int *periodic,
                            const int64_t *boundary, double *elemtocoord, int64_t *elemtobndy, int64_t *vmapM,
                            int64_t *vmapP, cb_stream_t stream) {
  if ((dim != 2 && dim != 3) || N < 1 || !n || !x || !periodic || !elemtocoord || !elemtobndy || !vmapM || !vmapP)
    return solver_fail(CB_ERR_ARG, "cb_brickmesh: bad arguments");
  Brick b{};
  b.dim = dim;
  b.nelem = 1;
  for (int d = 0; d < dim; ++d) {
    if (n[d] < 1 || !x[d]) return solver_fail(CB_ERR_ARG, "cb_brickmesh: bad extent or coordinates");
    b.n[d] = n[d];
    b.x[d] = x[d];
    b.per[d] = periodic[d] != 0;
    b.bnd[0][d] = boundary ? boundary[2 * d] : 1;
    b.bnd[1][d] = boundary ? boundary[2 * d + 1] : 1;
    b.nelem *= n[d];
  }
  if (b.nelem > (1ll << 31)) return solver_fail(CB_ERR_ARG, "cb_brickmesh: too many elements");
  cudaStream_t st = (cudaStream_t)stream;
  const int64_t ne = b.nelem;
  const int T = 256;
  const int G = (int)std::min<int64_t>((ne + T - 1) / T, 148 * 32);
  double *cen = nullptr, *mm = nullptr;
  uint64_t *code = nullptr, *k0 = nullptr, *k1 = nullptr;
  int64_t *o0 = nullptr, *o1 = nullptr;
  void *tmp = nullptr;
  size_t tmpb = 0;
  cudaError_t e = cub::DeviceRadixSort::SortPairs(nullptr, tmpb, k0, k1, o0, o1, (int)ne, 0, 64, st);
  auto A = [&](void **p, size_t bytes) {
    if (e == cudaSuccess) e = cudaMallocAsync(p, bytes, st);
  };
  A((void **)&cen, sizeof(double) * dim * ne);
  A((void **)&mm, sizeof(double) * 6);
  A((void **)&code, sizeof(uint64_t) * dim * ne);
  A((void **)&k0, sizeof(uint64_t) * ne);
  A((void **)&k1, sizeof(uint64_t) * ne);
  A((void **)&o0, sizeof(int64_t) * ne);
  A((void **)&o1, sizeof(int64_t) * ne);
  A(&tmp, tmpb);
  if (e == cudaSuccess) {
    k_centroid<<<G, T, 0, st>>>(b, cen);
    k_minmax<<<1, 256, 0, st>>>(cen, dim, ne, mm);
    k_codes<<<G, T, 0, st>>>(b, cen, mm, code, o0);
    e = cudaGetLastError();
  }
  // stable LSD passes: word dim-1 (least significant) first, word 0 last
  for (int w = dim - 1; w >= 0 && e == cudaSuccess; --w) {
    k_gather_keys<<<G, T, 0, st>>>(code + (int64_t)w * ne, o0, ne, k0);
    if ((e = cudaGetLastError()) != cudaSuccess) break;
    e = cub::DeviceRadixSort::SortPairs(tmp, tmpb, k0, k1, o0, o1, (int)ne, 0, 64, st);
    std::swap(o0, o1);
  }
  int64_t *inv = (int64_t *)k1;  // the last key buffer is free
  if (e == cudaSuccess) {
    k_inverse<<<G, T, 0, st>>>(o0, ne, inv);
    if (dim == 2)
      k_connect<2><<<G, T, 0, st>>>(b, N + 1, o0, inv, elemtocoord, elemtobndy, vmapM, vmapP);
    else
      k_connect<3><<<G, T, 0, st>>>(b, N + 1, o0, inv, elemtocoord, elemtobndy, vmapM, vmapP);
    e = cudaGetLastError();
  }
  for (void *p : {(void *)cen, (void *)mm, (void *)code, (void *)k0, (void *)k1, (void *)o0, (void *)o1, tmp})
    if (p) cudaFreeAsync(p, st);
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "cb_brickmesh: %s", cudaGetErrorString(e));
}
