// Persistent, software-pipelined fused LSRK stage for sm_100a.
//
// One thread block per SM walks element groups g = blockIdx.x, +gridDim.x,...
// Each group's state slab Q[:, :, e0:e0+EPB] and geometry slab
// vgeo[:, 1:MJI, e0:e0+EPB] are contiguous in HBM, so they are staged into
// shared memory with bulk asynchronous copies (cp.async.bulk, completion
// tracked by an mbarrier) one group ahead: while group g is computed, group
// g+gridDim.x is in flight.  When a slab's byte size is not a multiple of 16
// (odd Nq) the same staging is done with per-thread cp.async copies.  The
// residual carry, the face normals and the neighbour traces of the current
// group are loaded into registers at the top of the iteration so that their
// latency overlaps the wait and the volume phase.
//
// Included from cb_kernels.cuh after the non-pipelined kernels.
#pragma once

namespace cb {

// ----------------------------------------------------------- PTX helpers
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: gives up after `limit` polls (each poll may suspend the warp
// for a short hardware-defined time) and reports failure.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, uint32_t limit) {
  for (uint32_t t = 0; t < limit; ++t)
    if (mbar_try_wait(bar, parity)) return true;
  return false;
}
template <int BYTES>
__device__ __forceinline__ void cp_async(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2;" ::"r"(smem_addr(dst)), "l"(src), "n"(BYTES)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Devices for which per-device launch facts (SM count, occupancy) are cached.
constexpr int MAX_DEVICES = 128;

inline int num_sms() {
  static int cached[MAX_DEVICES] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= MAX_DEVICES) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }
  if (!cached[dev]) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    cached[dev] = v > 0 ? v : 148;
  }
  return cached[dev];
}

constexpr uint32_t WAIT_LIMIT = 1u << 22;
// Poll limit of the timeout test hook (a wait that is meant to give up).
constexpr uint32_t PROBE_WAIT_LIMIT = 1u << 12;
constexpr size_t SMEM_LIMIT = 227 * 1024;

// Row stride (in elements) of the contraction buffers: >= Nq, a multiple of
// the 16-byte vector width, and an odd number of 16-byte chunks so that the
// rows read by the 8-32 lanes of a warp fall into distinct shared-memory banks.
template <typename T>
__host__ __device__ constexpr int row_stride(int nq) {
  int vw = 16 / (int)sizeof(T), rs = ((nq + vw - 1) / vw) * vw;
  return ((rs / vw) % 2 == 1) ? rs : rs + vw;
}

// Shared-memory plan of the pipelined stage for one (dim, Nq, T) and X times
// the elements per group of Cfg.
template <int DIM, int Nq, typename T, int X = 1>
struct Pipe {
  using C = CfgX<DIM, Nq, X>;
  static constexpr int NS = Lay<DIM>::NS;
  static constexpr int NG = DIM * DIM + 2;  // staged vgeo fields: metric, MJ, MJI
  static constexpr int VW = 16 / (int)sizeof(T);   // elements per 16-byte vector
  static constexpr int MV = ((Nq + VW - 1) / VW) * VW;  // contraction length, padded
  static constexpr int RS = row_stride<T>(Nq);
  static constexpr int NR = ipow(Nq, DIM - 1);     // rows per element and field
  static constexpr size_t QB = sizeof(T) * (size_t)C::Np * NS;   // bytes per element
  static constexpr size_t GB = sizeof(T) * (size_t)C::Np * NG;
  static constexpr bool BULK =
      QB % 16 == 0 && GB % 16 == 0 && (sizeof(T) * (size_t)C::Np * Lay<DIM>::NVG) % 16 == 0;
  static constexpr size_t pad16(size_t b) { return (b + 15) & ~size_t(15); }
  static constexpr size_t OFF_D = 16;  // D^T rows, padded like the flux rows
  static constexpr size_t OFF_ST = OFF_D + pad16(sizeof(T) * Nq * RS);
  static constexpr size_t STAGE = C::EPB * (QB + GB);
  static constexpr size_t OFF_F = OFF_ST + 2 * pad16(STAGE);
  static constexpr size_t FDIR = (size_t)NS * C::EPB * NR * RS;  // elements per direction
  static constexpr size_t FLUX = sizeof(T) * DIM * FDIR;
  static constexpr size_t FFB = sizeof(T) * (size_t)C::NFACE * NS * C::EPB * C::Nfp;
  // face fluxes have their own buffer: they are produced in the same phase
  // as the volume fluxes
  static constexpr size_t OFF_FF = OFF_F + pad16(FLUX);
  static constexpr size_t smem() { return OFF_FF + FFB; }
  static constexpr bool OK = smem() <= SMEM_LIMIT;
};

template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using type = double2;
};
template <>
struct Vec16<float> {
  using type = float4;
};

// Load MV consecutive elements (16-byte aligned) into registers.
template <typename T, int MV>
__device__ __forceinline__ void load_row(const T *src, T *dst) {
  using V = typename Vec16<T>::type;
  constexpr int VW = 16 / (int)sizeof(T);
#pragma unroll
  for (int q = 0; q < MV / VW; ++q) {
    const V v = reinterpret_cast<const V *>(src)[q];
    const T *pv = reinterpret_cast<const T *>(&v);
#pragma unroll
    for (int t = 0; t < VW; ++t) dst[q * VW + t] = pv[t];
  }
}

// Tensor-product contraction of one node from direction-major flux rows:
// R[s] += Σ_m D[m,i] Fξ[m;j,k] (then η, then ζ), each sum in m order.
template <int DIM, int Nq, typename T, int X = 1>
__device__ __forceinline__ void contract_rows(const T *flux, const T *DT, int el, int n, T *R) {
  using PP = Pipe<DIM, Nq, T, X>;
  constexpr int NS = Lay<DIM>::NS, MV = PP::MV, RS = PP::RS, NR = PP::NR, EPB = CfgX<DIM, Nq, X>::EPB;
  const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
#pragma unroll
  for (int r = 0; r < DIM; ++r) {
    const int idx = r == 0 ? i : (r == 1 ? j : k);
    const int row = DIM == 2 ? (r == 0 ? j : i) : (r == 0 ? j + Nq * k : (r == 1 ? i + Nq * k : i + Nq * j));
    T d[MV];
    load_row<T, MV>(DT + idx * RS, d);
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      T f[MV];
      load_row<T, MV>(flux + r * PP::FDIR + ((size_t)(s * EPB + el) * NR + row) * RS, f);
      T acc = R[s];
#pragma unroll
      for (int m = 0; m < MV; ++m) acc += d[m] * f[m];
      R[s] = acc;
    }
  }
}

template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS, 1)
k_stage_pipe(const T *__restrict__ Qin, T *__restrict__ Qout, T *__restrict__ rhs,
             const T *__restrict__ vgeo, const T *__restrict__ sgeo,
             const int32_t *__restrict__ nbr, const T *__restrict__ D, int64_t nelem,
             PhysT<T> p, Offs<T, Lay<DIM>::NS> qref, T rka, T rkbdt, unsigned *status) {
  using C = Cfg<DIM, Nq>;
  using PP = Pipe<DIM, Nq, T>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, EPB = C::EPB, SP = C::SLOTS;
  constexpr int NG = PP::NG, MJI = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  constexpr int FS = EPB * Nfp;
  constexpr int RS = PP::RS, NR = PP::NR;
  constexpr size_t STRIDE = PP::pad16(PP::STAGE) / sizeof(T);  // elements between the two stages
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem_raw);
  T *DT = reinterpret_cast<T *>(smem_raw + PP::OFF_D);
  T *stage0 = reinterpret_cast<T *>(smem_raw + PP::OFF_ST);
  T *sF = reinterpret_cast<T *>(smem_raw + PP::OFF_F);
  T *FF = reinterpret_cast<T *>(smem_raw + PP::OFF_FF);
  const int tid = threadIdx.x;
  const int64_t ngroups = (nelem + EPB - 1) / EPB;

  // stage b layout: [EPB][NS][Np] state, then [EPB][NG][Np] geometry
  auto issue = [&](int64_t g, int b) {
    const int64_t e0 = g * EPB;
    const int nv = (int)((nelem - e0) < EPB ? (nelem - e0) : EPB);
    T *dq = stage0 + b * STRIDE, *dg = dq + EPB * Np * NS;
    if constexpr (PP::BULK) {
      if (tid == 0) {
        fence_proxy_async();
        mbar_expect_tx(&bars[b], (uint32_t)(nv * (PP::QB + PP::GB)));
        bulk_g2s(dq, Qin + e0 * Np * NS, (uint32_t)(nv * PP::QB), &bars[b]);
        for (int el = 0; el < nv; ++el)
          bulk_g2s(dg + el * Np * NG, vgeo + (e0 + el) * Np * NVG, (uint32_t)PP::GB, &bars[b]);
      }
    } else {
      const T *srcQ = Qin + e0 * Np * NS;
      for (int t = tid; t < nv * Np * NS; t += C::THREADS) cp_async<sizeof(T)>(dq + t, srcQ + t);
      for (int t = tid; t < nv * Np * NG; t += C::THREADS) {
        const int el = t / (Np * NG), r = t % (Np * NG);
        cp_async<sizeof(T)>(dg + t, vgeo + (e0 + el) * Np * NVG + r);
      }
      cp_async_commit();
    }
  };

  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  // D^T rows (DT[i][m] = D[m, i]) and the padded flux columns start at zero
  for (int t = tid; t < Nq * RS; t += C::THREADS) {
    const int i = t / RS, m = t % RS;
    DT[t] = m < Nq ? D[m + Nq * i] : T(0);
  }
  if constexpr (PP::MV > Nq)
    for (size_t t = tid; t < (size_t)DIM * PP::FDIR; t += C::THREADS)
      if ((int)(t % RS) >= Nq) sF[t] = T(0);
  __syncthreads();
  if ((int64_t)blockIdx.x < ngroups) issue(blockIdx.x, 0);

  // neighbour codes of this thread's face slots, loaded one group ahead so
  // that the dependent neighbour-trace loads can start at the top of the
  // iteration
  int32_t nbn[C::FPT];
  auto load_nbr = [&](int64_t g, int32_t *dst) {
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF;
      const int64_t e = g * EPB + el;
      dst[u] = (g < ngroups && fs < C::FSLOTS && e < nelem) ? nbr[f + NF * e] : NBR_WALL;
    }
  };
  load_nbr(blockIdx.x, nbn);

  bool bad = false, timed_out = false;
  int it = 0;
  for (int64_t g = blockIdx.x; g < ngroups; g += gridDim.x, ++it) {
    const int b = it & 1;
    const int64_t e0 = g * EPB;
    const int64_t gn = g + gridDim.x;
    if (gn < ngroups) issue(gn, b ^ 1);
    else if constexpr (!PP::BULK) cp_async_commit();  // keep one group per iteration

    // ---- register prefetch: residual carry, face normals, neighbour traces
    T R[C::NPT][NS];
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = tid + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      if (slot < SP && e0 + el < nelem)
#pragma unroll
        for (int s = 0; s < NS; ++s) R[u][s] = rhs[n + Np * (s + NS * (e0 + el))];
    }
    T qP[C::FPT][NS], nrm[C::FPT][DIM], smj[C::FPT];
    int32_t nbv[C::FPT];
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) nbv[u] = nbn[u];
    load_nbr(gn, nbn);
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
      const int64_t e = e0 + el;
      if (fs < C::FSLOTS && e < nelem) {
        const T *sg = sgeo + (int64_t)NSG * (fn + (int64_t)Nfp * (f + NF * e));
#pragma unroll
        for (int c = 0; c < DIM; ++c) nrm[u][c] = sg[c];
        smj[u] = sg[DIM];
        if (nbv[u] >= 0) {
          const int64_t e2 = nbv[u] >> 3;
          const int vP = face_node<DIM, Nq>(nbv[u] & 7, fn);
#pragma unroll
          for (int s = 0; s < NS; ++s) qP[u][s] = Qin[vP + Np * (s + NS * e2)] + qref.v[s];
        }
      }
    }

    // ---- wait for this group's slabs (each thread observes the mbarrier; a
    // wait that gives up is agreed on at the mid-iteration barrier)
    if constexpr (PP::BULK) {
      if (!mbar_wait_bounded(&bars[b], (uint32_t)((it >> 1) & 1), WAIT_LIMIT)) timed_out = true;
    } else {
      cp_async_wait<1>();
      __syncthreads();
    }
    const T *Qs = stage0 + b * STRIDE, *Gs = Qs + EPB * Np * NS;

    // ---- phase A: contravariant volume fluxes and face fluxes
    T buoy[C::NPT];
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = tid + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      buoy[u] = T(0);
      if (slot < SP && e0 + el < nelem) {
        T q[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) q[s] = Qs[(el * NS + s) * Np + n] + qref.v[s];
        T met[DIM][DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int c = 0; c < DIM; ++c) met[r][c] = Gs[(el * NG + r + DIM * c) * Np + n];
        const T MJ = Gs[(el * NG + DIM * DIM) * Np + n];
        const T gc = p.grav != T(0) ? vgeo[n + Np * (GC + NVG * (e0 + el))] : T(0);
        const T ri = T(1) / q[IR];
        const T P = pressure_ri<DIM, T>(q, ri, gc, p);
        T f[NS][DIM];
        euler_flux_ri<DIM, T>(q, ri, P, f);
        const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          // row of this node in direction r and its position along the row
          const int row = DIM == 2 ? (r == 0 ? j : i) : (r == 0 ? j + Nq * k : (r == 1 ? i + Nq * k : i + Nq * j));
          const int pos = r == 0 ? i : (r == 1 ? j : k);
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            T a = met[r][0] * f[s][0] + met[r][1] * f[s][1];
            if (DIM == 3) a = a + met[r][2] * f[s][2];
            sF[r * PP::FDIR + ((size_t)(s * EPB + el) * NR + row) * RS + pos] = MJ * a;
          }
        }
        buoy[u] = MJ * q[IR] * p.grav;
      }
    }
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
      if (fs < C::FSLOTS && e0 + el < nelem) {
        const int vM = face_node<DIM, Nq>(f, fn);
        T qM[NS], qq[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) qM[s] = Qs[(el * NS + s) * Np + vM] + qref.v[s];
        const T gM = p.grav != T(0) ? vgeo[vM + Np * (GC + NVG * (e0 + el))] : T(0);
        const T riM = T(1) / qM[IR];
        const T PM = pressure_ri<DIM, T>(qM, riM, gM, p);
        T PPv, riP;
        if (nbv[u] >= 0) {
#pragma unroll
          for (int s = 0; s < NS; ++s) qq[s] = qP[u][s];
          T gP = T(0);
          if (p.grav != T(0)) {
            const int64_t e2 = nbv[u] >> 3;
            gP = vgeo[face_node<DIM, Nq>(nbv[u] & 7, fn) + Np * (GC + NVG * e2)];
          }
          riP = T(1) / qq[IR];
          PPv = pressure_ri<DIM, T>(qq, riP, gP, p);
        } else {
          wall_state<DIM, T>(qM, nrm[u], qq);
          riP = riM;
          PPv = PM;
        }
        T out[NS];
        rusanov_n<DIM, T>(qM, riM, PM, qq, riP, PPv, nrm[u], p, out);
#pragma unroll
        for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = smj[u] * out[s];
      }
    }
    // A wait that gave up: store nothing for this group, flag the status,
    // let the issued copies land (bounded) and leave.
    if (__syncthreads_or(timed_out)) {
      if (tid == 0) {
        atomicOr(status, ST_TIMEOUT);
        if constexpr (PP::BULK) {
          mbar_wait_bounded(&bars[b], (uint32_t)((it >> 1) & 1), WAIT_LIMIT);
          if (gn < ngroups) mbar_wait_bounded(&bars[b ^ 1], (uint32_t)(((it + 1) >> 1) & 1), WAIT_LIMIT);
        }
      }
      if constexpr (!PP::BULK) cp_async_wait<0>();
      return;
    }
    // ---- phase B: carry - source + volume contraction - face terms, update
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = tid + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      const int64_t e = e0 + el;
      if (slot < SP && e < nelem) {
        R[u][DIM - 1] -= buoy[u];
        contract_rows<DIM, Nq, T>(sF, DT, el, n, R[u]);
        gather_face_terms<DIM, Nq, EPB, T>(FF, el, n, R[u]);
        const T mji = Gs[(el * NG + MJI) * Np + n];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const T qn = Qs[(el * NS + s) * Np + n] + rkbdt * R[u][s] * mji;
          bad |= !isfinite(qn);
          Qout[n + Np * (s + NS * e)] = qn;
          rhs[n + Np * (s + NS * e)] = R[u][s] * rka;
        }
      }
    }
    __syncthreads();  // stage b, the flux rows and FF are free for reuse
  }
  if constexpr (!PP::BULK) cp_async_wait<0>();
  if (bad) atomicOr(status, ST_NONFINITE);
}

}  // namespace cb
