// Fused LSRK stage with the D contraction on the FP64 tensor cores (sm_100a).
//
// 3-D hexahedra at N = 7 (Nq = 8, 512 nodes per element), FP64 and FP32
// storage (the contraction in FP64 either way).  The same
// stage as k_stage_pipe2 (volume + Rusanov face + LSRK update, state read
// from one buffer and written to the other), with a different division of
// the work inside an element:
//
//   * 256 threads (8 warps) per element; warp k owns plane k of the element
//     and lane (g = lane / 4, t = lane % 4) the two nodes i = 2t, 2t + 1,
//     j = g — the positions of an 8 x 8 accumulator fragment of
//     mma.sync.m8n8k4.f64;
//   * the tensor-product contraction with D runs as 8 x 8 x 8 matrix
//     products on the FP64 tensor pipe (DMMA).  With F, G, H the
//     contravariant fluxes of the three directions, plane k of an element
//     needs  R_xi  = F_kᵀ·D (rows j, columns i),  R_eta = Dᵀ·G_k (rows j,
//     columns i)  — both land in the owning lanes — and the zeta term
//     R_zeta[(i, j), k] = H[(i, j), :]·D, whose 8 x 8 tiles (one j per warp)
//     are computed by one warp and handed to the plane owners through shared
//     memory.  All three products use the same D fragment
//     (D[t + 4 ks, g], ks = 0, 1), kept in two registers.  Each flux value
//     is read from shared memory once per direction (one 8-byte fragment
//     element), instead of a whole row per node as in the CUDA-core
//     contraction;
//   * the neighbours' state traces of each face slot are loaded into
//     registers before the wait for the state slab (FP64), or copied into
//     shared memory one group ahead by the thread that owns the slot
//     (cp.async, issued as soon as it has used the current ones; FP32);
//   * only the state (read by the face phase for other threads' nodes) is
//     staged in shared memory, by a bulk copy one group ahead; the metric,
//     the residual carry and the face geometry are each read by the one
//     thread that needs them, straight from L2, where a bulk L2 prefetch
//     issued one group ahead has placed them.  That leaves room for two
//     blocks (16 warps) per SM.
//
// Summation order: R = carry - buoyancy; R += (xi + eta products, each
// accumulated by the tensor core); R += zeta product; face terms in face
// order; the reference sums the same terms left to right, so FP64 results
// agree to round-off (the oracle parity tests hold them to 1e-12).
#pragma once

namespace cb {

// D = A·B + C for one 8x8x4 FP64 tile: a = A[g][t], b = B[t][g],
// (c0, c1) = C[g][2t], C[g][2t + 1] with g = lane / 4, t = lane % 4.
__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b, double c0, double c1) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%4, %5};"
               : "=d"(d0), "=d"(d1)
               : "d"(a), "d"(b), "d"(c0), "d"(c1));
}

__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Shared-memory plan of the tensor-core stage (per block, one element per
// group) for state, geometry, carry and flux planes stored in T.  The FP32
// form (T = float) computes its fluxes in FP32, contracts them with D on the
// FP64 tensor pipe (the FP32 plane values and D converted to FP64 as the
// fragments are loaded: the products are exact, the sums are rounded once)
// and rounds the result to FP32.
template <typename T>
struct PipeMT {
  static constexpr int DIM = 3, Nq = 8, Np = 512, Nfp = 64, NF = 6, NS = 5, NVG = 14, NSG = 5;
  static constexpr int THREADS = 256, WARPS = 8;
  static constexpr int FSLOTS = NF * Nfp, FPT = (FSLOTS + THREADS - 1) / THREADS;
  static constexpr size_t QB = sizeof(T) * Np * NS;             // state slab (bulk copy)
  static constexpr size_t GB = sizeof(T) * Np * (DIM * DIM + 2);  // metric, MJ, MJI (L2 prefetch)
  static constexpr size_t SB = sizeof(T) * NSG * Nfp * NF;      // face geometry (L2 prefetch)
  // F and G planes of one warp: [NS][2][64] (row j, swizzled column i)
  static constexpr int FGW = NS * 2 * 64;
  // H (then the zeta products in place): [NS][8 planes][68], planes padded so
  // that the fragment loads of a half warp hit distinct banks
  static constexpr int HP = 68, HS = 8 * HP;
  static constexpr size_t OFF_S = 16;
  static constexpr size_t OFF_FG = OFF_S + QB;
  static constexpr size_t OFF_HZ = OFF_FG + sizeof(T) * WARPS * FGW;
  static constexpr size_t OFF_FF = OFF_HZ + sizeof(T) * NS * HS;
  static constexpr size_t FFB = sizeof(T) * NF * NS * Nfp;
  // FP32: neighbour state traces of each face slot, [NS][FSLOTS]: every
  // thread copies its own slots' traces of the next group asynchronously
  // (cp.async) once it has used this group's, and reads them only itself.
  // FP64 loads them into registers at the top of the group instead: with
  // the 15 KB buffer its two blocks leave 28 KB of L1 per SM and the stage
  // took 1.13 ms instead of 0.98 at 32^3; FP32 went from 0.530 to 0.519 ms.
  static constexpr bool ASYNC_QP = sizeof(T) == 4;
  static constexpr size_t OFF_QP = OFF_FF + FFB;
  static constexpr size_t QPB = ASYNC_QP ? sizeof(T) * NS * FSLOTS : 0;
  static constexpr size_t smem() { return OFF_QP + QPB; }  // item sources append their ring here
  // PFD = -1: each group's metric, carry and face geometry are prefetched
  // into L2 at the top of its own iteration.  Measured on B200 (16^3-hex
  // launch, ncu): prefetching one or two groups ahead lets the streaming
  // traffic evict the lines before use, so they are read from HBM twice
  // (DRAM reads 1.17x / 1.62x the algorithmic bytes); same-group prefetch
  // reads 1.00x and is the fastest (127.6 us against 135 us without a
  // prefetch and 162 us for the CUDA-core stage).
  // FP32: the half-size plan (about 50 KB) leaves room for three blocks per
  // SM if the registers fit 85 per thread (measured at 32^3: 0.566 ms per
  // stage; four blocks at 64 registers spill and take 0.637 ms)
  // (FP32 with the prefetch one group ahead: 0.567 ms, the same)
  static constexpr int MINB = sizeof(T) == 8 ? 2 : 3, PFD = -1;
  // whether this stage is the default of its shape (the faster on B200 at
  // 32^3 hexes: FP64 0.974 ms per stage against 1.17 ms for the CUDA-core
  // stage, FP32 0.719 against 0.744 ms)
  static constexpr bool DEFAULT = true;
};
using PipeM = PipeMT<double>;

template <typename T>
struct Vec2;
template <>
struct Vec2<double> {
  using type = double2;
};
template <>
struct Vec2<float> {
  using type = float2;
};

// Position of (i, j) in an 8 x 8 plane (a warp's F or G plane, a plane of
// H / zeta products): row j, column i XOR 5 on rows 2, 3, 6, 7.  With it the
// three access patterns of a half warp touch 16 distinct 8-byte banks: the
// owners' stores (i = 2t + c, j = g, one node c at a time), the A-fragment
// loads (i = t + 4 ks, j = g) and the B-fragment loads (i = g, j = t + 4 ks).
__device__ __forceinline__ int fg_pos(int i, int j) { return j * 8 + (i ^ (((j >> 1) & 1) * 5)); }

// MINB: resident blocks per SM the registers are sized for; PFD: how many
// groups ahead the bulk L2 prefetch of a group's metric, carry and face
// geometry is issued (0: none, the loads go to HBM directly; -1: for the
// group itself, at the top of its iteration).
template <typename Src, int MINB = PipeM::MINB, int PFD = PipeM::PFD>
__global__ void __launch_bounds__(PipeM::THREADS, MINB)
    k_stage_mma(Src src, PhysT<typename Src::Real> p, typename Src::Real rka) {
  using T = typename Src::Real;  // storage (and, for float, flux and update arithmetic)
  using A = double;              // tensor-core operands and products (planes stored in T)
  using V2 = typename Vec2<T>::type;
  using PM = PipeMT<T>;
  constexpr int DIM = 3, Nq = 8, Np = 512, Nfp = 64, NF = 6, NS = 5, NVG = 14, NSG = 5, IR = 3;
  constexpr int MJF = DIM * DIM, MJIF = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *barS = reinterpret_cast<uint64_t *>(smem_raw);
  T *S = reinterpret_cast<T *>(smem_raw + PM::OFF_S);
  T *FGall = reinterpret_cast<T *>(smem_raw + PM::OFF_FG);
  T *HZ = reinterpret_cast<T *>(smem_raw + PM::OFF_HZ);
  T *FF = reinterpret_cast<T *>(smem_raw + PM::OFF_FF);
  T *QPs = reinterpret_cast<T *>(smem_raw + PM::OFF_QP);
  const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31, g = lane >> 2, t = lane & 3;
  T *FG = FGall + w * PM::FGW;
  const int n0 = 2 * t + 8 * g + 64 * w;  // the lane's nodes n0, n0 + 1

  auto issue_S = [&](int it) {  // thread 0 only
    if (src.skip_copy(it)) return;
    fence_proxy_async();
    mbar_expect_tx(&barS[0], (uint32_t)PM::QB);
    bulk_g2s(S, src.Qin(it) + src.e0(it) * Np * NS, (uint32_t)PM::QB, &barS[0]);
  };
  auto prefetch_group = [&](int it) {  // thread 0 only: metric, carry, face geometry into L2
    const int64_t e = src.e0(it);
    prefetch_l2(src.vgeo(it) + e * Np * NVG, (uint32_t)PM::GB);
    prefetch_l2(src.rhs(it) + e * Np * NS, (uint32_t)PM::QB);
    prefetch_l2(src.sgeo(it) + e * (int64_t)(NSG * Nfp * NF), (uint32_t)PM::SB);
  };

  src.begin(smem_raw + PM::smem());
  if (tid == 0) {
    mbar_init(&barS[0], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (tid == 0 && src.valid(0)) {
    issue_S(0);
    for (int j = 0; j < PFD && src.valid(j); ++j) prefetch_group(j);  // PFD > 0
  }

  int32_t nbn[PM::FPT];
  auto load_nbr = [&](int it, int32_t *dst) {
    const bool ok = src.valid(it);
    const int64_t e0 = ok ? src.e0(it) : 0;
    const int32_t *nb = src.nbr(it);
#pragma unroll
    for (int u = 0; u < PM::FPT; ++u) {
      const int fs = tid + u * PM::THREADS;
      dst[u] = (ok && fs < PM::FSLOTS) ? nb[fs / Nfp + NF * e0] : NBR_WALL;
    }
  };
  load_nbr(0, nbn);
  // this thread's face slots' neighbour traces of group `it` (stored values,
  // without the offsets) into QPs, as one cp.async group
  auto issue_qp = [&](int it, const int32_t *codes) {
    if constexpr (!PM::ASYNC_QP) return;
    const T *Qn = src.Qin(it);
#pragma unroll
    for (int u = 0; u < PM::FPT; ++u) {
      const int fs = tid + u * PM::THREADS;
      if (fs < PM::FSLOTS && codes[u] >= 0) {
        const int64_t e2 = codes[u] >> 3;
        const int vP = face_node<DIM, Nq>(codes[u] & 7, fs % Nfp);
#pragma unroll
        for (int s = 0; s < NS; ++s) cp_async<sizeof(T)>(QPs + s * PM::FSLOTS + fs, Qn + vP + Np * (s + NS * e2));
      }
    }
    cp_async_commit();
  };
  if (PM::ASYNC_QP && src.valid(0)) issue_qp(0, nbn);

  const T *curD = nullptr;
  A Dg0 = A(0), Dg1 = A(0);  // D[t, g] and D[t + 4, g] (column-major D[m + Nq i])
  bool timed_out = false;
  for (int it = 0; src.valid(it); ++it) {
    const int64_t e0 = src.e0(it);
    const bool more = src.valid(it + 1);
    if (PFD > 0 && tid == 0 && src.valid(it + PFD)) prefetch_group(it + PFD);
    if (PFD < 0 && tid == 0) prefetch_group(it);
    if (tid == Src::PUBLISHER) src.prefetch();
    const T *__restrict__ Qin = src.Qin(it);
    const T *__restrict__ vg = src.vgeo(it) + e0 * Np * NVG;
    const T *__restrict__ sg = src.sgeo(it) + e0 * (int64_t)(NSG * Nfp * NF);
    T qr[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qr[s] = src.qref(it, s);
    if (src.D(it) != curD) {
      curD = src.D(it);
      Dg0 = A(curD[t + Nq * g]);
      Dg1 = A(curD[t + 4 + Nq * g]);
    }

    // ---- loads that do not need the staged state: neighbour traces and
    // face geometry
    T *__restrict__ rhs = src.rhs(it) + e0 * Np * NS;
    int32_t nbv[PM::FPT];
#pragma unroll
    for (int u = 0; u < PM::FPT; ++u) nbv[u] = nbn[u];
    load_nbr(it + 1, nbn);
    T qP[PM::FPT][NS], nrm[PM::FPT][DIM], smj[PM::FPT];  // qP: register traces (FP64)
#pragma unroll
    for (int u = 0; u < PM::FPT; ++u) {
      const int fs = tid + u * PM::THREADS;
      if (fs < PM::FSLOTS) {
        const int f = fs / Nfp, fn = fs % Nfp;
        const T *sgp = sg + NSG * (fn + Nfp * f);
#pragma unroll
        for (int c = 0; c < DIM; ++c) nrm[u][c] = sgp[c];
        smj[u] = sgp[DIM];
        if constexpr (!PM::ASYNC_QP) {
          if (nbv[u] >= 0) {
            const int64_t e2 = nbv[u] >> 3;
            const int vP = face_node<DIM, Nq>(nbv[u] & 7, fn);
#pragma unroll
            for (int s = 0; s < NS; ++s) qP[u][s] = Qin[vP + Np * (s + NS * e2)] + qr[s];
          }
        }
      }
    }
    // the lane's metric (+ MJ): FP32 loads it here, so that its latency
    // overlaps the wait for the state slab and the face phase (FP64 waits
    // until after the face phase, whose registers it would crowd: 100 bytes
    // of spill at 128 registers)
    V2 met[DIM * DIM + 1];
    if constexpr (sizeof(T) == 4) {
#pragma unroll
      for (int f = 0; f <= MJF; ++f) met[f] = *reinterpret_cast<const V2 *>(vg + n0 + Np * f);
    }
    if (!mbar_wait_bounded(&barS[0], (uint32_t)(it & 1), src.wait_limit())) timed_out = true;

    // ---- face fluxes (any thread, any face node) into FF; FP32: the
    // neighbour traces were copied by this thread during the previous group
    if constexpr (PM::ASYNC_QP) cp_async_wait<0>();
#pragma unroll
    for (int u = 0; u < PM::FPT; ++u) {
      const int fs = tid + u * PM::THREADS;
      if (fs < PM::FSLOTS) {
        const int f = fs / Nfp, fn = fs % Nfp;
        const int vM = face_node<DIM, Nq>(f, fn);
        T qM[NS], qq[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) qM[s] = S[s * Np + vM] + qr[s];
        const T gM = p.grav != T(0) ? vg[vM + Np * GC] : T(0);
        const T riM = T(1) / qM[IR];
        const T PMv = pressure_ri<DIM, T>(qM, riM, gM, p);
        T PPv, riP;
        if (nbv[u] >= 0) {
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            if constexpr (PM::ASYNC_QP)
              qq[s] = QPs[s * PM::FSLOTS + fs] + qr[s];
            else
              qq[s] = qP[u][s];
          }
          T gP = T(0);
          if (p.grav != T(0)) {
            const int64_t e2 = nbv[u] >> 3;
            gP = src.vgeo(it)[face_node<DIM, Nq>(nbv[u] & 7, fn) + Np * (GC + NVG * e2)];
          }
          riP = T(1) / qq[IR];
          PPv = pressure_ri<DIM, T>(qq, riP, gP, p);
        } else {
          wall_state<DIM, T>(qM, nrm[u], qq);
          riP = riM;
          PPv = PMv;
        }
        T out[NS];
        rusanov_n<DIM, T>(qM, riM, PMv, qq, riP, PPv, nrm[u], p, out);
#pragma unroll
        for (int s = 0; s < NS; ++s) FF[(f * NS + s) * Nfp + fn] = smj[u] * out[s];
      }
    }
    // this thread has read its slots: copy the next group's traces into them
    if (PM::ASYNC_QP && more) issue_qp(it + 1, nbn);

    // ---- volume fluxes of the lane's two nodes, one node at a time: F, G
    // into the warp's planes, H into the shared zeta buffer
    if constexpr (sizeof(T) == 8) {
#pragma unroll
      for (int f = 0; f <= MJF; ++f) met[f] = *reinterpret_cast<const V2 *>(vg + n0 + Np * f);
    }
    T qd[2][NS], buoy[2];
#pragma unroll
    for (int c = 0; c < 2; ++c) {
      const int n = n0 + c;
      T q[NS];
#pragma unroll
      for (int s = 0; s < NS; ++s) {
        qd[c][s] = S[s * Np + n];
        q[s] = qd[c][s] + qr[s];
      }
      T mt[DIM][DIM], MJ;
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int cc = 0; cc < DIM; ++cc) mt[r][cc] = c ? met[r + DIM * cc].y : met[r + DIM * cc].x;
      MJ = c ? met[MJF].y : met[MJF].x;
      const T gc = p.grav != T(0) ? vg[n + Np * GC] : T(0);
      const T ri = T(1) / q[IR];
      const T P = pressure_ri<DIM, T>(q, ri, gc, p);
      T f[NS][DIM];
      euler_flux_ri<DIM, T>(q, ri, P, f);
      const int pf = fg_pos(2 * t + c, g);
#pragma unroll
      for (int r = 0; r < DIM; ++r)
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          T a = mt[r][0] * f[s][0] + mt[r][1] * f[s][1];
          a = a + mt[r][2] * f[s][2];
          T *dst = r < 2 ? FG + (s * 2 + r) * 64 : HZ + s * PM::HS + w * PM::HP;
          dst[pf] = MJ * a;
        }
      buoy[c] = MJ * q[IR] * p.grav;
    }
    __syncwarp();
    // ---- xi and eta products of this warp's plane (warp-private planes)
    A acc[NS][2];
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      const T *Fp = FG + (s * 2 + 0) * 64, *Gp = FG + (s * 2 + 1) * 64;
      A c0 = A(0), c1 = A(0);
      // xi: C[j][i] += Σ_m F[m, j]·D[m, i]   (A = F_kᵀ, B = D)
      dmma(c0, c1, A(Fp[fg_pos(t, g)]), Dg0, c0, c1);
      dmma(c0, c1, A(Fp[fg_pos(t + 4, g)]), Dg1, c0, c1);
      // eta: C[j][i] += Σ_m D[m, j]·G[i, m]   (A = Dᵀ, B = G_k)
      dmma(c0, c1, Dg0, A(Gp[fg_pos(g, t)]), c0, c1);
      dmma(c0, c1, Dg1, A(Gp[fg_pos(g, t + 4)]), c0, c1);
      acc[s][0] = c0;
      acc[s][1] = c1;
    }

    // Mid-group barrier: H and FF are complete, S is no longer read.  It
    // also agrees on whether any wait gave up (then: store nothing, flag the
    // status, let the issued copy land, leave).
    if (__syncthreads_or(timed_out)) {
      if (tid == 0) {
        atomicOr(src.status(it), ST_TIMEOUT);
        mbar_wait_bounded(&barS[0], (uint32_t)(it & 1), src.wait_limit());
      }
      if constexpr (PM::ASYNC_QP) cp_async_wait<0>();  // this thread's trace copies land before the block leaves
      return;
    }
    if (tid == 0 && more) issue_S(it + 1);
    if ((tid >> 5) == (Src::PUBLISHER >> 5)) src.publish(it);

    // ---- zeta products: warp w computes rows (i, j = w), columns k, and
    // writes them over the H values it has just read (the same positions)
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      T *Hs = HZ + s * PM::HS;
      const int pz = fg_pos(g, w);
      const A a0 = A(Hs[t * PM::HP + pz]), a1 = A(Hs[(t + 4) * PM::HP + pz]);
      A z0 = A(0), z1 = A(0);
      dmma(z0, z1, a0, Dg0, z0, z1);
      dmma(z0, z1, a1, Dg1, z0, z1);
      // (FP32: rounded here instead of when added to R — the same rounding)
      Hs[(2 * t) * PM::HP + pz] = T(z0);
      Hs[(2 * t + 1) * PM::HP + pz] = T(z1);
    }
    // residual carry and 1/MJ of the lane's nodes
    V2 cr[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) cr[s] = *reinterpret_cast<const V2 *>(rhs + n0 + Np * s);
    const V2 mji = *reinterpret_cast<const V2 *>(vg + n0 + Np * MJIF);
    __syncthreads();  // zeta products complete

    // ---- carry - source + products - face terms, update
    T *__restrict__ Qout = src.Qout(it) + e0 * Np * NS;
    const T rkbdt = src.rkbdt(it);
    bool bad = false;
    const int j = g, k = w;
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      // the lane's two zeta products: one 16-byte pair, in swapped order on
      // the rows whose column index is XOR-ed with 5
      const V2 zp = *reinterpret_cast<const V2 *>(HZ + s * PM::HS + w * PM::HP + fg_pos(2 * t, g) - (((g >> 1) & 1)));
      const V2 z = ((g >> 1) & 1) ? V2{zp.y, zp.x} : zp;
      T R[2] = {cr[s].x, cr[s].y};
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (s == DIM - 1) R[c] -= buoy[c];
        R[c] += T(acc[s][c]);
        R[c] += c ? z.y : z.x;
        const int i = 2 * t + c;
        if (i == 0) R[c] -= FF[(0 * NS + s) * Nfp + j + Nq * k];
        if (i == Nq - 1) R[c] -= FF[(1 * NS + s) * Nfp + j + Nq * k];
        if (j == 0) R[c] -= FF[(2 * NS + s) * Nfp + i + Nq * k];
        if (j == Nq - 1) R[c] -= FF[(3 * NS + s) * Nfp + i + Nq * k];
        if (k == 0) R[c] -= FF[(4 * NS + s) * Nfp + i + Nq * j];
        if (k == Nq - 1) R[c] -= FF[(5 * NS + s) * Nfp + i + Nq * j];
      }
      const T q0 = qd[0][s] + rkbdt * R[0] * mji.x, q1 = qd[1][s] + rkbdt * R[1] * mji.y;
      bad |= !isfinite(q0) || !isfinite(q1);
      *reinterpret_cast<V2 *>(Qout + n0 + Np * s) = V2{q0, q1};
      *reinterpret_cast<V2 *>(rhs + n0 + Np * s) = V2{R[0] * rka, R[1] * rka};
    }
    if (bad) atomicOr(src.status(it), ST_NONFINITE);
    __syncthreads();  // FF, the zeta buffer and the item ring are free for reuse
  }
}

}  // namespace cb
