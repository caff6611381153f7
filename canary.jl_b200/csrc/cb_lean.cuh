// Lean pipelined LSRK stage (sm_100a): k_stage_pipe2's arithmetic on the
// memory schedule of the tensor-core stage, for any order.
//
// k_stage_pipe2 stages each group's state and metric (slab S) and its
// residual carry and face geometry (slabs T, double-buffered) in shared
// memory.  For the middle 3-D orders that plan is large (3-D N=3 / N=4 FP64:
// 146 / 124 KB), so one block of 256 threads runs per SM.  Here only the
// state is staged — the face phase reads it for other threads' nodes — by a
// bulk copy issued one group ahead; the metric, carry and face geometry are
// each read by the one thread that needs them, from L2, where a block-wide
// L2 prefetch at the top of the group's own iteration has placed them; FP32
// copies each face slot's neighbour traces one group ahead with cp.async.
// The plan shrinks to the state slab, the flux rows and the face buffer
// (3-D N=4 FP64: 58 KB), two blocks per SM.
//
// The arithmetic — volume fluxes, contraction rows, Rusanov face fluxes in
// face order, update — is k_stage_pipe2's term for term, so the two agree
// bit for bit (per-node geometry; gravity as there).
#pragma once

namespace cb {

template <int DIM, int Nq, typename T>
struct Lean {
  using C = Cfg<DIM, Nq>;
  using P1 = Pipe<DIM, Nq, T>;
  static constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG;
  static constexpr int RS = P1::RS, NR = P1::NR, MV = P1::MV;
  static constexpr size_t pad16(size_t b) { return (b + 15) & ~size_t(15); }
  static constexpr size_t QB = P1::QB;  // state bytes per element
  static constexpr bool RAG = QB % 16 != 0;
  static constexpr size_t SLK = RAG ? 32 : 0;
  static constexpr size_t QS = pad16(C::EPB * QB + SLK);
  static constexpr size_t OFF_D = 16;  // one mbarrier, then the D rows
  static constexpr size_t OFF_S = OFF_D + pad16(sizeof(T) * Nq * RS);
  static constexpr size_t OFF_F = OFF_S + QS;
  static constexpr size_t FDIR = P1::FDIR;
  static constexpr size_t OFF_FF = OFF_F + pad16(sizeof(T) * DIM * FDIR);
  static constexpr bool ASYNC_QP = sizeof(T) == 4;
  static constexpr size_t OFF_QP = OFF_FF + pad16(P1::FFB);
  static constexpr size_t QPB = ASYNC_QP ? sizeof(T) * NS * (size_t)C::FSLOTS : 0;
  static constexpr size_t smem() { return OFF_QP + pad16(QPB); }  // sources append their ring here
  static constexpr size_t RING_MAX = 640;
  static constexpr bool fits(int blocks) { return blocks * (smem() + RING_MAX + 1024) <= 228 * 1024; }
  // blocks of up to 256 threads: two (FP64) or three (FP32) per SM where
  // shared memory holds them
  static constexpr int MINB = C::THREADS > 256 ? 1 : sizeof(T) == 8 ? (fits(2) ? 2 : 1) : (fits(3) ? 3 : fits(2) ? 2 : 1);
  static constexpr bool OK = smem() + RING_MAX <= SMEM_LIMIT;
};

template <int DIM, int Nq, typename T, typename Src, int MINB = Lean<DIM, Nq, T>::MINB>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS, MINB)
k_stage_lean(Src src, PhysT<T> p, T rka) {
  using C = Cfg<DIM, Nq>;
  using PP = Lean<DIM, Nq, T>;
  static_assert(Src::AHEAD >= 1, "the source must publish the next group before the top of an iteration");
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, EPB = C::EPB, SP = C::SLOTS;
  constexpr int MJF = DIM * DIM, MJIF = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  constexpr int FS = EPB * Nfp, RS = PP::RS, NR = PP::NR;
  constexpr int64_t SE = (int64_t)NSG * Nfp * NF;  // face-geometry values per element
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
  T *DT = reinterpret_cast<T *>(smem_raw + PP::OFF_D);
  T *Sq0 = reinterpret_cast<T *>(smem_raw + PP::OFF_S);  // [EPB][NS][Np] state
  T *sF = reinterpret_cast<T *>(smem_raw + PP::OFF_F);
  T *FF = reinterpret_cast<T *>(smem_raw + PP::OFF_FF);
  T *QPs = reinterpret_cast<T *>(smem_raw + PP::OFF_QP);  // [NS][FSLOTS] (ASYNC_QP)
  const int tid = threadIdx.x;

  auto head_of = [](const T *g) -> uint32_t {
    return PP::RAG ? (uint32_t)(reinterpret_cast<uintptr_t>(g) & 15) : 0u;
  };
  auto issue = [&](int it) {  // thread 0 only: the group's state slab (see Lean::RAG)
    if (src.skip_copy(it)) return;
    const int64_t e0 = src.e0(it);
    const int nv = src.nv(it);
    const bool last = PP::RAG && src.last(it);
    const T *q = src.Qin(it) + e0 * Np * NS;
    const uint32_t head = head_of(q);
    const uint32_t end = head + (uint32_t)(nv * PP::QB);
    const uint32_t L = PP::RAG ? (last ? (end & ~15u) : ((end + 15u) & ~15u)) : end;
    const unsigned char *base = reinterpret_cast<const unsigned char *>(q) - head;
    if (last)  // the last (< 16) bytes of the array by plain loads
      for (uint32_t b = L > head ? L : head; b < end; b += sizeof(T))
        *reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(Sq0) + b) = *reinterpret_cast<const T *>(base + b);
    fence_proxy_async();
    mbar_expect_tx(bar, L);
    if (L) bulk_g2s(Sq0, base, L, bar);
  };

  src.begin(smem_raw + PP::smem());
  if (tid == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
  }
  if constexpr (PP::MV > Nq)
    for (size_t t = tid; t < (size_t)DIM * PP::FDIR; t += C::THREADS)
      if ((int)(t % RS) >= Nq) sF[t] = T(0);
  __syncthreads();
  if (tid == 0 && src.valid(0)) issue(0);

  int32_t nbn[C::FPT];
  auto load_nbr = [&](int it, int32_t *dst) {
    const bool ok = src.valid(it);
    const int64_t e0 = ok ? src.e0(it) : 0;
    const int nv = ok ? src.nv(it) : 0;
    const int32_t *nb = src.nbr(it);
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF;
      dst[u] = (fs < C::FSLOTS && el < nv) ? nb[f + NF * (e0 + el)] : NBR_WALL;
    }
  };
  load_nbr(0, nbn);
  // this thread's face slots' neighbour traces of group `it` (as stored) into
  // QPs, one cp.async group (ASYNC_QP)
  auto issue_qp = [&](int it, const int32_t *codes) {
    const T *Qn = src.Qin(it);
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      if (fs < C::FSLOTS && codes[u] >= 0) {
        const int64_t e2 = codes[u] >> 3;
        const int vP = face_node<DIM, Nq>(codes[u] & 7, fs % Nfp);
#pragma unroll
        for (int s = 0; s < NS; ++s) cp_async<sizeof(T)>(QPs + s * C::FSLOTS + fs, Qn + vP + Np * (s + NS * e2));
      }
    }
    cp_async_commit();
  };
  if constexpr (PP::ASYNC_QP)
    if (src.valid(0)) issue_qp(0, nbn);

  bool timed_out = false;
  const T *curD = nullptr;
  for (int it = 0; src.valid(it); ++it) {
    const int64_t e0 = src.e0(it);
    const int nv = src.nv(it);
    const bool more = src.valid(it + 1);
    if (tid == Src::PUBLISHER) src.prefetch();
    const T *__restrict__ Qin = src.Qin(it);
    const T *__restrict__ vgeo = src.vgeo(it);
    const T *__restrict__ vg = vgeo + e0 * Np * NVG;
    const T *__restrict__ sg = src.sgeo(it) + e0 * SE;
    T *__restrict__ rhs = src.rhs(it) + e0 * Np * NS;
    // this group's metric (+ MJ, MJI), carry and face geometry into L2
    for (int el = 0; el < nv; ++el) prefetch_lines_l2(vg + el * Np * NVG, sizeof(T) * Np * (MJIF + 1));
    prefetch_lines_l2(rhs, sizeof(T) * nv * Np * NS);
    prefetch_lines_l2(sg, sizeof(T) * nv * SE);
    T qr[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qr[s] = src.qref(it, s);

    // ---- neighbour traces: FP64 into registers now (codes loaded one
    // group ago), FP32 copied a group ago
    T qP[C::FPT][NS];
    int32_t nbv[C::FPT];
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) nbv[u] = nbn[u];
    load_nbr(it + 1, nbn);
    if constexpr (!PP::ASYNC_QP) {
#pragma unroll
      for (int u = 0; u < C::FPT; ++u) {
        const int fs = tid + u * C::THREADS;
        if (nbv[u] >= 0) {
          const int64_t e2 = nbv[u] >> 3;
          const int vP = face_node<DIM, Nq>(nbv[u] & 7, fs % Nfp);
#pragma unroll
          for (int s = 0; s < NS; ++s) qP[u][s] = Qin[vP + Np * (s + NS * e2)] + qr[s];
        }
      }
    }

    // ---- wait for the state slab
    if (!mbar_wait_bounded(bar, (uint32_t)(it & 1), src.wait_limit())) timed_out = true;
    const T *Sq = Sq0 + head_of(Qin + e0 * Np * NS) / sizeof(T);
    if (src.D(it) != curD) {  // read in phase B only; visible after the mid barrier
      curD = src.D(it);
      for (int t = tid; t < Nq * RS; t += C::THREADS) {
        const int i = t / RS, m = t % RS;
        DT[t] = m < Nq ? curD[m + Nq * i] : T(0);
      }
    }

    // ---- phase A: volume fluxes (state and 1/MJ kept in registers)
    T qd[C::NPT][NS], mji[C::NPT], buoy[C::NPT];
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = tid + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      buoy[u] = T(0);
      mji[u] = T(0);
      if (slot < SP && el < nv) {
        T q[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          qd[u][s] = Sq[(el * NS + s) * Np + n];
          q[s] = qd[u][s] + qr[s];
        }
        const T *G = vg + (int64_t)el * Np * NVG;
        const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
        T met[DIM][DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int c = 0; c < DIM; ++c) met[r][c] = G[(r + DIM * c) * Np + n];
        const T MJ = G[MJF * Np + n];
        mji[u] = G[MJIF * Np + n];
        const T gc = p.grav != T(0) ? G[GC * Np + n] : T(0);
        const T ri = T(1) / q[IR];
        const T P = pressure_ri<DIM, T>(q, ri, gc, p);
        T f[NS][DIM];
        euler_flux_ri<DIM, T>(q, ri, P, f);
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
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
    // ---- face fluxes into FF
    if constexpr (PP::ASYNC_QP) cp_async_wait<0>();
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
      if (fs < C::FSLOTS && el < nv) {
        const T *sgp = sg + NSG * (fn + Nfp * (f + NF * el));
        T nrm[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) nrm[c] = sgp[c];
        const T smj = sgp[DIM];
        const int vM = face_node<DIM, Nq>(f, fn);
        T qM[NS], qq[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) qM[s] = Sq[(el * NS + s) * Np + vM] + qr[s];
        const T gM = p.grav != T(0) ? vg[vM + Np * (GC + (int64_t)NVG * el)] : T(0);
        const T riM = T(1) / qM[IR];
        const T PM = pressure_ri<DIM, T>(qM, riM, gM, p);
        T PPv, riP;
        if (nbv[u] >= 0) {
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            if constexpr (PP::ASYNC_QP)
              qq[s] = QPs[s * C::FSLOTS + fs] + qr[s];
            else
              qq[s] = qP[u][s];
          }
          T gP = T(0);
          if (p.grav != T(0)) {
            const int64_t e2 = nbv[u] >> 3;
            gP = vgeo[face_node<DIM, Nq>(nbv[u] & 7, fn) + Np * (GC + NVG * e2)];
          }
          riP = T(1) / qq[IR];
          PPv = pressure_ri<DIM, T>(qq, riP, gP, p);
        } else {
          wall_state<DIM, T>(qM, nrm, qq);
          riP = riM;
          PPv = PM;
        }
        T out[NS];
        rusanov_n<DIM, T>(qM, riM, PM, qq, riP, PPv, nrm, p, out);
#pragma unroll
        for (int s = 0; s < NS; ++s) FF[(f * NS + s) * FS + el * Nfp + fn] = smj * out[s];
      }
    }
    // this thread has read its slots: copy the next group's traces into them
    if constexpr (PP::ASYNC_QP)
      if (more) issue_qp(it + 1, nbn);
    // Mid-group barrier; agrees on whether a wait gave up (then: store
    // nothing, flag the status, let the issued copies land, leave).
    if (__syncthreads_or(timed_out)) {
      if (tid == 0) {
        atomicOr(src.status(it), ST_TIMEOUT);
        mbar_wait_bounded(bar, (uint32_t)(it & 1), src.wait_limit());
      }
      if constexpr (PP::ASYNC_QP) cp_async_wait<0>();
      return;
    }
    // the state slab is no longer read: refill it while phase B runs
    if (tid == 0 && more) issue(it + 1);
    if ((tid >> 5) == (Src::PUBLISHER >> 5)) src.publish(it);

    // ---- phase B: carry - source + volume contraction - face terms, update
    T *__restrict__ Qout = src.Qout(it);
    const T rkbdt = src.rkbdt(it);
    bool bad = false;
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = tid + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      const int64_t e = e0 + el;
      if (slot < SP && el < nv) {
        T R[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) R[s] = rhs[n + Np * (s + NS * el)];
        R[DIM - 1] -= buoy[u];
        contract_rows<DIM, Nq, T>(sF, DT, el, n, R);
        gather_face_terms<DIM, Nq, EPB, T>(FF, el, n, R);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const T qn = qd[u][s] + rkbdt * R[s] * mji[u];
          bad |= !isfinite(qn);
          Qout[n + Np * (s + NS * e)] = qn;
          rhs[n + Np * (s + NS * el)] = R[s] * rka;
        }
      }
    }
    if (bad) atomicOr(src.status(it), ST_NONFINITE);
    __syncthreads();  // the flux rows, FF and the item ring are free for reuse
  }
}

}  // namespace cb
