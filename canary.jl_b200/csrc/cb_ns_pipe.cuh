// Pipelined LDG Navier–Stokes stage pass (sm_100a).
//
// The second of the two fused viscous passes per RK stage (the first writes
// the gradient gQ of the primitives): inviscid and viscous flux rows in one
// contraction, Rusanov minus the viscous face average, LSRK update — the
// arithmetic of ns_stage_group (nse3d.jl:475-955, nse2d.jl:396-778 with the
// inviscid volumerhs!/fluxrhs!), on the memory schedule of k_stage_pipe2 /
// k_stage_mma:
//
//   * the group's state and gradient slabs (read by the face phase for other
//     threads' nodes) are staged in shared memory by bulk copies issued one
//     group ahead; the slot is refilled right after the mid-group barrier,
//     while the contraction and update run;
//   * the metric, residual carry and face geometry are each read by the one
//     thread that needs them, from L2, where a block-wide L2 prefetch issued
//     at the top of the group's iteration has placed them;
//   * neighbour codes are loaded one group ahead; the neighbour traces
//     (state and gradient) are read in the face phase (FP64) or copied into
//     shared memory one group ahead by the face slot's thread (cp.async;
//     FP32).
//
// Groups, flux rows and the face buffer are those of k_stage_pipe2
// (Cfg<DIM, Nq>), so a batch's work list is the same for the grouped
// gradient pass (BCfg<DIM, Nq, 0> groups, the same element count) and this
// pass.  Item sources as for k_stage_pipe2, with gq(it): the instance's
// gradient buffer.
#pragma once

namespace cb {

template <int DIM, int Nq, typename T>
struct NsPipe {
  using C = Cfg<DIM, Nq>;
  using P1 = Pipe<DIM, Nq, T>;
  static constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG;
  static constexpr int RS = P1::RS, NR = P1::NR, MV = P1::MV;
  static constexpr size_t pad16(size_t b) { return (b + 15) & ~size_t(15); }
  static constexpr size_t QB = P1::QB;     // state bytes per element
  static constexpr size_t GQB = QB * DIM;  // gradient bytes per element
  // element slabs that are not 16-byte multiples (3-D even orders in FP64 and
  // FP32): copies rounded out to 16-byte boundaries as in k_stage_pipe2
  static constexpr bool RAG = QB % 16 != 0;
  static constexpr size_t SLK = RAG ? 32 : 0;
  static constexpr size_t QS = pad16(C::EPB * QB + SLK), GS = pad16(C::EPB * GQB + SLK);
  static constexpr size_t OFF_D = 16;  // one mbarrier, then the D rows
  static constexpr size_t OFF_S = OFF_D + pad16(sizeof(T) * Nq * RS);
  static constexpr size_t OFF_G = OFF_S + QS;
  static constexpr size_t OFF_F = OFF_G + GS;
  static constexpr size_t FDIR = P1::FDIR;
  static constexpr size_t OFF_FF = OFF_F + pad16(sizeof(T) * DIM * FDIR);
  // FP32: the neighbour traces of each face slot — state [NS] and gradient
  // [NS*DIM] — copied by the slot's thread one group ahead (cp.async),
  // [NS*(DIM+1)][FSLOTS]
  static constexpr bool ASYNC_TR = sizeof(T) == 4;
  static constexpr int TRV = NS * (DIM + 1);
  static constexpr size_t OFF_TR = OFF_FF + pad16(P1::FFB);
  static constexpr size_t TRB = ASYNC_TR ? sizeof(T) * TRV * (size_t)C::FSLOTS : 0;
  static constexpr size_t smem() { return OFF_TR + pad16(TRB); }  // sources append their ring here
  static constexpr size_t RING_MAX = 640;
  static constexpr int MINB = C::THREADS <= 256 ? 2 : 1;
  static constexpr bool OK = MINB * (smem() + RING_MAX + 1024) <= 228 * 1024 && smem() + RING_MAX <= SMEM_LIMIT;
};

// Block-wide L2 prefetch of `bytes` bytes from p (one request per 128-byte
// line; every address stays inside [p, p + bytes)).
__device__ __forceinline__ void prefetch_lines_l2(const void *p, size_t bytes) {
  const char *c = static_cast<const char *>(p);
  for (size_t off = (size_t)threadIdx.x * 128; off < bytes; off += (size_t)blockDim.x * 128)
    asm volatile("prefetch.global.L2 [%0];" ::"l"(c + off));
}

template <int DIM, int Nq, typename T, typename Src, int MINB = NsPipe<DIM, Nq, T>::MINB>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS, MINB)
k_ns_stage_pipe(Src src, PhysT<T> p, T rka) {
  using C = Cfg<DIM, Nq>;
  using PP = NsPipe<DIM, Nq, T>;
  static_assert(Src::AHEAD >= 1, "the source must publish the next group before the top of an iteration");
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, EPB = C::EPB, SP = C::SLOTS;
  constexpr int MJF = DIM * DIM, MJIF = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  constexpr int FS = EPB * Nfp, RS = PP::RS, NR = PP::NR;
  constexpr int64_t SE = (int64_t)NSG * Nfp * NF;  // face-geometry values per element
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
  T *DT = reinterpret_cast<T *>(smem_raw + PP::OFF_D);
  T *Sq0 = reinterpret_cast<T *>(smem_raw + PP::OFF_S);  // [EPB][NS][Np] state
  T *Sg0 = reinterpret_cast<T *>(smem_raw + PP::OFF_G);  // [EPB][DIM][NS][Np] gradient
  T *sF = reinterpret_cast<T *>(smem_raw + PP::OFF_F);
  T *FF = reinterpret_cast<T *>(smem_raw + PP::OFF_FF);
  T *TR = reinterpret_cast<T *>(smem_raw + PP::OFF_TR);  // [TRV][FSLOTS] (ASYNC_TR)
  const int tid = threadIdx.x;

  auto head_of = [](const T *g) -> uint32_t {
    return PP::RAG ? (uint32_t)(reinterpret_cast<uintptr_t>(g) & 15) : 0u;
  };
  // one slab copy of n bytes from g (see NsPipe::RAG): returns the bulk bytes
  // and issues the copy when `go`; `last`: the copy ends its array
  auto rag = [&](T *dst, const T *g, size_t n, bool last, bool go) -> uint32_t {
    const uint32_t head = head_of(g);
    const uint32_t end = head + (uint32_t)n;
    const uint32_t L = PP::RAG ? (last ? (end & ~15u) : ((end + 15u) & ~15u)) : end;
    if (go && L) bulk_g2s(dst, reinterpret_cast<const unsigned char *>(g) - head, L, bar);
    return L;
  };
  auto tail = [&](T *dst, const T *g, size_t n) {
    const uint32_t head = head_of(g);
    const uint32_t end = head + (uint32_t)n;
    const unsigned char *base = reinterpret_cast<const unsigned char *>(g) - head;
    for (uint32_t b = (end & ~15u) > head ? (end & ~15u) : head; b < end; b += sizeof(T))
      *reinterpret_cast<T *>(reinterpret_cast<unsigned char *>(dst) + b) = *reinterpret_cast<const T *>(base + b);
  };
  auto issue = [&](int it) {  // thread 0 only: the group's state and gradient slabs
    if (src.skip_copy(it)) return;
    const int64_t e0 = src.e0(it);
    const int nv = src.nv(it);
    const bool last = PP::RAG && src.last(it);
    const T *q = src.Qin(it) + e0 * Np * NS, *g = src.gq(it) + e0 * Np * NS * DIM;
    const uint32_t tx = rag(Sq0, q, nv * PP::QB, last, false) + rag(Sg0, g, nv * PP::GQB, last, false);
    if (last) {
      tail(Sq0, q, nv * PP::QB);
      tail(Sg0, g, nv * PP::GQB);
    }
    fence_proxy_async();
    mbar_expect_tx(bar, tx);
    rag(Sq0, q, nv * PP::QB, last, true);
    rag(Sg0, g, nv * PP::GQB, last, true);
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
  // this thread's face slots' neighbour traces of group `it` (state as
  // stored, without offsets, and gradient) into TR, one cp.async group
  auto issue_tr = [&](int it, const int32_t *codes) {
    const T *Qn = src.Qin(it), *Gn = src.gq(it);
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      if (fs < C::FSLOTS && codes[u] >= 0) {
        const int64_t e2 = codes[u] >> 3;
        const int vP = face_node<DIM, Nq>(codes[u] & 7, fs % Nfp);
#pragma unroll
        for (int s = 0; s < NS; ++s) cp_async<sizeof(T)>(TR + s * C::FSLOTS + fs, Qn + vP + Np * (s + NS * e2));
#pragma unroll
        for (int v = 0; v < NS * DIM; ++v)  // v = s + NS * c
          cp_async<sizeof(T)>(TR + (NS + v) * C::FSLOTS + fs, Gn + vP + Np * (v + (int64_t)NS * DIM * e2));
      }
    }
    cp_async_commit();
  };
  if constexpr (PP::ASYNC_TR)
    if (src.valid(0)) issue_tr(0, nbn);

  bool timed_out = false;
  const T *curD = nullptr;
  for (int it = 0; src.valid(it); ++it) {
    const int64_t e0 = src.e0(it);
    const int nv = src.nv(it);
    const bool more = src.valid(it + 1);
    if (tid == Src::PUBLISHER) src.prefetch();
    const T *__restrict__ Qin = src.Qin(it);
    const T *__restrict__ vgeo = src.vgeo(it);
    const T *__restrict__ gq = src.gq(it);
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

    // ---- neighbour codes (loaded one group ago); the traces themselves are
    // read in the face phase (holding them across phase A would spill)
    int32_t nbv[C::FPT];
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) nbv[u] = nbn[u];
    load_nbr(it + 1, nbn);

    // ---- wait for the state and gradient slabs
    if (!mbar_wait_bounded(bar, (uint32_t)(it & 1), src.wait_limit())) timed_out = true;
    const T *Sq = Sq0 + head_of(Qin + e0 * Np * NS) / sizeof(T);
    const T *Sg = Sg0 + head_of(gq + e0 * Np * NS * DIM) / sizeof(T);
    if (src.D(it) != curD) {  // read in phase B only; visible after the mid barrier
      curD = src.D(it);
      for (int t = tid; t < Nq * RS; t += C::THREADS) {
        const int i = t / RS, m = t % RS;
        DT[t] = m < Nq ? curD[m + Nq * i] : T(0);
      }
    }

    // ---- phase A: flux rows MJ ξ·F_inv - μ MJ ξ·F_visc (state, 1/MJ and the
    // buoyancy source kept in registers)
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
        T g[NS][DIM], vel[DIM], fv[NS][DIM];
#pragma unroll
        for (int s = 0; s < NS; ++s)
#pragma unroll
          for (int c = 0; c < DIM; ++c) g[s][c] = Sg[((el * DIM + c) * NS + s) * Np + n];
#pragma unroll
        for (int c = 0; c < DIM; ++c) vel[c] = q[c] / q[IR];
        visc_flux<DIM, T>(g, vel, p, fv);
        const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
#pragma unroll
        for (int r = 0; r < DIM; ++r) {
          const int row = DIM == 2 ? (r == 0 ? j : i) : (r == 0 ? j + Nq * k : (r == 1 ? i + Nq * k : i + Nq * j));
          const int pos = r == 0 ? i : (r == 1 ? j : k);
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            T a = met[r][0] * f[s][0] + met[r][1] * f[s][1];
            T b = met[r][0] * fv[s][0] + met[r][1] * fv[s][1];
            if (DIM == 3) {
              a = a + met[r][2] * f[s][2];
              b = b + met[r][2] * fv[s][2];
            }
            sF[r * PP::FDIR + ((size_t)(s * EPB + el) * NR + row) * RS + pos] = MJ * a - p.visc * (MJ * b);
          }
        }
        buoy[u] = MJ * q[IR] * p.grav;
      }
    }

    // ---- face terms sMJ (Rusanov - μ n·(F_visc⁻ + F_visc⁺)/2) into FF
    // (FP32: the neighbour traces were copied by this thread a group ago)
    if constexpr (PP::ASYNC_TR) cp_async_wait<0>();
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
      if (fs < C::FSLOTS && el < nv) {
        const int vM = face_node<DIM, Nq>(f, fn);
        const T *sgp = sg + NSG * (fn + Nfp * (f + NF * el));
        T nrm[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) nrm[c] = sgp[c];
        const T smj = sgp[DIM];
        T qM[NS], qq[NS], vM_[DIM], vP_[DIM];
#pragma unroll
        for (int s = 0; s < NS; ++s) qM[s] = Sq[(el * NS + s) * Np + vM] + qr[s];
        const T gM = p.grav != T(0) ? vg[vM + Np * (GC + (int64_t)NVG * el)] : T(0);
        const T riM = T(1) / qM[IR];
        const T PM = pressure_ri<DIM, T>(qM, riM, gM, p);
#pragma unroll
        for (int c = 0; c < DIM; ++c) vM_[c] = qM[c] / qM[IR];
        const int32_t nb = nbv[u];
        const int64_t e2 = nb >= 0 ? (int64_t)(nb >> 3) : e0 + el;
        const int vP = nb >= 0 ? face_node<DIM, Nq>(nb & 7, fn) : vM;
        T PPv, riP;
        if (nb >= 0) {
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            if constexpr (PP::ASYNC_TR)
              qq[s] = TR[s * C::FSLOTS + fs] + qr[s];
            else
              qq[s] = Qin[vP + Np * (s + NS * e2)] + qr[s];
          }
          const T gP = p.grav != T(0) ? vgeo[vP + Np * (GC + NVG * e2)] : T(0);
          riP = T(1) / qq[IR];
          PPv = pressure_ri<DIM, T>(qq, riP, gP, p);
#pragma unroll
          for (int c = 0; c < DIM; ++c) vP_[c] = qq[c] / qq[IR];
        } else {  // reflective wall (nse3d.jl:880-900): mirrored state and velocity
          wall_state<DIM, T>(qM, nrm, qq);
          riP = riM;
          PPv = PM;
          T un = nrm[0] * vM_[0] + nrm[1] * vM_[1];
          if (DIM == 3) un = un + nrm[2] * vM_[2];
#pragma unroll
          for (int c = 0; c < DIM; ++c) vP_[c] = vM_[c] - T(2) * un * nrm[c];
        }
        T out[NS];
        rusanov_n<DIM, T>(qM, riM, PM, qq, riP, PPv, nrm, p, out);
        // n · (F_visc⁻ + F_visc⁺), one side at a time (fewer live registers)
        T av[NS];
        {
          T g[NS][DIM], fv[NS][DIM];
#pragma unroll
          for (int s = 0; s < NS; ++s)
#pragma unroll
            for (int c = 0; c < DIM; ++c) g[s][c] = Sg[((el * DIM + c) * NS + s) * Np + vM];
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
              for (int c = 0; c < DIM; ++c) {
                if constexpr (PP::ASYNC_TR)
                  g[s][c] = TR[(NS + s + NS * c) * C::FSLOTS + fs];
                else
                  g[s][c] = gq[vP + Np * (s + NS * (c + (int64_t)DIM * e2))];
              }
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
        for (int s = 0; s < NS; ++s)
          FF[(f * NS + s) * FS + el * Nfp + fn] = smj * out[s] - p.visc * (smj * (T(0.5) * av[s]));
      }
    }
    // this thread has read its slots: copy the next group's traces into them
    if constexpr (PP::ASYNC_TR)
      if (more) issue_tr(it + 1, nbn);
    // Mid-group barrier; agrees on whether a wait gave up (then: store
    // nothing, flag the status, let the issued copy land, leave).
    if (__syncthreads_or(timed_out)) {
      if (tid == 0) {
        atomicOr(src.status(it), ST_TIMEOUT);
        mbar_wait_bounded(bar, (uint32_t)(it & 1), src.wait_limit());
      }
      if constexpr (PP::ASYNC_TR) cp_async_wait<0>();  // this thread's trace copies land before it leaves
      return;
    }
    // the slabs are no longer read: refill them while the update runs
    if (tid == 0 && more) issue(it + 1);
    if ((tid >> 5) == (Src::PUBLISHER >> 5)) src.publish(it);

    // ---- phase B: carry - source + contraction - face terms, update
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

// Gradient pass on the same schedule (k_ns_grad_pipe): the group's state
// slab by bulk copy one group ahead, metric and face geometry from L2
// (prefetched at the top of the group's iteration), the primitives' face
// averages for every gradient component computed once, then per component
// the flux rows MJ ξ_r,c prim, the contraction with Dᵀ (subtracted), the face
// terms in face order and ×MJI into gQ — ns_grad_group's arithmetic.
template <int DIM, int Nq, typename T>
struct NsGradPipe {
  using C = Cfg<DIM, Nq>;
  using P1 = Pipe<DIM, Nq, T>;
  using PS = NsPipe<DIM, Nq, T>;
  static constexpr int NS = Lay<DIM>::NS, ND = NS * DIM;
  static constexpr size_t pad16(size_t b) { return (b + 15) & ~size_t(15); }
  static constexpr size_t OFF_D = 16;
  static constexpr size_t OFF_S = OFF_D + pad16(sizeof(T) * Nq * P1::RS);
  static constexpr size_t OFF_F = OFF_S + PS::QS;
  static constexpr size_t OFF_FF = OFF_F + pad16(sizeof(T) * DIM * P1::FDIR);
  static constexpr size_t FFB = sizeof(T) * (size_t)C::NFACE * ND * C::EPB * C::Nfp;
  // FP32: the neighbour state traces of each face slot, [NS][FSLOTS], copied
  // by the slot's thread one group ahead (cp.async)
  static constexpr bool ASYNC_TR = sizeof(T) == 4;
  static constexpr size_t OFF_TR = OFF_FF + pad16(FFB);
  static constexpr size_t TRB = ASYNC_TR ? sizeof(T) * NS * (size_t)C::FSLOTS : 0;
  static constexpr size_t smem() { return OFF_TR + pad16(TRB); }  // sources append their ring here
  static constexpr int MINB = PS::MINB;
  static constexpr bool OK = MINB * (smem() + PS::RING_MAX + 1024) <= 228 * 1024 && smem() + PS::RING_MAX <= SMEM_LIMIT;
};

template <int DIM, int Nq, typename T, typename Src, int MINB = NsGradPipe<DIM, Nq, T>::MINB>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS, MINB)
k_ns_grad_pipe(Src src, PhysT<T> p, T) {
  using C = Cfg<DIM, Nq>;
  using PP = NsGradPipe<DIM, Nq, T>;
  using PS = NsPipe<DIM, Nq, T>;
  static_assert(Src::AHEAD >= 1, "the source must publish the next group before the top of an iteration");
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR, IE = Lay<DIM>::IE;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, EPB = C::EPB, SP = C::SLOTS, ND = NS * DIM;
  constexpr int MJF = DIM * DIM, MJIF = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  constexpr int FS = EPB * Nfp, RS = PS::RS, NR = PS::NR;
  constexpr int64_t SE = (int64_t)NSG * Nfp * NF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw);
  T *DT = reinterpret_cast<T *>(smem_raw + PP::OFF_D);
  T *Sq0 = reinterpret_cast<T *>(smem_raw + PP::OFF_S);  // [EPB][NS][Np] state
  T *sF = reinterpret_cast<T *>(smem_raw + PP::OFF_F);   // flux rows of one gradient component
  T *FF = reinterpret_cast<T *>(smem_raw + PP::OFF_FF);  // [NF][NS*DIM][FS] face terms
  T *TR = reinterpret_cast<T *>(smem_raw + PP::OFF_TR);  // [NS][FSLOTS] (ASYNC_TR)
  const int tid = threadIdx.x;

  auto head_of = [](const T *g) -> uint32_t {
    return PS::RAG ? (uint32_t)(reinterpret_cast<uintptr_t>(g) & 15) : 0u;
  };
  auto issue = [&](int it) {  // thread 0 only: the group's state slab (see NsPipe::RAG)
    if (src.skip_copy(it)) return;
    const int64_t e0 = src.e0(it);
    const int nv = src.nv(it);
    const bool last = PS::RAG && src.last(it);
    const T *q = src.Qin(it) + e0 * Np * NS;
    const uint32_t head = head_of(q);
    const uint32_t end = head + (uint32_t)(nv * PS::QB);
    const uint32_t L = PS::RAG ? (last ? (end & ~15u) : ((end + 15u) & ~15u)) : end;
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
  if constexpr (PS::MV > Nq)
    for (size_t t = tid; t < (size_t)DIM * PS::FDIR; t += C::THREADS)
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
  // this thread's face slots' neighbour state traces of group `it` (as
  // stored) into TR, one cp.async group (ASYNC_TR)
  auto issue_tr = [&](int it, const int32_t *codes) {
    const T *Qn = src.Qin(it);
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      if (fs < C::FSLOTS && codes[u] >= 0) {
        const int64_t e2 = codes[u] >> 3;
        const int vP = face_node<DIM, Nq>(codes[u] & 7, fs % Nfp);
#pragma unroll
        for (int s = 0; s < NS; ++s) cp_async<sizeof(T)>(TR + s * C::FSLOTS + fs, Qn + vP + Np * (s + NS * e2));
      }
    }
    cp_async_commit();
  };
  if constexpr (PP::ASYNC_TR)
    if (src.valid(0)) issue_tr(0, nbn);

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
    T *__restrict__ gq = const_cast<T *>(src.gq(it)) + e0 * Np * NS * DIM;
    for (int el = 0; el < nv; ++el) prefetch_lines_l2(vg + el * Np * NVG, sizeof(T) * Np * (MJIF + 1));
    prefetch_lines_l2(sg, sizeof(T) * nv * SE);
    T qr[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qr[s] = src.qref(it, s);
    int32_t nbv[C::FPT];
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) nbv[u] = nbn[u];
    load_nbr(it + 1, nbn);

    if (!mbar_wait_bounded(bar, (uint32_t)(it & 1), src.wait_limit())) timed_out = true;
    const T *Sq = Sq0 + head_of(Qin + e0 * Np * NS) / sizeof(T);
    if (src.D(it) != curD) {  // read after the first component's barrier
      curD = src.D(it);
      for (int t = tid; t < Nq * RS; t += C::THREADS) {
        const int i = t / RS, m = t % RS;
        DT[t] = m < Nq ? curD[m + Nq * i] : T(0);
      }
    }

    // ---- primitives of the thread's nodes, metric kept in registers
    T prim[C::NPT][NS], met[C::NPT][DIM][DIM], MJ[C::NPT], mji[C::NPT];
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = tid + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      if (slot < SP && el < nv) {
        T q[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) q[s] = Sq[(el * NS + s) * Np + n] + qr[s];
        const T *G = vg + (int64_t)el * Np * NVG;
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int c = 0; c < DIM; ++c) met[u][r][c] = G[(r + DIM * c) * Np + n];
        MJ[u] = G[MJF * Np + n];
        mji[u] = G[MJIF * Np + n];
        const T gc = p.grav != T(0) ? G[GC * Np + n] : T(0);
        primitives<DIM, T>(q, gc, p, prim[u]);
      }
    }
    // ---- face averages of the primitives (flux_grad!) for every component
    // (FP32: the neighbour traces were copied by this thread a group ago)
    if constexpr (PP::ASYNC_TR) cp_async_wait<0>();
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
      if (fs < C::FSLOTS && el < nv) {
        const int vM = face_node<DIM, Nq>(f, fn);
        const T *sgp = sg + NSG * (fn + Nfp * (f + NF * el));
        T nrm[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) nrm[c] = sgp[c];
        const T sMJ = sgp[DIM];
        T qM[NS], pM[NS], pP[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) qM[s] = Sq[(el * NS + s) * Np + vM] + qr[s];
        const T gM = p.grav != T(0) ? vg[vM + Np * (GC + (int64_t)NVG * el)] : T(0);
        primitives<DIM, T>(qM, gM, p, pM);
        const int32_t nb = nbv[u];
        if (nb >= 0) {
          const int64_t e2 = nb >> 3;
          const int vP = face_node<DIM, Nq>(nb & 7, fn);
          T qP[NS];
#pragma unroll
          for (int s = 0; s < NS; ++s) {
            if constexpr (PP::ASYNC_TR)
              qP[s] = TR[s * C::FSLOTS + fs] + qr[s];
            else
              qP[s] = Qin[vP + Np * (s + NS * e2)] + qr[s];
          }
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
    }
    // this thread has read its slots: copy the next group's traces into them
    if constexpr (PP::ASYNC_TR)
      if (more) issue_tr(it + 1, nbn);
    // ---- per gradient component: flux rows, contraction (subtracted), face
    // terms in face order, ×MJI into gQ (unrolled: the metric column is
    // chosen at compile time, not by indexing a register array)
#pragma unroll
    for (int c = 0; c < DIM; ++c) {
#pragma unroll
      for (int u = 0; u < C::NPT; ++u) {
        const int slot = tid + u * C::THREADS;
        const int el = slot / Np, n = slot % Np;
        if (slot < SP && el < nv) {
          const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
#pragma unroll
          for (int r = 0; r < DIM; ++r) {
            const int row = DIM == 2 ? (r == 0 ? j : i) : (r == 0 ? j + Nq * k : (r == 1 ? i + Nq * k : i + Nq * j));
            const int pos = r == 0 ? i : (r == 1 ? j : k);
#pragma unroll
            for (int s = 0; s < NS; ++s)
              sF[r * PS::FDIR + ((size_t)(s * EPB + el) * NR + row) * RS + pos] = MJ[u] * (met[u][r][c] * prim[u][s]);
          }
        }
      }
      if (c == 0) {
        // first barrier of the group: FF and the first rows are complete, the
        // state slab is no longer read; agree on a wait that gave up
        if (__syncthreads_or(timed_out)) {
          if (tid == 0) {
            atomicOr(src.status(it), ST_TIMEOUT);
            mbar_wait_bounded(bar, (uint32_t)(it & 1), src.wait_limit());
          }
          if constexpr (PP::ASYNC_TR) cp_async_wait<0>();  // this thread's trace copies land before it leaves
          return;
        }
        if (tid == 0 && more) issue(it + 1);
        if ((tid >> 5) == (Src::PUBLISHER >> 5)) src.publish(it);
      } else {
        __syncthreads();
      }
#pragma unroll
      for (int u = 0; u < C::NPT; ++u) {
        const int slot = tid + u * C::THREADS;
        const int el = slot / Np, n = slot % Np;
        if (slot < SP && el < nv) {
          T R[NS];
#pragma unroll
          for (int s = 0; s < NS; ++s) R[s] = T(0);
          contract_rows<DIM, Nq, T>(sF, DT, el, n, R);
#pragma unroll
          for (int s = 0; s < NS; ++s) R[s] = -R[s];
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
#pragma unroll
          for (int s = 0; s < NS; ++s) gq[n + Np * (s + NS * (c + (int64_t)DIM * el))] = R[s] * mji[u];
        }
      }
      __syncthreads();  // the rows are rewritten for the next component (the last: FF and the ring are free)
    }
  }
}

}  // namespace cb
