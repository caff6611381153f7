// Persistent fused LSRK stage with early-released staging (sm_100a).
//
// Same work and results as k_stage_pipe, different memory schedule:
//   * slab S (state + metric of the current group) is read only in phase A;
//     each thread keeps its nodes' state and 1/MJ in registers, so S is
//     refilled with the next group by a bulk copy issued right after the
//     mid-iteration barrier and lands while phase B runs;
//   * slabs T[0], T[1] (residual carry + face geometry sgeo) are double
//     buffered and fetched one group ahead;
//   * neighbour traces are prefetched into registers, their neighbour codes
//     one group ahead.
// Used when every slab is a multiple of 16 bytes (bulk copies) and the
// shared-memory plan fits; otherwise k_stage_pipe / k_stage are used.
#pragma once

namespace cb {

template <int DIM, int Nq, typename T>
struct Pipe2 {
  using C = Cfg<DIM, Nq>;
  using P1 = Pipe<DIM, Nq, T>;
  static constexpr int NS = Lay<DIM>::NS, NSG = Lay<DIM>::NSG;
  static constexpr int NG = P1::NG, RS = P1::RS, NR = P1::NR, MV = P1::MV;
  static constexpr size_t QB = P1::QB, GB = P1::GB;
  static constexpr size_t SB = sizeof(T) * (size_t)NSG * C::Nfp * C::NFACE;  // sgeo per element
  static constexpr bool BULK = P1::BULK && SB % 16 == 0;
  static constexpr size_t pad16(size_t b) { return (b + 15) & ~size_t(15); }
  static constexpr size_t OFF_D = 32;  // 3 mbarriers before
  static constexpr size_t OFF_S = OFF_D + pad16(sizeof(T) * Nq * RS);
  static constexpr size_t SBYTES = C::EPB * (QB + GB);
  static constexpr size_t OFF_T = OFF_S + pad16(SBYTES);
  static constexpr size_t TBYTES = C::EPB * (QB + SB);
  static constexpr size_t OFF_F = OFF_T + 2 * pad16(TBYTES);
  static constexpr size_t FDIR = P1::FDIR;
  static constexpr size_t FLUX = sizeof(T) * DIM * FDIR;
  static constexpr size_t OFF_FF = OFF_F + pad16(FLUX);
  static constexpr size_t FFB = P1::FFB;
  static constexpr size_t smem() { return OFF_FF + FFB; }
  static constexpr bool OK = BULK && smem() <= SMEM_LIMIT;
};

template <int DIM, int Nq, typename T>
__global__ void __launch_bounds__(Cfg<DIM, Nq>::THREADS, 1)
k_stage_pipe2(const T *__restrict__ Qin, T *__restrict__ Qout, T *__restrict__ rhs,
              const T *__restrict__ vgeo, const T *__restrict__ sgeo,
              const int32_t *__restrict__ nbr, const T *__restrict__ D, int64_t nelem,
              PhysT<T> p, Offs<T, Lay<DIM>::NS> qref, T rka, T rkbdt, unsigned *status) {
  using C = Cfg<DIM, Nq>;
  using PP = Pipe2<DIM, Nq, T>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, EPB = C::EPB, SP = C::SLOTS;
  constexpr int NG = PP::NG, MJI = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  constexpr int FS = EPB * Nfp, RS = PP::RS, NR = PP::NR;
  constexpr size_t TSTRIDE = PP::pad16(PP::TBYTES) / sizeof(T);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *barS = reinterpret_cast<uint64_t *>(smem_raw);
  uint64_t *barT = barS + 1;  // barT[0], barT[1]
  T *DT = reinterpret_cast<T *>(smem_raw + PP::OFF_D);
  T *Sq = reinterpret_cast<T *>(smem_raw + PP::OFF_S);  // [EPB][NS][Np]
  T *Sg = Sq + EPB * Np * NS;                             // [EPB][NG][Np]
  T *T0 = reinterpret_cast<T *>(smem_raw + PP::OFF_T);   // [EPB][NS][Np] carry, then [EPB] sgeo
  T *sF = reinterpret_cast<T *>(smem_raw + PP::OFF_F);
  T *FF = reinterpret_cast<T *>(smem_raw + PP::OFF_FF);
  const int tid = threadIdx.x;
  const int64_t ngroups = (nelem + EPB - 1) / EPB;

  auto nvalid = [&](int64_t g) { return (int)((nelem - g * EPB) < EPB ? (nelem - g * EPB) : EPB); };
  auto issue_S = [&](int64_t g) {  // thread 0 only
    const int64_t e0 = g * EPB;
    const int nv = nvalid(g);
    fence_proxy_async();
    mbar_expect_tx(barS, (uint32_t)(nv * (PP::QB + PP::GB)));
    bulk_g2s(Sq, Qin + e0 * Np * NS, (uint32_t)(nv * PP::QB), barS);
    for (int el = 0; el < nv; ++el)
      bulk_g2s(Sg + el * Np * NG, vgeo + (e0 + el) * Np * NVG, (uint32_t)PP::GB, barS);
  };
  auto issue_T = [&](int64_t g, int b) {  // thread 0 only
    const int64_t e0 = g * EPB;
    const int nv = nvalid(g);
    T *dc = T0 + b * TSTRIDE, *ds = dc + EPB * Np * NS;
    fence_proxy_async();
    mbar_expect_tx(&barT[b], (uint32_t)(nv * (PP::QB + PP::SB)));
    bulk_g2s(dc, rhs + e0 * Np * NS, (uint32_t)(nv * PP::QB), &barT[b]);
    bulk_g2s(ds, sgeo + e0 * (PP::SB / sizeof(T)), (uint32_t)(nv * PP::SB), &barT[b]);
  };

  if (tid == 0) {
    mbar_init(barS, 1);
    mbar_init(&barT[0], 1);
    mbar_init(&barT[1], 1);
    fence_mbar_init();
  }
  for (int t = tid; t < Nq * RS; t += C::THREADS) {
    const int i = t / RS, m = t % RS;
    DT[t] = m < Nq ? D[m + Nq * i] : T(0);
  }
  if constexpr (PP::MV > Nq)
    for (size_t t = tid; t < (size_t)DIM * PP::FDIR; t += C::THREADS)
      if ((int)(t % RS) >= Nq) sF[t] = T(0);
  __syncthreads();
  if (tid == 0 && (int64_t)blockIdx.x < ngroups) {
    issue_S(blockIdx.x);
    issue_T(blockIdx.x, 0);
  }

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
    if (tid == 0 && gn < ngroups) issue_T(gn, b ^ 1);

    // ---- neighbour traces of this group (codes were loaded one group ago)
    T qP[C::FPT][NS];
    int32_t nbv[C::FPT];
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) nbv[u] = nbn[u];
    load_nbr(gn, nbn);
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int fn = fs % Nfp;
      if (nbv[u] >= 0) {
        const int64_t e2 = nbv[u] >> 3;
        const int vP = face_node<DIM, Nq>(nbv[u] & 7, fn);
#pragma unroll
        for (int s = 0; s < NS; ++s) qP[u][s] = Qin[vP + Np * (s + NS * e2)] + qref.v[s];
      }
    }

    // ---- wait for S (state + metric) and T[b] (carry + sgeo)
    if (!mbar_wait_bounded(barS, (uint32_t)(it & 1), WAIT_LIMIT)) timed_out = true;
    if (!mbar_wait_bounded(&barT[b], (uint32_t)((it >> 1) & 1), WAIT_LIMIT)) timed_out = true;
    const T *Tc = T0 + b * TSTRIDE, *Ts = Tc + EPB * Np * NS;

    // ---- phase A: volume fluxes (state and 1/MJ kept in registers) and face fluxes
    T qd[C::NPT][NS], mji[C::NPT], buoy[C::NPT];
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = tid + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      buoy[u] = T(0);
      mji[u] = T(0);
      if (slot < SP && e0 + el < nelem) {
        T q[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          qd[u][s] = Sq[(el * NS + s) * Np + n];
          q[s] = qd[u][s] + qref.v[s];
        }
        T met[DIM][DIM];
#pragma unroll
        for (int r = 0; r < DIM; ++r)
#pragma unroll
          for (int c = 0; c < DIM; ++c) met[r][c] = Sg[(el * NG + r + DIM * c) * Np + n];
        const T MJ = Sg[(el * NG + DIM * DIM) * Np + n];
        mji[u] = Sg[(el * NG + MJI) * Np + n];
        const T gc = p.grav != T(0) ? vgeo[n + Np * (GC + NVG * (e0 + el))] : T(0);
        const T ri = T(1) / q[IR];
        const T P = pressure_ri<DIM, T>(q, ri, gc, p);
        T f[NS][DIM];
        euler_flux_ri<DIM, T>(q, ri, P, f);
        const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
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
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
      if (fs < C::FSLOTS && e0 + el < nelem) {
        const T *sg = Ts + (size_t)NSG * (fn + Nfp * (f + NF * el));
        T nrm[DIM];
#pragma unroll
        for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
        const T smj = sg[DIM];
        const int vM = face_node<DIM, Nq>(f, fn);
        T qM[NS], qq[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) qM[s] = Sq[(el * NS + s) * Np + vM] + qref.v[s];
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
    __syncthreads();
    // S is no longer read: refill it with the next group while phase B runs
    if (tid == 0 && gn < ngroups) issue_S(gn);
    // ---- phase B: carry - source + volume contraction - face terms, update
#pragma unroll
    for (int u = 0; u < C::NPT; ++u) {
      const int slot = tid + u * C::THREADS;
      const int el = slot / Np, n = slot % Np;
      const int64_t e = e0 + el;
      if (slot < SP && e < nelem) {
        T R[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) R[s] = Tc[(el * NS + s) * Np + n];
        R[DIM - 1] -= buoy[u];
        contract_rows<DIM, Nq, T>(sF, DT, el, n, R);
        gather_face_terms<DIM, Nq, EPB, T>(FF, el, n, R);
#pragma unroll
        for (int s = 0; s < NS; ++s) {
          const T qn = qd[u][s] + rkbdt * R[s] * mji[u];
          bad |= !isfinite(qn);
          Qout[n + Np * (s + NS * e)] = qn;
          rhs[n + Np * (s + NS * e)] = R[s] * rka;
        }
      }
    }
    __syncthreads();  // T[b], the flux rows and FF are free for reuse
  }
  if (bad) atomicOr(status, ST_NONFINITE);
  if (timed_out) atomicOr(status, ST_TIMEOUT);
}

}  // namespace cb
