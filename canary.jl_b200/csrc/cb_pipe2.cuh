// Persistent fused LSRK stage with early-released staging (sm_100a).
//
// Same work and results as k_stage_pipe, different memory schedule:
//   * slab S (state + metric of the current group) is read only in phase A;
//     each thread keeps its nodes' state and 1/MJ in registers, so S is
//     refilled with the next group by a bulk copy issued right after the
//     mid-iteration barrier and lands while phase B runs;
//   * slabs T[0], T[1] (residual carry + face geometry sgeo) are double
//     buffered and fetched one group ahead (DEEP: two S and three T slabs,
//     copies two groups ahead);
//   * neighbour traces are prefetched into registers, their neighbour codes
//     one group ahead.
// Used when every slab is a multiple of 16 bytes (bulk copies) and the
// shared-memory plan fits; otherwise k_stage_pipe / k_stage are used.
//
// The kernel walks a sequence of element groups given by a source policy
// `Src`: MeshSrc is one mesh (group g of block b at iteration it is
// b + it * gridDim.x, all pointers kernel parameters); the batched driver
// supplies a source whose groups come from a work list over many instances,
// with per-group pointers published by one thread into a small shared-memory
// ring.  A source provides, for the block's iteration `it`:
//   valid(it), e0(it), nv(it) (elements in the group), Qin/Qout/rhs/vgeo/
//   sgeo/nbr/D(it), qref(it, s), rkbdt(it), status(it);
// begin(ring) (all threads, before the first barrier), prefetch() (thread
// PUBLISHER, at the top of each iteration) and publish(it) (the warp of
// thread PUBLISHER, during phase B of iteration it, for iteration it + 2).
#pragma once

namespace cb {

// AFF: affine-element geometry.  Instead of the per-node metric (vgeo) and
// per-face-node face geometry (sgeo), every element has one record of AW
// values — its metric terms, J, and per face the unit normal and sJ — and
// MJ, MJI and sMJ are formed from the LGL weights as computegeometry does
// (euler3d_set3c.jl:222-246).  The geometry array is then
// [w (Nq, padded to 16 bytes) | record of element 0 | record of element 1 ...]
// (built by cb_mesh_create for meshes whose elements are all affine).
//
// RAG: element slabs whose byte sizes are not multiples of 16 (3-D even
// orders, where Np is odd).  Each copy then starts at the 16-byte boundary
// at or below its source and lands `head` bytes into its shared-memory slab,
// and ends at the boundary at or above its end — the extra bytes belong to
// the neighbouring elements of the same array and are not used — except for
// a group that ends its array: there the last (< 16) bytes are loaded by the
// issuing thread with plain loads.  Slabs carry 32 bytes of slack.
//
// DEEP: copies run two groups ahead instead of one — two S slabs (S of group
// it + 2 is issued when group it releases its slab) and three T slabs (T of
// group it + 2 is issued at the top of iteration it) — so that a block keeps
// about twice the bytes in flight, for small groups whose copy latency a
// single group of work does not cover.
//
// X, Y: X times the elements per group of Cfg on X / Y times the threads
// (CfgX): each block barrier shared by more nodes, or Y nodes per thread.
template <int DIM, int Nq, typename T, bool AFF = false, bool DEEP = false, int X = 1, int Y = 1>
struct Pipe2 {
  using C = CfgX<DIM, Nq, X, Y>;
  using P1 = Pipe<DIM, Nq, T, X>;
  static constexpr int NS = Lay<DIM>::NS, NSG = Lay<DIM>::NSG, NVG = Lay<DIM>::NVG;
  static constexpr int NG = P1::NG, RS = P1::RS, NR = P1::NR, MV = P1::MV;
  static constexpr size_t QB = P1::QB, GB = P1::GB;
  static constexpr size_t pad16(size_t b) { return (b + 15) & ~size_t(15); }
  static constexpr int AW = DIM * DIM + 1 + 2 * DIM * (DIM + 1);  // affine record values
  static constexpr size_t AGB = pad16(sizeof(T) * AW);             // affine record bytes
  static constexpr int WOFF = (int)(pad16(sizeof(T) * Nq) / sizeof(T));  // records after the weights
  static constexpr size_t VB = sizeof(T) * (size_t)C::Np * NVG;  // vgeo bytes per element
  static constexpr size_t SB = AFF ? 0 : sizeof(T) * (size_t)NSG * C::Nfp * C::NFACE;  // sgeo per element
  static constexpr bool RAG = QB % 16 != 0 || VB % 16 != 0 || SB % 16 != 0;
  static constexpr size_t SLK = RAG ? 32 : 0;
  // the metric fields of an element are copied as one padded run (the pad
  // reads the start of the coordinate fields, which are never used)
  static constexpr size_t GBP = AFF ? AGB : pad16(GB) + (RAG ? 16 : 0);
  static constexpr size_t GCOPY = RAG ? GB : GBP;  // bytes asked for per element metric copy
  static constexpr int GS = (int)(GBP / sizeof(T));  // element stride of the staged metric / record
  static constexpr size_t QBS = pad16(C::EPB * QB + SLK);            // staged state / carry per slab
  static constexpr size_t SGS = AFF ? 0 : pad16(C::EPB * SB + SLK);  // staged sgeo per slab
  static constexpr bool BULK = AFF || pad16(GB) + 16 <= VB;
  static constexpr int LOOK = DEEP ? 2 : 1;  // groups ahead whose copies are issued
  static constexpr int NSB = DEEP ? 2 : 1, NTB = LOOK + 1;  // S and T slabs
  static constexpr size_t OFF_D = pad16(8 * (NSB + NTB));  // the mbarriers before
  // D rows (DTS elements), then (AFF) the LGL weights
  static constexpr size_t DTS = pad16(sizeof(T) * Nq * RS) / sizeof(T);
  static constexpr size_t OFF_S = OFF_D + sizeof(T) * DTS + (AFF ? pad16(sizeof(T) * Nq) : 0);
  static constexpr size_t SBYTES = QBS + C::EPB * GBP;
  static constexpr size_t OFF_T = OFF_S + NSB * pad16(SBYTES);
  static constexpr size_t TBYTES = QBS + SGS;
  static constexpr size_t OFF_F = OFF_T + NTB * pad16(TBYTES);
  static constexpr size_t FDIR = P1::FDIR;
  static constexpr size_t FLUX = sizeof(T) * DIM * FDIR;
  static constexpr size_t OFF_FF = OFF_F + pad16(FLUX);
  static constexpr size_t FFB = P1::FFB;
  // FP32: the neighbour state traces of each face slot, [NS][FSLOTS], copied
  // by the slot's thread one group ahead (cp.async) instead of loaded into
  // registers at the top of the group
  static constexpr bool ASYNC_QP = sizeof(T) == 4;  // (FP64 batches: no gain measured)
  static constexpr size_t OFF_QP = OFF_FF + pad16(FFB);
  static constexpr size_t QPB = ASYNC_QP ? sizeof(T) * NS * (size_t)C::FSLOTS : 0;
  static constexpr size_t smem() { return OFF_QP + pad16(QPB); }  // sources append their ring here
  static constexpr size_t RING_MAX = 640;
  static constexpr bool OK = BULK && smem() + RING_MAX <= SMEM_LIMIT;
  // whether `blocks` blocks fit in one SM's shared memory (228 KB, 1 KB of
  // it reserved per block)
  static constexpr bool fits(int blocks) { return blocks * (smem() + RING_MAX + 1024) <= 228 * 1024; }
  // Y > 1: as many blocks per SM as shared memory holds, up to 2048 threads
  // and at least 72 registers per thread
  static constexpr int minb_fit() {
    int b = 1;
    while (b < 8 && fits(b + 1) && (b + 1) * C::THREADS <= 2048 && (b + 1) * C::THREADS * 72 <= 65536) ++b;
    return b;
  }
  // blocks of up to 256 threads are sized for two (FP64) or four (FP32) per SM
  // (larger groups of X > 1: 512-thread FP32 blocks two per SM)
  static constexpr int MINB =
      Y > 1 ? minb_fit()
            : C::THREADS <= 256 ? (sizeof(T) == 4 ? 4 : 2) : (X > 1 && C::THREADS <= 512 && sizeof(T) == 4 ? 2 : 1);
};

// One mesh: groups of EPB consecutive elements, pointers and constants are
// kernel parameters.
template <typename T, int NS, int EPB>
struct MeshSrc {
  using Real = T;
  static constexpr size_t RING_BYTES = 0;
  static constexpr int PUBLISHER = 0;
  static constexpr int AHEAD = 1 << 20;  // groups ahead known at the top of an iteration
  const T *Qin_;
  T *Qout_, *rhs_;
  const T *vgeo_, *sgeo_;
  const int32_t *nbr_;
  const T *D_;
  int64_t nelem;
  Offs<T, NS> qref_;
  T rkbdt_;
  unsigned *status_;
  // Test hook (0 in every production launch): the state copy of each block's
  // first group is never issued and waits give up after PROBE_WAIT_LIMIT
  // polls, so that the bounded wait runs out on an mbarrier nobody arrives on.
  int probe_;
  // The launch covers elements ebeg_ .. nelem - 1 (a partitioned solve runs
  // the elements that read no ghost first, the others once ghosts arrived).
  int64_t ebeg_;
  const T *gq_ = nullptr;  // gradient buffer (the viscous stage pass only)
  __device__ bool skip_copy(int it) const { return probe_ != 0 && it == 0; }
  __device__ uint32_t wait_limit() const { return probe_ ? PROBE_WAIT_LIMIT : WAIT_LIMIT; }
  __device__ void begin(unsigned char *) {}
  __device__ void prefetch() {}
  __device__ void publish(int) {}
  __device__ int64_t g(int it) const { return (int64_t)blockIdx.x + (int64_t)it * gridDim.x; }
  __device__ bool valid(int it) const { return e0(it) < nelem; }
  // the group ends the launch's range (taken as the end of the arrays: the
  // last bytes are then loaded with plain loads, which is safe either way)
  __device__ bool last(int it) const { return e0(it) + EPB >= nelem; }
  __device__ int64_t e0(int it) const { return ebeg_ + g(it) * EPB; }
  __device__ int nv(int it) const {
    const int64_t r = nelem - e0(it);
    return r < EPB ? (int)r : EPB;
  }
  __device__ const T *Qin(int) const { return Qin_; }
  __device__ T *Qout(int) const { return Qout_; }
  __device__ T *rhs(int) const { return rhs_; }
  __device__ const T *vgeo(int) const { return vgeo_; }
  __device__ const T *sgeo(int) const { return sgeo_; }
  __device__ const int32_t *nbr(int) const { return nbr_; }
  __device__ const T *D(int) const { return D_; }
  __device__ const T *gq(int) const { return gq_; }
  __device__ T qref(int, int s) const { return qref_.v[s]; }
  __device__ T rkbdt(int) const { return rkbdt_; }
  __device__ unsigned *status(int) const { return status_; }
};

// MINB: resident blocks per SM that the register allocation is sized for;
// AFF: affine-element geometry (see Pipe2; gravity must be zero); DEEP:
// copies two groups ahead (see Pipe2); X, Y: X times the elements per group
// on X / Y times the threads.
template <int DIM, int Nq, typename T, typename Src, int MINB = Pipe2<DIM, Nq, T>::MINB, bool AFF = false,
          bool DEEP = false, int X = 1, int Y = 1>
__global__ void __launch_bounds__(CfgX<DIM, Nq, X, Y>::THREADS, MINB)
k_stage_pipe2(Src src, PhysT<T> p, T rka) {
  using C = CfgX<DIM, Nq, X, Y>;
  using PP = Pipe2<DIM, Nq, T, AFF, DEEP, X, Y>;
  static_assert(Src::AHEAD >= PP::LOOK, "the source must publish the groups whose copies are issued");
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, EPB = C::EPB, SP = C::SLOTS;
  constexpr int MJI = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  constexpr int FS = EPB * Nfp, RS = PP::RS, NR = PP::NR, GS = PP::GS;
  constexpr size_t TSTRIDE = PP::pad16(PP::TBYTES) / sizeof(T);
  constexpr size_t SSTRIDE = PP::pad16(PP::SBYTES) / sizeof(T);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  uint64_t *barS = reinterpret_cast<uint64_t *>(smem_raw);  // barS[NSB]
  uint64_t *barT = barS + PP::NSB;                         // barT[NTB]
  T *DT = reinterpret_cast<T *>(smem_raw + PP::OFF_D);
  T *S0 = reinterpret_cast<T *>(smem_raw + PP::OFF_S);  // per slab [EPB][NS][Np] state, then [EPB][GS]
  T *T0 = reinterpret_cast<T *>(smem_raw + PP::OFF_T);  // per slab [EPB][NS][Np] carry, then [EPB] sgeo
  T *sF = reinterpret_cast<T *>(smem_raw + PP::OFF_F);
  T *FF = reinterpret_cast<T *>(smem_raw + PP::OFF_FF);
  T *QPs = reinterpret_cast<T *>(smem_raw + PP::OFF_QP);  // [NS][FSLOTS] (ASYNC_QP)
  const int tid = threadIdx.x;

  // Byte offset of a source within its 16-byte line (0 unless RAG).
  auto head_of = [](const T *g) -> uint32_t {
    return PP::RAG ? (uint32_t)(reinterpret_cast<uintptr_t>(g) & 15) : 0u;
  };
  // One slab copy of n bytes from g into the 16-byte aligned dst (see RAG):
  // returns the bulk bytes and issues the copy when `go`; `last`: the copy
  // ends its array, so it stops at the boundary below the end and `tail`
  // loads the rest.
  auto rag = [&](T *dst, const T *g, size_t n, bool last, uint64_t *bar, bool go) -> uint32_t {
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
  auto issue_S = [&](int it, int b) {  // thread 0 only
    if (src.skip_copy(it)) return;
    const int64_t e0 = src.e0(it);
    const int nv = src.nv(it);
    const bool last = PP::RAG && src.last(it);
    const T *q = src.Qin(it) + e0 * Np * NS, *vg = src.vgeo(it);
    T *dq = S0 + b * SSTRIDE, *dg = dq + PP::QBS / sizeof(T);
    uint32_t tx = rag(dq, q, nv * PP::QB, last, &barS[b], false);
    if constexpr (AFF) {
      tx += (uint32_t)(nv * PP::GBP);
    } else {
      for (int el = 0; el < nv; ++el) tx += rag(dg + el * GS, vg + (e0 + el) * Np * NVG, PP::GCOPY, false, &barS[b], false);
    }
    if (last) tail(dq, q, nv * PP::QB);
    fence_proxy_async();
    mbar_expect_tx(&barS[b], tx);
    rag(dq, q, nv * PP::QB, last, &barS[b], true);
    if constexpr (AFF) {  // the group's records are contiguous
      bulk_g2s(dg, vg + PP::WOFF + e0 * GS, (uint32_t)(nv * PP::GBP), &barS[b]);
    } else {
      for (int el = 0; el < nv; ++el) rag(dg + el * GS, vg + (e0 + el) * Np * NVG, PP::GCOPY, false, &barS[b], true);
    }
  };
  auto issue_T = [&](int it, int b) {  // thread 0 only
    const int64_t e0 = src.e0(it);
    const int nv = src.nv(it);
    const bool last = PP::RAG && src.last(it);
    const T *c = src.rhs(it) + e0 * Np * NS, *sg = src.sgeo(it) + e0 * (int64_t)(PP::SB / sizeof(T));
    T *dc = T0 + b * TSTRIDE, *ds = dc + PP::QBS / sizeof(T);
    uint32_t tx = rag(dc, c, nv * PP::QB, last, &barT[b], false);
    if constexpr (!AFF) tx += rag(ds, sg, nv * PP::SB, last, &barT[b], false);
    if (last) {
      tail(dc, c, nv * PP::QB);
      if constexpr (!AFF) tail(ds, sg, nv * PP::SB);
    }
    fence_proxy_async();
    mbar_expect_tx(&barT[b], tx);
    rag(dc, c, nv * PP::QB, last, &barT[b], true);
    if constexpr (!AFF) rag(ds, sg, nv * PP::SB, last, &barT[b], true);
  };

  src.begin(smem_raw + PP::smem());
  if (tid == 0) {
    for (int b = 0; b < PP::NSB + PP::NTB; ++b) mbar_init(&barS[b], 1);
    fence_mbar_init();
  }
  if constexpr (PP::MV > Nq)
    for (size_t t = tid; t < (size_t)DIM * PP::FDIR; t += C::THREADS)
      if ((int)(t % RS) >= Nq) sF[t] = T(0);
  __syncthreads();
  if (tid == 0)
    for (int j = 0; j < PP::LOOK && src.valid(j); ++j) {
      issue_S(j, j);
      issue_T(j, j);
    }

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
  // this thread's face slots' neighbour traces of group `it` (stored values,
  // without the offsets) into QPs, as one cp.async group (ASYNC_QP)
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
  // AFF: the LGL weights head every mesh's record array (the same for every
  // mesh of this order)
  const T *WS = DT + PP::DTS;
  if constexpr (AFF) {
    if (tid < Nq && src.valid(0)) const_cast<T *>(WS)[tid] = src.vgeo(0)[tid];
    __syncthreads();
  }

  bool timed_out = false;
  const T *curD = nullptr;  // derivative matrix held in DT (rows padded like the flux rows)
  for (int it = 0; src.valid(it); ++it) {
    const int sb = it % PP::NSB, tb = it % PP::NTB;
    const int64_t e0 = src.e0(it);
    const int nv = src.nv(it);
    const bool more = src.valid(it + PP::LOOK);  // a group whose copies are issued in this iteration
    if (tid == 0 && more) issue_T(it + PP::LOOK, (it + PP::LOOK) % PP::NTB);
    if (tid == Src::PUBLISHER) src.prefetch();
    const T *__restrict__ Qin = src.Qin(it);
    T qr[NS];
#pragma unroll
    for (int s = 0; s < NS; ++s) qr[s] = src.qref(it, s);

    // ---- neighbour traces of this group (codes were loaded one group ago)
    T qP[C::FPT][NS];  // FP64: in registers; FP32: copied into QPs a group ago
    int32_t nbv[C::FPT];
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) nbv[u] = nbn[u];
    load_nbr(it + 1, nbn);
    if constexpr (!PP::ASYNC_QP) {
#pragma unroll
      for (int u = 0; u < C::FPT; ++u) {
        const int fs = tid + u * C::THREADS;
        const int fn = fs % Nfp;
        if (nbv[u] >= 0) {
          const int64_t e2 = nbv[u] >> 3;
          const int vP = face_node<DIM, Nq>(nbv[u] & 7, fn);
#pragma unroll
          for (int s = 0; s < NS; ++s) qP[u][s] = Qin[vP + Np * (s + NS * e2)] + qr[s];
        }
      }
    }

    // ---- wait for S[sb] (state + metric) and T[tb] (carry + sgeo)
    if (!mbar_wait_bounded(&barS[sb], (uint32_t)((it / PP::NSB) & 1), src.wait_limit())) timed_out = true;
    if (!mbar_wait_bounded(&barT[tb], (uint32_t)((it / PP::NTB) & 1), src.wait_limit())) timed_out = true;
    // staged slabs (RAG: each source's data starts `head` bytes into its slab)
    const T *Sq = S0 + sb * SSTRIDE + head_of(Qin + e0 * Np * NS) / sizeof(T);
    const T *Sg = S0 + sb * SSTRIDE + PP::QBS / sizeof(T);
    const T *Tc = T0 + tb * TSTRIDE + head_of(src.rhs(it) + e0 * Np * NS) / sizeof(T);
    const T *Ts = T0 + tb * TSTRIDE + PP::QBS / sizeof(T) +
                  (AFF ? 0 : head_of(src.sgeo(it) + e0 * (int64_t)(PP::SB / sizeof(T))) / sizeof(T));
    const T *__restrict__ vgeo = src.vgeo(it);
    if (src.D(it) != curD) {  // read in phase B only; visible after the mid barrier
      curD = src.D(it);
      for (int t = tid; t < Nq * RS; t += C::THREADS) {
        const int i = t / RS, m = t % RS;
        DT[t] = m < Nq ? curD[m + Nq * i] : T(0);
      }
    }

    // ---- phase A: volume fluxes (state and 1/MJ kept in registers) and face fluxes
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
        const T *G = Sg + el * GS + (AFF ? 0 : head_of(vgeo + (e0 + el) * Np * NVG) / sizeof(T));
        const int i = n % Nq, j = (n / Nq) % Nq, k = DIM == 3 ? n / (Nq * Nq) : 0;
        T met[DIM][DIM], MJ, gc = T(0);
        if constexpr (AFF) {
#pragma unroll
          for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int c = 0; c < DIM; ++c) met[r][c] = G[r + DIM * c];
          // M = kron(w, w[, w]) in computegeometry's multiplication order
          const T M = DIM == 2 ? WS[j] * WS[i] : (WS[k] * WS[j]) * WS[i];
          MJ = M * G[DIM * DIM];
          mji[u] = T(1) / MJ;
        } else {
#pragma unroll
          for (int r = 0; r < DIM; ++r)
#pragma unroll
            for (int c = 0; c < DIM; ++c) met[r][c] = G[(r + DIM * c) * Np + n];
          MJ = G[DIM * DIM * Np + n];
          mji[u] = G[MJI * Np + n];
          gc = p.grav != T(0) ? vgeo[n + Np * (GC + NVG * (e0 + el))] : T(0);
        }
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
    if constexpr (PP::ASYNC_QP) cp_async_wait<0>();  // this thread's traces, copied a group ago
#pragma unroll
    for (int u = 0; u < C::FPT; ++u) {
      const int fs = tid + u * C::THREADS;
      const int el = fs / (NF * Nfp), f = (fs / Nfp) % NF, fn = fs % Nfp;
      if (fs < C::FSLOTS && el < nv) {
        T nrm[DIM], smj;
        if constexpr (AFF) {
          const T *rec = Sg + el * GS + DIM * DIM + 1 + f * (DIM + 1);
#pragma unroll
          for (int c = 0; c < DIM; ++c) nrm[c] = rec[c];
          const T sM = DIM == 2 ? WS[fn] : WS[fn / Nq] * WS[fn % Nq];
          smj = sM * rec[DIM];
        } else {
          const T *sg = Ts + (size_t)NSG * (fn + Nfp * (f + NF * el));
#pragma unroll
          for (int c = 0; c < DIM; ++c) nrm[c] = sg[c];
          smj = sg[DIM];
        }
        const int vM = face_node<DIM, Nq>(f, fn);
        T qM[NS], qq[NS];
#pragma unroll
        for (int s = 0; s < NS; ++s) qM[s] = Sq[(el * NS + s) * Np + vM] + qr[s];
        const T gM = (!AFF && p.grav != T(0)) ? vgeo[vM + Np * (GC + NVG * (e0 + el))] : T(0);
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
          if (!AFF && p.grav != T(0)) {
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
    // (only for a valid group: an empty ring entry holds no instance)
    if constexpr (PP::ASYNC_QP)
      if (src.valid(it + 1)) issue_qp(it + 1, nbn);
    // The mid-iteration barrier also agrees on whether any thread's wait gave
    // up.  If one did, the block stores nothing for this group (its slabs may
    // be incomplete), flags the status word, lets the copies it has issued
    // land (bounded waits, so a copy that never completes cannot hold the
    // block) and leaves: later groups of this block are not computed either.
    if (__syncthreads_or(timed_out)) {
      if (tid == 0) {
        atomicOr(src.status(it), ST_TIMEOUT);
        // in flight: S of groups it .. it + LOOK - 1 (the copy of it + LOOK
        // is issued after this barrier), T of groups it .. it + LOOK; each
        // barrier holds at most one pending phase, the group's parity
        for (int g = it; g < it + PP::LOOK && src.valid(g); ++g)
          mbar_wait_bounded(&barS[g % PP::NSB], (uint32_t)((g / PP::NSB) & 1), src.wait_limit());
        for (int g = it; g <= it + PP::LOOK && src.valid(g); ++g)
          mbar_wait_bounded(&barT[g % PP::NTB], (uint32_t)((g / PP::NTB) & 1), src.wait_limit());
      }
      if constexpr (PP::ASYNC_QP) cp_async_wait<0>();  // this thread's trace copies land before it leaves
      return;
    }
    // S[sb] is no longer read: refill it while phase B runs
    if (tid == 0 && more) issue_S(it + PP::LOOK, sb);
    if ((tid >> 5) == (Src::PUBLISHER >> 5)) src.publish(it);
    // ---- phase B: carry - source + volume contraction - face terms, update
    T *__restrict__ Qout = src.Qout(it);
    T *__restrict__ rhs = src.rhs(it);
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
        for (int s = 0; s < NS; ++s) R[s] = Tc[(el * NS + s) * Np + n];
        R[DIM - 1] -= buoy[u];
        contract_rows<DIM, Nq, T, X>(sF, DT, el, n, R);
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
    if (bad) atomicOr(src.status(it), ST_NONFINITE);
    __syncthreads();  // T[tb], the flux rows, FF and the item ring are free for reuse
  }
}

}  // namespace cb
