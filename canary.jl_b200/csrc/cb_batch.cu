// Batched LSRK(5,4) over many independent DG instances of uneven order and
// size: cb_mesh_* and cb_batch_* in include/canary_b200.h.
//
// Every admitted instance advances in one graph launch per LSRK step.  Each
// group shape (dim, order N, variant) present has its own persistent kernel
// that walks a device-resident work list of element groups (slot, first
// element, generation) of that shape; the kernels of different shapes are
// independent chains of the graph and run concurrently, and a small kernel at
// the end of the step advances the per-slot step counters.  A group holds EPB
// consecutive elements of one instance, EPB chosen so that a group carries
// about 256 (variant 0) or 512 (variant 1) nodes; one kernel per shape keeps
// each shape's registers and shared memory at what that shape needs.
//
// Membership is dynamic, for continuous batching: admitting an instance
// launches one small kernel that writes its descriptor into the slot table and
// appends its items to its shape's work list (no host staging buffer);
// releasing it invalidates the slot, so stale items are skipped by their
// generation tag, and a list is compacted when dead items dominate.  The
// kernels read the lists through a device header, so admissions and releases
// re-build the graph only when the set of shapes present changes.  Each
// instance has its own dt and step target: its items are skipped once it has
// taken all of its steps.  The state ping-pongs between the caller's buffer
// and a batch-owned twin from a stream-ordered pool; the current buffer of an
// instance at stage s of its step k is (k + s) mod 2.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/canary_b200.h"
#include "cb_kernels.cuh"
#include "cb_ops.h"

namespace cb {
int solver_fail(int code, const char *fmt, ...);

constexpr int BT = 256;                // threads per block of the batched stage
constexpr int BMAXN2 = 8, BMAXN3 = 7;  // orders compiled into the batched stage

// Group shape for (dim, Nq, variant) at BT threads.
template <int DIM, int Nq, int V>
struct BCfg {
  static constexpr int Np = ipow(Nq, DIM), Nfp = ipow(Nq, DIM - 1), NFACE = 2 * DIM;
  static constexpr int BASE = Np >= BT ? 1 : BT / Np;
  static constexpr int EPB = BASE * (V + 1);
  static constexpr int SLOTS = EPB * Np;
  static constexpr int NPT = cdiv(SLOTS, BT);
  static constexpr int FSLOTS = EPB * NFACE * Nfp;
  static constexpr int FPT = cdiv(FSLOTS, BT);
  static constexpr bool OK = NPT <= 2;  // variants with more nodes per thread are not built
};

template <typename T>
struct BInst {
  T *Q[2];  // Q[0]: the caller's state, Q[1]: the batch-owned twin
  T *rhs;   // residual carry (caller's)
  const T *vgeo, *sgeo, *D;
  const int32_t *nbr;
  int64_t nelem;
  double dt;
  int64_t done, target;  // steps taken / steps to take
  int32_t N, var, gen, pad;
  T qref[5];
};
struct BWork {
  int32_t slot, e0, gen, pad;
};
// Shape id of (dim, N, variant); ids of orders that are not built stay unused.
constexpr int NSHAPE = 2 * 2 * (BMAXN2 + 1);
__host__ __device__ constexpr int shape_id(int dim, int N, int var) {
  return (dim - 2) * 2 * (BMAXN2 + 1) + 2 * N + var;
}
struct BHdr {
  BWork *work[NSHAPE];
  int32_t nwork[NSHAPE];
};

// One group of the fused stage (volume + face + LSRK update) of one instance.
template <int DIM, int Nq, int V, typename T>
__device__ __forceinline__ void stage_group(const BInst<T> &I, int64_t e0, int par, const PhysT<T> &p, T rka,
                                            T rkbdt, unsigned *ist, unsigned char *smem) {
  using C = BCfg<DIM, Nq, V>;
  constexpr int NS = Lay<DIM>::NS, NVG = Lay<DIM>::NVG, NSG = Lay<DIM>::NSG, IR = Lay<DIM>::IR;
  constexpr int Np = C::Np, Nfp = C::Nfp, NF = C::NFACE, SP = C::SLOTS, FS = C::EPB * Nfp;
  constexpr int MJI = DIM * DIM + 1, GC = DIM * DIM + 2 + DIM - 1;
  const T *__restrict__ Qin = I.Q[par];
  T *__restrict__ Qout = I.Q[par ^ 1];
  T *__restrict__ rhs = I.rhs;
  const T *__restrict__ vgeo = I.vgeo;
  const int64_t nelem = I.nelem;
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
    if (slot < SP && e < nelem) {
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
    if (slot < SP && e0 + el < nelem) contract<DIM, Nq, C::EPB, T>(sF, Ds, el, n, R[u]);
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
    if (e >= nelem) continue;
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
    if (slot < SP && e < nelem) {
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
  if (bad) atomicOr(ist, ST_NONFINITE);
  __syncthreads();  // shared memory is reused by the block's next item
}

// Persistent stage kernel of one group shape: the blocks stride over the
// shape's work list.
template <int DIM, int Nq, int V, typename T>
__global__ void __launch_bounds__(BT, 2)
k_stage_batch(const BInst<T> *__restrict__ insts, const BHdr *__restrict__ hdr, int stage, PhysT<T> p, T rka,
              double rkb, unsigned *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  constexpr int SID = shape_id(DIM, Nq - 1, V);
  const int nwork = hdr->nwork[SID];
  const BWork *__restrict__ work = hdr->work[SID];
  for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
    const BWork it = work[w];
    const BInst<T> &I = insts[it.slot];
    if (I.gen != it.gen || I.done >= I.target) continue;  // uniform over the block
    const int par = (int)((I.done + stage) & 1);
    stage_group<DIM, Nq, V, T>(I, it.e0, par, p, rka, T(rkb * I.dt), status + it.slot, smem_raw);
  }
}

// Advance the step counter of every slot that still has steps to take.
template <typename T>
__global__ void k_batch_step_end(BInst<T> *insts, int cap) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < cap && insts[i].done < insts[i].target) insts[i].done += 1;
}

// Write a slot descriptor (when `write`) and the work items [pos, pos+ngroups)
// of that slot into list `sid`; set the list length to pos+ngroups when
// `set_count`.
template <typename T>
__global__ void k_batch_admit(BInst<T> *insts, int slot, BInst<T> val, int write, unsigned *status, BHdr *hdr,
                              int sid, int pos, int ngroups, int epb, int set_count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    if (write) {
      insts[slot] = val;
      status[slot] = 0;
    }
    if (set_count) hdr->nwork[sid] = pos + ngroups;
  }
  BWork *work = hdr->work[sid];
  for (int g = t; g < ngroups; g += gridDim.x * blockDim.x) work[pos + g] = BWork{slot, g * epb, val.gen, 0};
}

__global__ void k_batch_hdr(BHdr *hdr, int sid, BWork *ptr, int nwork) {
  if (threadIdx.x == 0) {
    if (ptr) hdr->work[sid] = ptr;
    hdr->nwork[sid] = nwork;
  }
}

inline int b_base(int dim, int N) {
  const int Nq = N + 1, Np = dim == 2 ? Nq * Nq : Nq * Nq * Nq;
  return Np >= BT ? 1 : BT / Np;
}
inline bool b_order_ok(int dim, int N) { return N >= 1 && N <= (dim == 2 ? BMAXN2 : BMAXN3); }
inline bool b_var_ok(int dim, int N, int var) {
  if (!b_order_ok(dim, N) || (var != 0 && var != 1)) return false;
  if (var == 0) return true;
  const int Nq = N + 1, Np = dim == 2 ? Nq * Nq : Nq * Nq * Nq;
  return (2 * b_base(dim, N) * Np + BT - 1) / BT <= 2;
}
template <typename T>
size_t b_smem(int dim, int N, int var) {
  const int Nq = N + 1, Np = dim == 2 ? Nq * Nq : Nq * Nq * Nq, NS = dim == 2 ? 4 : 5;
  const size_t slots = (size_t)b_base(dim, N) * (var + 1) * Np;
  return sizeof(T) * (((Nq * Nq + 1) & ~1) + NS * slots + (size_t)dim * NS * slots);
}

// Host table of the stage kernels, indexed by shape id.
template <typename T>
struct BKernels {
  const void *fn[NSHAPE] = {};
  int grid[NSHAPE] = {};
  bool ready[NSHAPE] = {};
};
template <int DIM, int Nq, typename T>
void b_fill(BKernels<T> &k) {
  k.fn[shape_id(DIM, Nq - 1, 0)] = (const void *)k_stage_batch<DIM, Nq, 0, T>;
  if (BCfg<DIM, Nq, 1>::OK)
    k.fn[shape_id(DIM, Nq - 1, 1)] = (const void *)k_stage_batch<DIM, Nq, BCfg<DIM, Nq, 1>::OK ? 1 : 0, T>;
}
template <typename T>
BKernels<T> &b_kernels() {
  static BKernels<T> k = [] {
    BKernels<T> t;
    b_fill<2, 2, T>(t); b_fill<2, 3, T>(t); b_fill<2, 4, T>(t); b_fill<2, 5, T>(t);
    b_fill<2, 6, T>(t); b_fill<2, 7, T>(t); b_fill<2, 8, T>(t); b_fill<2, 9, T>(t);
    b_fill<3, 2, T>(t); b_fill<3, 3, T>(t); b_fill<3, 4, T>(t); b_fill<3, 5, T>(t);
    b_fill<3, 6, T>(t); b_fill<3, 7, T>(t); b_fill<3, 8, T>(t);
    return t;
  }();
  return k;
}
// Shared-memory limit and persistent grid (all SMs at the occupancy that the
// shape's registers and shared memory allow) of one shape, set up once per
// process on the current device.
template <typename T>
cudaError_t b_prepare(int dim, int N, int var, const void **fn, size_t *smem, int *grid) {
  BKernels<T> &k = b_kernels<T>();
  const int sid = shape_id(dim, N, var);
  *fn = k.fn[sid];
  *smem = b_smem<T>(dim, N, var);
  if (!k.ready[sid]) {
    cudaError_t e = cudaFuncSetAttribute(k.fn[sid], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn[sid], BT, *smem)) != cudaSuccess) return e;
    k.grid[sid] = num_sms() * std::max(per_sm, 1);
    k.ready[sid] = true;
  }
  *grid = k.grid[sid];
  return cudaSuccess;
}

}  // namespace cb

using namespace cb;

struct cb_mesh {
  int dim = 0, N = 0, prec = 64;
  int64_t nelem = 0;
  const void *vgeo = nullptr, *sgeo = nullptr, *D = nullptr;
  void *owned = nullptr;  // FP32 copies of vgeo | sgeo | D (precision 32)
  int32_t *nbr = nullptr;
};

namespace {

const double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                       -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double RKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                       1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                       2277821191437.0 / 14882151754819.0};

struct BSlot {
  bool used = false;
  int dim = 0, N = 0, var = 0, sid = 0, epb = 1, gen = 0;
  int64_t nelem = 0, start = 0, target = 0;
  int pos = 0, ngroups = 0;
  size_t qbytes = 0;
  void *Q = nullptr, *alt = nullptr;
};

// Work list of one shape.
struct BList {
  BWork *buf = nullptr;
  int cap = 0, tail = 0, live = 0;
};

}  // namespace

struct cb_batch {
  int prec = 64, cap = 0, device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  cudaMemPool_t pool = nullptr;  // stream-ordered pool of state twins and work lists
  cb_phys phys{};
  void *insts = nullptr;  // BInst<T>[cap]
  unsigned *status = nullptr;
  BHdr *hdr = nullptr;
  BList list[NSHAPE];
  int nslots[NSHAPE] = {};  // live instances per shape
  std::vector<BSlot> slots;
  int64_t steps = 0;
  int var[2][BMAXN2 + 1] = {};
  // one step as a graph; re-built when the set of shapes present changes
  cudaGraphExec_t exec = nullptr;
  uint64_t g_shapes = 0;
};

namespace {

void drop_graph(cb_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->g_shapes = 0;
}

template <typename T>
cudaError_t launch_admit(cb_batch *b, int slot, const BInst<T> &val, bool write, int sid, int pos, int ngroups,
                         int epb, bool set_count) {
  const int blocks = std::max(1, std::min(1024, (ngroups + 255) / 256));
  k_batch_admit<T><<<blocks, 256, 0, b->stream>>>((BInst<T> *)b->insts, slot, val, write ? 1 : 0, b->status,
                                                  b->hdr, sid, pos, ngroups, epb, set_count ? 1 : 0);
  return cudaGetLastError();
}

// Rewrite work list `sid` from its live slots, starting at position 0 (into
// `dst` when given, which then becomes the list).
template <typename T>
cudaError_t compact(cb_batch *b, int sid, BWork *dst) {
  if (dst) {
    k_batch_hdr<<<1, 32, 0, b->stream>>>(b->hdr, sid, dst, 0);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  int pos = 0;
  BInst<T> none{};
  for (int s = 0; s < b->cap; ++s) {
    BSlot &sl = b->slots[s];
    if (!sl.used || sl.sid != sid) continue;
    none.gen = sl.gen;
    cudaError_t e = launch_admit<T>(b, s, none, false, sid, pos, sl.ngroups, sl.epb, false);
    if (e != cudaSuccess) return e;
    sl.pos = pos;
    pos += sl.ngroups;
  }
  b->list[sid].tail = pos;
  k_batch_hdr<<<1, 32, 0, b->stream>>>(b->hdr, sid, nullptr, pos);
  return cudaGetLastError();
}

// Make room for `need` more items in list `sid`: compact in place when the
// live items then fill at most three quarters of it, else move to a larger
// list.
template <typename T>
cudaError_t ensure_work(cb_batch *b, int sid, int need) {
  BList &L = b->list[sid];
  if ((int64_t)L.tail + need <= L.cap) return cudaSuccess;
  if (((int64_t)L.live + need) * 4 <= (int64_t)L.cap * 3) return compact<T>(b, sid, nullptr);
  const int64_t ncap = std::max<int64_t>({(int64_t)L.cap * 2, ((int64_t)L.live + need) * 2, 1024});
  if (ncap > (1ll << 30)) return cudaErrorMemoryAllocation;
  BWork *nw = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync((void **)&nw, sizeof(BWork) * ncap, b->pool, b->stream);
  if (e != cudaSuccess) return e;
  if ((e = compact<T>(b, sid, nw)) != cudaSuccess) return e;
  if (L.buf) cudaFreeAsync(L.buf, b->stream);
  L.buf = nw;
  L.cap = (int)ncap;
  return cudaSuccess;
}

// One LSRK step as a graph: per shape present a chain of five persistent stage
// kernels (the chains are independent and run concurrently), then the step
// counter kernel after all chains.
template <typename T>
cudaError_t build_graph(cb_batch *b, uint64_t shapes) {
  const PhysT<T> p(Phys{b->phys.gamma, b->phys.R_gas, b->phys.c_p, b->phys.c_v, b->phys.gravity, b->phys.Pr,
                        b->phys.lambda, b->phys.visc});
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  std::vector<cudaGraphNode_t> lasts;
  const BInst<T> *insts = (const BInst<T> *)b->insts;
  const BHdr *hdr = b->hdr;
  unsigned *status = b->status;
  for (int sid = 0; sid < NSHAPE && e == cudaSuccess; ++sid) {
    if (!(shapes >> sid & 1)) continue;
    const int dim = 2 + sid / (2 * (BMAXN2 + 1)), N = (sid % (2 * (BMAXN2 + 1))) / 2, var = sid % 2;
    const void *fn;
    size_t smem;
    int grid;
    if ((e = b_prepare<T>(dim, N, var, &fn, &smem, &grid)) != cudaSuccess) break;
    cudaGraphNode_t prev = nullptr;
    for (int st = 0; st < 5 && e == cudaSuccess; ++st) {
      int stage = st;
      T rka = T(RKA[(st + 1) % 5]);
      double rkb = RKB[st];
      PhysT<T> pp = p;
      void *args[] = {(void *)&insts, (void *)&hdr, (void *)&stage, (void *)&pp, (void *)&rka, (void *)&rkb,
                      (void *)&status};
      cudaKernelNodeParams kp{};
      kp.func = (void *)fn;
      kp.gridDim = dim3(grid);
      kp.blockDim = dim3(BT);
      kp.sharedMemBytes = (unsigned)smem;
      kp.kernelParams = args;
      cudaGraphNode_t node;
      e = cudaGraphAddKernelNode(&node, g, prev ? &prev : nullptr, prev ? 1 : 0, &kp);
      prev = node;
    }
    if (e == cudaSuccess) lasts.push_back(prev);
  }
  if (e == cudaSuccess) {
    BInst<T> *mi = (BInst<T> *)b->insts;
    int cap = b->cap;
    void *args[] = {(void *)&mi, (void *)&cap};
    cudaKernelNodeParams kp{};
    kp.func = (void *)k_batch_step_end<T>;
    kp.gridDim = dim3((b->cap + 255) / 256);
    kp.blockDim = dim3(256);
    kp.kernelParams = args;
    cudaGraphNode_t node;
    e = cudaGraphAddKernelNode(&node, g, lasts.data(), lasts.size(), &kp);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, g, 0);
  cudaGraphDestroy(g);
  if (e == cudaSuccess) b->g_shapes = shapes;
  return e;
}

template <typename T>
int batch_run(cb_batch *b, int64_t nsteps) {
  int64_t need = 0;  // steps that some live instance still has to take
  uint64_t shapes = 0;
  for (const BSlot &s : b->slots)
    if (s.used && s.start + s.target > b->steps) {
      need = std::max<int64_t>(need, s.start + s.target - b->steps);
      shapes |= 1ull << s.sid;
    }
  const int64_t launch = std::min(need, nsteps);
  if (launch > 0) {
    if (!b->exec || shapes != b->g_shapes) {
      drop_graph(b);
      cudaError_t e = build_graph<T>(b, shapes);
      if (e != cudaSuccess) {
        drop_graph(b);
        return solver_fail(CB_ERR_CUDA, "cb_batch_run: step graph: %s", cudaGetErrorString(e));
      }
    }
    for (int64_t r = 0; r < launch; ++r) {
      cudaError_t e = cudaGraphLaunch(b->exec, b->stream);
      if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "cb_batch_run: graph launch: %s", cudaGetErrorString(e));
    }
  }
  b->steps += nsteps;
  return CB_OK;
}

template <typename T>
int batch_add(cb_batch *b, const cb_mesh *m, void *Q, void *rhs, double dt, int64_t nsteps, const double *qref,
              int *slot_out) {
  int slot = -1;
  for (int s = 0; s < b->cap; ++s)
    if (!b->slots[s].used) {
      slot = s;
      break;
    }
  if (slot < 0) return solver_fail(CB_ERR_NOMEM, "cb_batch_add: all %d slots are in use", b->cap);
  const int Nq = m->N + 1, ns = m->dim == 2 ? 4 : 5;
  const int64_t Np = m->dim == 2 ? (int64_t)Nq * Nq : (int64_t)Nq * Nq * Nq;
  BSlot &sl = b->slots[slot];
  const int var = b->var[m->dim - 2][m->N];
  const int sid = shape_id(m->dim, m->N, var);
  const int epb = b_base(m->dim, m->N) * (var + 1);
  const int64_t ngroups = (m->nelem + epb - 1) / epb;
  const size_t qbytes = sizeof(T) * Np * ns * m->nelem;
  void *alt = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&alt, qbytes, b->pool, b->stream);
  if (e != cudaSuccess) return solver_fail(CB_ERR_NOMEM, "cb_batch_add: state twin: %s", cudaGetErrorString(e));
  if ((e = ensure_work<T>(b, sid, (int)ngroups)) != cudaSuccess) {
    cudaFreeAsync(alt, b->stream);
    return solver_fail(CB_ERR_NOMEM, "cb_batch_add: work list: %s", cudaGetErrorString(e));
  }
  BInst<T> v{};
  v.Q[0] = (T *)Q;
  v.Q[1] = (T *)alt;
  v.rhs = (T *)rhs;
  v.vgeo = (const T *)m->vgeo;
  v.sgeo = (const T *)m->sgeo;
  v.D = (const T *)m->D;
  v.nbr = m->nbr;
  v.nelem = m->nelem;
  v.dt = dt;
  v.done = 0;
  v.target = nsteps;
  v.N = m->N;
  v.var = var;
  v.gen = sl.gen + 1;
  for (int k = 0; k < 5; ++k) v.qref[k] = qref ? T(qref[k]) : T(0);
  BList &L = b->list[sid];
  const int pos = L.tail;
  if ((e = launch_admit<T>(b, slot, v, true, sid, pos, (int)ngroups, epb, true)) != cudaSuccess) {
    cudaFreeAsync(alt, b->stream);
    return solver_fail(CB_ERR_CUDA, "cb_batch_add: %s", cudaGetErrorString(e));
  }
  sl.used = true;
  sl.dim = m->dim;
  sl.N = m->N;
  sl.var = var;
  sl.sid = sid;
  sl.epb = epb;
  sl.gen = v.gen;
  sl.nelem = m->nelem;
  sl.start = b->steps;
  sl.target = nsteps;
  sl.pos = pos;
  sl.ngroups = (int)ngroups;
  sl.qbytes = qbytes;
  sl.Q = Q;
  sl.alt = alt;
  L.tail = pos + (int)ngroups;
  L.live += (int)ngroups;
  *slot_out = slot;
  return CB_OK;
}

template <typename T>
int batch_release(cb_batch *b, int slot) {
  BSlot &sl = b->slots[slot];
  BList &L = b->list[sl.sid];
  const int64_t done = std::min(sl.target, b->steps - sl.start);
  cudaError_t e = cudaSuccess;
  if (done & 1) e = cudaMemcpyAsync(sl.Q, sl.alt, sl.qbytes, cudaMemcpyDeviceToDevice, b->stream);
  if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "cb_batch_release: copy: %s", cudaGetErrorString(e));
  BInst<T> none{};
  none.gen = sl.gen;  // target 0: the slot's items are skipped until the slot is reused
  L.live -= sl.ngroups;
  const int ntail = L.live == 0 ? 0 : sl.pos + sl.ngroups == L.tail ? sl.pos : L.tail;
  if ((e = launch_admit<T>(b, slot, none, true, sl.sid, ntail, 0, 1, true)) != cudaSuccess)
    return solver_fail(CB_ERR_CUDA, "cb_batch_release: %s", cudaGetErrorString(e));
  L.tail = ntail;
  cudaFreeAsync(sl.alt, b->stream);
  const int gen = sl.gen;
  sl = BSlot{};
  sl.gen = gen;
  return CB_OK;
}

}  // namespace

extern "C" {

int cb_mesh_create(cb_mesh **out, int dim, int N, int precision, int64_t nelem, const double *vgeo,
                   const double *sgeo, const int64_t *vmapM, const int64_t *vmapP, const int64_t *elemtobndy,
                   const double *D, cb_stream_t stream) {
  if (!out) return solver_fail(CB_ERR_ARG, "cb_mesh_create: null handle");
  *out = nullptr;
  if (dim != 2 && dim != 3) return solver_fail(CB_ERR_ARG, "dim must be 2 or 3 (got %d)", dim);
  if (precision != 32 && precision != 64) return solver_fail(CB_ERR_ARG, "precision must be 32 or 64");
  if (!b_order_ok(dim, N))
    return solver_fail(CB_ERR_UNSUPPORTED, "batched form: N must be 1..%d for dim %d (got %d)",
                       dim == 2 ? BMAXN2 : BMAXN3, dim, N);
  if (nelem <= 0 || nelem > (1ll << 28)) return solver_fail(CB_ERR_ARG, "cb_mesh_create: bad element count");
  if (!vgeo || !sgeo || !vmapM || !vmapP || !elemtobndy || !D)
    return solver_fail(CB_ERR_ARG, "cb_mesh_create: null array");
  cudaStream_t st = (cudaStream_t)stream;
  cb_mesh *m = new cb_mesh();
  m->dim = dim;
  m->N = N;
  m->prec = precision;
  m->nelem = nelem;
  const int Nq = N + 1, nvg = dim == 2 ? 8 : 14, nsg = dim == 2 ? 4 : 5;
  const int64_t Np = dim == 2 ? (int64_t)Nq * Nq : (int64_t)Nq * Nq * Nq, Nfp = dim == 2 ? Nq : (int64_t)Nq * Nq;
  unsigned *status = nullptr;
  cudaError_t e = cudaMalloc((void **)&m->nbr, sizeof(int32_t) * 2 * dim * nelem);
  if (e == cudaSuccess) e = cudaMalloc((void **)&status, sizeof(unsigned));
  if (e != cudaSuccess) {
    cb_mesh_destroy(m);
    cudaFree(status);
    return solver_fail(CB_ERR_NOMEM, "cb_mesh_create: %s", cudaGetErrorString(e));
  }
  cudaMemsetAsync(status, 0, sizeof(unsigned), st);
  const Ops<double> *o = dim == 2 ? get_ops<2, double>(N) : get_ops<3, double>(N);
  e = o->build_nbr(m->nbr, vmapM, vmapP, elemtobndy, nelem, status, st);
  if (e == cudaSuccess && precision == 32) {
    const int64_t nv = Np * nvg * nelem, nsv = nsg * Nfp * 2 * dim * nelem, nd = (int64_t)Nq * Nq;
    e = cudaMalloc(&m->owned, sizeof(float) * (nv + nsv + nd));
    if (e == cudaSuccess) {
      float *g = (float *)m->owned;
      if ((e = round_to_f32(g, vgeo, nv, st)) == cudaSuccess &&
          (e = round_to_f32(g + nv, sgeo, nsv, st)) == cudaSuccess)
        e = round_to_f32(g + nv + nsv, D, nd, st);
      m->vgeo = g;
      m->sgeo = g + nv;
      m->D = g + nv + nsv;
    }
  } else {
    m->vgeo = vgeo;
    m->sgeo = sgeo;
    m->D = D;
  }
  unsigned h = 0;
  if (e == cudaSuccess && (e = cudaMemcpyAsync(&h, status, sizeof h, cudaMemcpyDeviceToHost, st)) == cudaSuccess)
    e = cudaStreamSynchronize(st);
  cudaFree(status);
  if (e != cudaSuccess) {
    cb_mesh_destroy(m);
    return solver_fail(CB_ERR_CUDA, "cb_mesh_create: %s", cudaGetErrorString(e));
  }
  if (h & (ST_BC | ST_MESH)) {
    cb_mesh_destroy(m);
    return (h & ST_BC) ? solver_fail(CB_ERR_BC, "cb_mesh_create: invalid boundary condition code")
                       : solver_fail(CB_ERR_MESH, "cb_mesh_create: vmaps do not describe a conforming mesh");
  }
  *out = m;
  return CB_OK;
}

int cb_mesh_destroy(cb_mesh *m) {
  if (!m) return CB_OK;
  cudaFree(m->nbr);
  cudaFree(m->owned);
  delete m;
  return CB_OK;
}

int cb_batch_create(cb_batch **out, int precision, int max_instances, const cb_phys *phys, cb_stream_t stream) {
  if (!out || !phys) return solver_fail(CB_ERR_ARG, "cb_batch_create: null argument");
  *out = nullptr;
  if (precision != 32 && precision != 64) return solver_fail(CB_ERR_ARG, "precision must be 32 or 64");
  if (max_instances <= 0 || max_instances > (1 << 20))
    return solver_fail(CB_ERR_ARG, "cb_batch_create: max_instances must be 1..%d", 1 << 20);
  if (phys->visc != 0.0) return solver_fail(CB_ERR_UNSUPPORTED, "the batched form is inviscid (visc must be 0)");
  cb_batch *b = new cb_batch();
  b->prec = precision;
  b->cap = max_instances;
  b->phys = *phys;
  b->slots.resize(max_instances);
  cudaGetDevice(&b->device);
  cudaError_t e = cudaSuccess;
  auto bail = [&](const char *what) {
    cb_batch_destroy(b);
    return solver_fail(CB_ERR_CUDA, "cb_batch_create: %s: %s", what, cudaGetErrorString(e));
  };
  if (stream) b->stream = (cudaStream_t)stream;
  else {
    if ((e = cudaStreamCreate(&b->stream)) != cudaSuccess) return bail("stream");
    b->own_stream = true;
  }
  {
    // a private pool that keeps freed blocks, so that admissions and releases
    // under continuous batching do not return memory to the driver
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = b->device;
    if ((e = cudaMemPoolCreate(&b->pool, &props)) != cudaSuccess) return bail("memory pool");
    uint64_t keep = UINT64_MAX;
    if ((e = cudaMemPoolSetAttribute(b->pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess)
      return bail("memory pool");
  }
  const size_t ib = precision == 64 ? sizeof(BInst<double>) : sizeof(BInst<float>);
  if ((e = cudaMalloc(&b->insts, ib * max_instances)) != cudaSuccess ||
      (e = cudaMalloc((void **)&b->status, sizeof(unsigned) * max_instances)) != cudaSuccess ||
      (e = cudaMalloc((void **)&b->hdr, sizeof(BHdr))) != cudaSuccess)
    return bail("tables");
  if ((e = cudaMemsetAsync(b->insts, 0, ib * max_instances, b->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->status, 0, sizeof(unsigned) * max_instances, b->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->hdr, 0, sizeof(BHdr), b->stream)) != cudaSuccess)
    return bail("tables");
  *out = b;
  return CB_OK;
}

int cb_batch_set_variant(cb_batch *b, int dim, int N, int variant) {
  if (!b || (dim != 2 && dim != 3) || !b_order_ok(dim, N))
    return solver_fail(CB_ERR_ARG, "cb_batch_set_variant: bad arguments");
  if (!b_var_ok(dim, N, variant))
    return solver_fail(CB_ERR_UNSUPPORTED, "cb_batch_set_variant: variant %d is not built for dim %d N %d",
                       variant, dim, N);
  b->var[dim - 2][N] = variant;
  return CB_OK;
}

int cb_batch_add(cb_batch *b, const cb_mesh *m, void *Q, void *rhs, double dt, int64_t nsteps, const double *qref,
                 int *slot) {
  if (!b || !m || !Q || !rhs || !slot || nsteps < 0 || !std::isfinite(dt))
    return solver_fail(CB_ERR_ARG, "cb_batch_add: bad arguments");
  if (m->prec != b->prec) return solver_fail(CB_ERR_ARG, "cb_batch_add: mesh precision differs from the batch's");
  return b->prec == 64 ? batch_add<double>(b, m, Q, rhs, dt, nsteps, qref, slot)
                       : batch_add<float>(b, m, Q, rhs, dt, nsteps, qref, slot);
}

int cb_batch_run(cb_batch *b, int64_t nsteps) {
  if (!b || nsteps < 0) return solver_fail(CB_ERR_ARG, "cb_batch_run: bad arguments");
  return b->prec == 64 ? batch_run<double>(b, nsteps) : batch_run<float>(b, nsteps);
}

int cb_batch_info(const cb_batch *b, int slot, int64_t *done, int64_t *target) {
  if (!b || slot < 0 || slot >= b->cap || !b->slots[slot].used)
    return solver_fail(CB_ERR_ARG, "cb_batch_info: slot is not in use");
  const BSlot &s = b->slots[slot];
  if (done) *done = std::min(s.target, b->steps - s.start);
  if (target) *target = s.target;
  return CB_OK;
}

int cb_batch_release(cb_batch *b, int slot) {
  if (!b || slot < 0 || slot >= b->cap || !b->slots[slot].used)
    return solver_fail(CB_ERR_ARG, "cb_batch_release: slot is not in use");
  return b->prec == 64 ? batch_release<double>(b, slot) : batch_release<float>(b, slot);
}

int cb_batch_status(cb_batch *b, unsigned *out_host) {
  if (!b || !out_host) return solver_fail(CB_ERR_ARG, "cb_batch_status: null argument");
  cudaError_t e;
  if ((e = cudaMemcpyAsync(out_host, b->status, sizeof(unsigned) * b->cap, cudaMemcpyDeviceToHost, b->stream)) !=
          cudaSuccess ||
      (e = cudaStreamSynchronize(b->stream)) != cudaSuccess)
    return solver_fail(CB_ERR_CUDA, "cb_batch_status: %s", cudaGetErrorString(e));
  return CB_OK;
}

int cb_batch_destroy(cb_batch *b) {
  if (!b) return CB_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (BSlot &s : b->slots)
    if (s.used && s.alt) cudaFreeAsync(s.alt, b->stream);
  for (BList &L : b->list)
    if (L.buf) cudaFreeAsync(L.buf, b->stream);
  if (b->stream) cudaStreamSynchronize(b->stream);
  cudaFree(b->insts);
  cudaFree(b->status);
  cudaFree(b->hdr);
  if (b->pool) cudaMemPoolDestroy(b->pool);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return CB_OK;
}

}  // extern "C"
