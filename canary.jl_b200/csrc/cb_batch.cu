// Batched LSRK(5,4) over many independent DG instances of uneven order and
// size: cb_mesh_* and cb_batch_* in include/canary_b200.h.
//
// Every admitted instance advances in one graph launch per LSRK step.  Each
// group shape (dim, order N, stage variant) present has its own persistent
// kernel that walks a device-resident work list of that shape; the kernels of
// different shapes are independent chains of the graph and run concurrently,
// and a one-thread kernel at the end of the step advances the batch step
// counter.  A work item (16 bytes) names a group of consecutive elements of
// one instance; the instance's pointers, dt, offsets and step window live in a
// small per-slot descriptor table that stays in cache.  One kernel per shape
// keeps each shape's registers and shared memory at what that shape needs;
// the variants (pipelined bulk-copy staging at several occupancies, or
// grouped staging with ~256 / ~512 nodes per block) are chosen per (dim, N)
// by an autotuner and do not change the results.
//
// Membership is dynamic, for continuous batching: admitting an instance
// launches one small kernel that writes its descriptor and appends its items
// to its shape's list (no host staging buffer); releasing it invalidates its
// items in place, and a list is compacted when invalid items dominate.  The kernels read the lists
// through a device header, so admissions and releases re-build the graph only
// when the set of shapes present changes.  Each instance has its own dt and
// step count: its records are skipped once it has taken all of its steps.
// The state ping-pongs between the caller's buffer and a batch-owned twin
// from a stream-ordered pool; at batch step k the current buffer of an
// instance admitted at step k0 is (k - k0 + stage) mod 2.
#include <cuda_runtime.h>

#include <algorithm>
#include <bitset>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/canary_b200.h"
#include "cb_batch.cuh"
#include "cb_ops.h"

namespace cb {
int solver_fail(int code, const char *fmt, ...);

// One batch step done: advance the batch step counter.
__global__ void k_batch_step_end(BHdr *hdr) {
  if (blockIdx.x == 0 && threadIdx.x == 0) hdr->step += 1;
}

// Write the work items [pos, pos + ngroups) of the instance in `slot` into
// list `sid` (groups of epb elements of nelem); when `write` is set, also its
// descriptor and gradient buffer `gq` (viscous batches), and reset its status
// word; set the list length to `count` when count >= 0.
template <typename T>
__global__ void k_batch_admit(BHdr *hdr, int sid, int slot, BDesc<T> d, void *gq, int write, int pos, int ngroups,
                              int epb, int64_t nelem, int count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) {
    if (write) {
      static_cast<BDesc<T> *>(hdr->desc)[slot] = d;
      if (hdr->gq) static_cast<void **>(hdr->gq)[slot] = gq;
      *d.status = 0;
    }
    if (count >= 0) hdr->nwork[sid] = count;
  }
  BWork *work = hdr->work[sid];
  for (int g = t; g < ngroups; g += gridDim.x * blockDim.x) {
    const int64_t e0 = (int64_t)g * epb, rem = nelem - e0;
    work[pos + g] = BWork{slot, (int32_t)e0, rem < epb ? (int32_t)rem : epb, rem <= epb ? 3 : 1};
  }
}

// Invalidate the work items [pos, pos + n) of list `sid` and set its length
// to `count`.
__global__ void k_batch_invalidate(BHdr *hdr, int sid, int pos, int n, int count) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t == 0) hdr->nwork[sid] = count;
  BWork *work = hdr->work[sid];
  for (int g = t; g < n; g += gridDim.x * blockDim.x) work[pos + g].valid = 0;
}

// LGL weights of order N (the Newton iteration on (1 - x^2) P_N'(x) = 0 from
// the Chebyshev-Gauss-Lobatto points, G. von Winckel's lglnodes; w_i =
// 2 / (N (N + 1) P_N(x_i)^2)), as GaussQuadrature.jl's lglpoints gives them
// to round-off.
void lgl_weights(int N, double *w) {
  const double pi = 3.14159265358979323846;
  for (int i = 0; i <= N; ++i) {
    double x = std::cos(pi * i / N), PN = 1.0;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = x;
      for (int k = 2; k <= N; ++k) {
        const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      PN = p1;
      const double dx = (x * p1 - p0) / ((N + 1) * p1);
      x -= dx;
      if (std::fabs(dx) <= 2.2e-16) break;
    }
    double p0 = 1.0, p1 = x;  // P_N at the converged node
    for (int k = 2; k <= N; ++k) {
      const double p2 = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    PN = p1;
    w[N - i] = 2.0 / (N * (N + 1) * PN * PN);
  }
}

struct WTab {
  double w[16];
};
// relative tolerance of the affine test: a few hundred ulps of the metric
// terms that D x gives for an affine map (their round-off grows with N and
// with the coordinates' magnitude over the element size)
constexpr double AFFINE_TOL = 1e-10;

// Affine-element records of a mesh (the element layout of the pipelined
// stage's AFF geometry): per element its metric terms and J at node 0 and per
// face the unit normal and sJ at face node 0, rounded to T, padded to `gs`
// values.  An element whose metric, J = MJ / M, normals or sJ = sMJ / sM
// differ at any node from node 0's by more than `tol` (relative to the
// element's largest metric term, to J, to 1 for the normals, to sJ) sets
// *flag: the mesh is then not affine and the records are not used.  Block 0
// also writes the weights (rounded to T) to wout.
template <typename T>
__global__ void k_affine(int dim, int Nq, int64_t nelem, const double *vgeo, const double *sgeo, WTab wt, T *wout,
                         T *out, int gs, double tol, unsigned *flag) {
  if (blockIdx.x == 0 && threadIdx.x < Nq) wout[threadIdx.x] = T(wt.w[threadIdx.x]);
  const int Np = dim == 2 ? Nq * Nq : Nq * Nq * Nq, Nfp = dim == 2 ? Nq : Nq * Nq, nf = 2 * dim;
  const int nvg = dim == 2 ? 8 : 14, nsg = dim == 2 ? 4 : 5, nm = dim * dim;
  const double *w = wt.w;
  const double M0 = dim == 2 ? w[0] * w[0] : (w[0] * w[0]) * w[0];
  const double sM0 = dim == 2 ? w[0] : w[0] * w[0];
  for (int64_t e = blockIdx.x; e < nelem; e += gridDim.x) {
    const double *vg = vgeo + (int64_t)Np * nvg * e;
    const double *sg = sgeo + (int64_t)nsg * Nfp * nf * e;
    double scale = 0.0;
    for (int f = 0; f < nm; ++f) scale = fmax(scale, fabs(vg[(int64_t)Np * f]));
    const double J0 = vg[(int64_t)Np * nm] / M0;
    bool bad = !(scale > 0.0) || !(J0 > 0.0);
    for (int q = threadIdx.x; q < Np; q += blockDim.x) {
      const int i = q % Nq, j = (q / Nq) % Nq, k = dim == 3 ? q / (Nq * Nq) : 0;
      const double M = dim == 2 ? w[j] * w[i] : (w[k] * w[j]) * w[i];
      for (int f = 0; f < nm; ++f)
        bad |= !(fabs(vg[q + (int64_t)Np * f] - vg[(int64_t)Np * f]) <= tol * scale);
      bad |= !(fabs(vg[q + (int64_t)Np * nm] - M * J0) <= tol * M * J0);
    }
    for (int t = threadIdx.x; t < nf * Nfp; t += blockDim.x) {
      const int f = t / Nfp, fn = t % Nfp;
      const double *s = sg + (int64_t)nsg * t, *s0 = sg + (int64_t)nsg * Nfp * f;
      const double sM = dim == 2 ? w[fn] : w[fn / Nq] * w[fn % Nq];
      const double sJ0 = s0[dim] / sM0;
      for (int c = 0; c < dim; ++c) bad |= !(fabs(s[c] - s0[c]) <= tol);
      bad |= !(fabs(s[dim] - sM * sJ0) <= tol * sM * sJ0);
    }
    if (bad) atomicOr(flag, 1u);
    T *rec = out + (int64_t)gs * e;
    for (int t = threadIdx.x; t < gs; t += blockDim.x) {
      double v = 0.0;
      if (t < nm) v = vg[(int64_t)Np * t];
      else if (t == nm) v = J0;
      else if (t < nm + 1 + nf * (dim + 1)) {
        const int f = (t - nm - 1) / (dim + 1), c = (t - nm - 1) % (dim + 1);
        const double *s0 = sg + (int64_t)nsg * Nfp * f;
        v = c < dim ? s0[c] : s0[dim] / sM0;
      }
      rec[t] = T(v);
    }
  }
}

__global__ void k_batch_hdr(BHdr *hdr, int sid, BWork *ptr, int nwork) {
  if (threadIdx.x == 0) {
    if (ptr) hdr->work[sid] = ptr;
    hdr->nwork[sid] = nwork;
  }
}

template <typename T>
BKernels<T> &b_kernels() {
  static BKernels<T> k = [] {
    BKernels<T> t;
    b_fill_dim<2, T>(t);
    b_fill_dim<3, T>(t);
    return t;
  }();
  return k;
}
template <typename T>
bool b_var_ok(int dim, int N, int var) {
  return b_order_ok(dim, N) && var >= 0 && var < NVAR &&
         b_kernels<T>().fn[shape_id(dim, N, var)] != nullptr;
}
// viscous batches run the grouped two-pass LDG stage (variant 1 shapes)
constexpr int VAR_VISC = 1;
// default variant: the pipelined stage where it is built, else 512-node groups
// (the autotuner may choose another)
template <typename T>
int b_default_var(int dim, int N) {
  // 3-D defaults from the autotuner's B200 timings of one 6 M-node warped
  // instance (ms per step): FP64 N=3 lean 3.03 against 4.11 for variant 0,
  // N=4 3.46 against 4.46; N=7 the tensor-core stage (FP64 / FP32 2.15 /
  // 1.12 against 2.26 / 1.42).  The FP32 3-D orders keep variant 0: their
  // tuner winners (N=4 variant 4, N=5 variant 3, N=6 variant 8) were timed
  // on one large instance, while a served stream's 3-D instances are small.
  auto pick = [&](int v) { return b_var_ok<T>(dim, N, v) ? v : -1; };
  int v = -1;
  if (dim == 3 && N == 7 && PipeMT<T>::DEFAULT) v = pick(VAR_MMA);
  else if (dim == 3 && sizeof(T) == 8 && (N == 3 || N == 4)) v = pick(VAR_LEAN);
  if (v >= 0) return v;
  return b_var_ok<T>(dim, N, 0) ? 0 : b_var_ok<T>(dim, N, 2) ? 2 : 1;
}
// Shared-memory limit and persistent grid (all SMs at the occupancy that the
// shape's registers and shared memory allow) of one shape, set up once per
// process on the current device.
template <typename T>
cudaError_t b_prepare(int sid) {
  BKernels<T> &k = b_kernels<T>();
  if (!k.ready[sid]) {
    cudaError_t e = cudaFuncSetAttribute(k.fn[sid], cudaFuncAttributeMaxDynamicSharedMemorySize, (int)k.smem[sid]);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.fn[sid], k.threads[sid], k.smem[sid]);
    if (e != cudaSuccess) return e;
    k.grid[sid] = num_sms() * std::max(per_sm, 1);
    k.ready[sid] = true;
  }
  return cudaSuccess;
}
template <typename T>
cudaError_t b_prepare_visc(int sid) {
  BKernels<T> &k = b_kernels<T>();
  if (!k.vready[sid]) {
    for (int pass = 0; pass < 2; ++pass) {
      cudaError_t e = cudaFuncSetAttribute(k.vfn[pass][sid], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)k.vsmem[pass][sid]);
      if (e != cudaSuccess) return e;
      int per_sm = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.vfn[pass][sid], k.vthreads[pass][sid],
                                                        k.vsmem[pass][sid]);
      if (e != cudaSuccess) return e;
      k.vgrid[pass][sid] = num_sms() * std::max(per_sm, 1);
    }
    k.vready[sid] = true;
  }
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
  // affine-element geometry: [LGL weights | one record per element], in the
  // mesh's precision; used when every element is affine
  void *aff = nullptr;
  // set-up status (vmap validation, affine test): device words, their pinned
  // host copy and the event that ends the set-up; read at the first use
  unsigned *dstat = nullptr, *hstat = nullptr;
  cudaEvent_t ready = nullptr;
  mutable int state = -1;  // -1: not read yet, else CB_OK, CB_ERR_BC or CB_ERR_MESH
  mutable bool affine = false;
};

namespace {

const double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                       -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double RKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                       1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                       2277821191437.0 / 14882151754819.0};

struct BSlot {
  bool used = false;
  int dim = 0, N = 0, var = 0, sid = 0, epb = 1;
  int64_t nelem = 0, start = 0, target = 0;
  int pos = 0, ngroups = 0;
  size_t qbytes = 0;
  void *Q = nullptr, *alt = nullptr, *gq = nullptr;
  BDesc<double> d64{};  // template record of the instance (the batch's precision)
  BDesc<float> d32{};
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
  unsigned *status = nullptr;  // per slot
  void *desc = nullptr;        // BDesc<T> per slot
  void *gqtab = nullptr;       // viscous batches: gradient buffer per slot
  bool visc = false;
  BHdr *hdr = nullptr;
  BList list[NSHAPE];
  std::vector<BSlot> slots;
  int64_t steps = 0;  // batch steps launched (the device counter after them)
  int var[2][BMAXN2 + 1] = {};
  bool var_set[2][BMAXN2 + 1] = {};  // chosen by cb_batch_set_variant (else the default)
  int64_t last_used[NSHAPE] = {};  // batch step at which each shape last had live instances
  bool affine = true;  // affine-element stages allowed (and the default where they apply)
  bool concurrent = true;  // shapes as concurrent graph branches (else one chain)
  // one step as a graph; re-built when the set of shapes present changes
  cudaGraphExec_t exec = nullptr;
  std::bitset<NSHAPE> g_shapes;
};

namespace {

void drop_graph(cb_batch *b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  b->exec = nullptr;
  b->g_shapes.reset();
}

template <typename T>
BDesc<T> &record(BSlot &s);
template <>
BDesc<double> &record<double>(BSlot &s) { return s.d64; }
template <>
BDesc<float> &record<float>(BSlot &s) { return s.d32; }

template <typename T>
cudaError_t launch_admit(cb_batch *b, int slot, const BSlot &sl, int pos, int count, bool write) {
  const int blocks = std::max(1, std::min(1024, (sl.ngroups + 255) / 256));
  k_batch_admit<T><<<blocks, 256, 0, b->stream>>>(b->hdr, sl.sid, slot, record<T>(const_cast<BSlot &>(sl)), sl.gq,
                                                  write ? 1 : 0, pos, sl.ngroups, sl.epb, sl.nelem, count);
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
  for (int s = 0; s < b->cap; ++s) {
    BSlot &sl = b->slots[s];
    if (!sl.used || sl.sid != sid) continue;
    cudaError_t e = launch_admit<T>(b, s, sl, pos, -1, false);
    if (e != cudaSuccess) return e;
    sl.pos = pos;
    pos += sl.ngroups;
  }
  b->list[sid].tail = pos;
  k_batch_hdr<<<1, 32, 0, b->stream>>>(b->hdr, sid, nullptr, pos);
  return cudaGetLastError();
}

// Make room for `need` more records in list `sid`: compact in place when the
// live records then fill at most three quarters of it, else move to a larger
// list.
template <typename T>
cudaError_t ensure_work(cb_batch *b, int sid, int need) {
  BList &L = b->list[sid];
  if ((int64_t)L.tail + need <= L.cap) return cudaSuccess;
  if (((int64_t)L.live + need) * 4 <= (int64_t)L.cap * 3) return compact<T>(b, sid, nullptr);
  const int64_t ncap = std::max<int64_t>({(int64_t)L.cap * 2, ((int64_t)L.live + need) * 2, 256});
  if (ncap > (1ll << 28)) return cudaErrorMemoryAllocation;
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
cudaError_t build_graph(cb_batch *b, const std::bitset<NSHAPE> &shapes) {
  const PhysT<T> p(Phys{b->phys.gamma, b->phys.R_gas, b->phys.c_p, b->phys.c_v, b->phys.gravity, b->phys.Pr,
                        b->phys.lambda, b->phys.visc});
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaGraphCreate(&g, 0);
  if (e != cudaSuccess) return e;
  std::vector<cudaGraphNode_t> lasts;
  const BHdr *hdr = b->hdr;
  const BKernels<T> &K = b_kernels<T>();
  // the pipelined kernels of every (dim, N) take a BatchSrc whose layout does
  // not depend on its template arguments
  using SrcArgs = BatchSrc<T, 5, 1>;
  static_assert(sizeof(SrcArgs) == sizeof(BatchSrc<T, 4, 64>) && sizeof(SrcArgs) == sizeof(BatchSrc<T, 4, 64, 4>),
                "BatchSrc layout");
  // one kernel node: stage `st` (pass `pass` of a viscous batch) of shape sid
  auto add = [&](int sid, int st, int pass, cudaGraphNode_t *dep, cudaGraphNode_t *node) {
    int stage = st;
    T rka = T(RKA[(st + 1) % 5]);
    double rkb = RKB[st];
    PhysT<T> pp = p;
    SrcArgs src{hdr, sid, st, rkb, nullptr, nullptr, -1};
    void *gargs[] = {(void *)&hdr, (void *)&stage, (void *)&pp, (void *)&rka, (void *)&rkb};
    void *pargs[] = {(void *)&src, (void *)&pp, (void *)&rka};
    cudaKernelNodeParams kp{};
    if (b->visc) {  // per stage: gradient pass, then the stage pass
      kp.func = (void *)K.vfn[pass][sid];
      kp.gridDim = dim3(K.vgrid[pass][sid]);
      kp.blockDim = dim3(K.vthreads[pass][sid]);
      kp.sharedMemBytes = (unsigned)K.vsmem[pass][sid];
      kp.kernelParams = K.vpipelined[pass][sid] ? pargs : gargs;
    } else {
      kp.func = (void *)K.fn[sid];
      kp.gridDim = dim3(K.grid[sid]);
      kp.blockDim = dim3(K.threads[sid]);
      kp.sharedMemBytes = (unsigned)K.smem[sid];
      kp.kernelParams = K.pipelined[sid] ? pargs : gargs;
    }
    return cudaGraphAddKernelNode(node, g, dep, dep ? 1 : 0, &kp);
  };
  std::vector<int> sids;
  for (int sid = 0; sid < NSHAPE && e == cudaSuccess; ++sid)
    if (shapes.test(sid)) {
      sids.push_back(sid);
      e = b->visc ? b_prepare_visc<T>(sid) : b_prepare<T>(sid);
    }
  const int npass = b->visc ? 2 : 1;
  if (b->concurrent) {
    // each shape's stages as its own chain, the chains side by side
    for (int sid : sids) {
      cudaGraphNode_t prev = nullptr;
      for (int st = 0; st < 5 && e == cudaSuccess; ++st)
        for (int pass = 0; pass < npass && e == cudaSuccess; ++pass) {
          cudaGraphNode_t node;
          e = add(sid, st, pass, prev ? &prev : nullptr, &node);
          prev = node;
        }
      if (e == cudaSuccess && prev) lasts.push_back(prev);
    }
  } else {
    // one chain: each stage of every shape in turn, so that every kernel has
    // the whole GPU (persistent grids sized for all SMs do not share them)
    cudaGraphNode_t prev = nullptr;
    for (int st = 0; st < 5 && e == cudaSuccess; ++st)
      for (int sid : sids)
        for (int pass = 0; pass < npass && e == cudaSuccess; ++pass) {
          cudaGraphNode_t node;
          e = add(sid, st, pass, prev ? &prev : nullptr, &node);
          prev = node;
        }
    if (e == cudaSuccess && prev) lasts.push_back(prev);
  }
  if (e == cudaSuccess) {
    BHdr *mh = b->hdr;
    void *args[] = {(void *)&mh};
    cudaKernelNodeParams kp{};
    kp.func = (void *)k_batch_step_end;
    kp.gridDim = dim3(1);
    kp.blockDim = dim3(32);
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
  std::bitset<NSHAPE> shapes;
  for (const BSlot &s : b->slots)
    if (s.used && s.start + s.target > b->steps) {
      need = std::max<int64_t>(need, s.start + s.target - b->steps);
      shapes.set(s.sid);
    }
  const int64_t launch = std::min(need, nsteps);
  if (launch <= 0) return CB_OK;
  // Under continuous batching shapes come and go; re-building the graph
  // costs milliseconds, an empty shape a few empty launches per step.  So a
  // graph keeps the shapes used in the last KEEP_STEPS steps: it is re-built
  // when a new shape appears or when a shape has been idle that long.
  constexpr int64_t KEEP_STEPS = 256;
  for (int sid = 0; sid < NSHAPE; ++sid)
    if (shapes.test(sid)) b->last_used[sid] = b->steps;
  std::bitset<NSHAPE> keep = shapes;
  for (int sid = 0; sid < NSHAPE; ++sid)
    if (b->g_shapes.test(sid) && b->steps - b->last_used[sid] < KEEP_STEPS) keep.set(sid);
  if (!b->exec || (shapes & ~b->g_shapes).any() || keep != b->g_shapes) {
    shapes = keep;
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
    ++b->steps;
  }
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
  // the stage variant of the instance: an affine variant runs where the mesh
  // allows it (else the shape's default per-node variant); a default
  // pipelined variant is replaced by VAR_AFFINE where the mesh allows it; an
  // explicitly chosen per-node variant runs as chosen
  const BKernels<T> &K = b_kernels<T>();
  const bool eligible = !b->visc && b->affine && m->affine && b->phys.gravity == 0.0;
  int var = b->visc ? VAR_VISC : b->var[m->dim - 2][m->N];
  if (var_affine(var) && !eligible) var = b_default_var<T>(m->dim, m->N);
  else if (!var_affine(var) && eligible && !b->var_set[m->dim - 2][m->N] && K.pipelined[shape_id(m->dim, m->N, var)] &&
           K.fn[shape_id(m->dim, m->N, VAR_AFFINE)])
    var = VAR_AFFINE;
  const int sid = shape_id(m->dim, m->N, var);
  const int epb = K.epb[sid];
  const int64_t ngroups = (m->nelem + epb - 1) / epb;
  const size_t qbytes = sizeof(T) * Np * ns * m->nelem;
  void *alt = nullptr, *gq = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&alt, qbytes, b->pool, b->stream);
  if (e != cudaSuccess) return solver_fail(CB_ERR_NOMEM, "cb_batch_add: state twin: %s", cudaGetErrorString(e));
  if (b->visc && (e = cudaMallocFromPoolAsync(&gq, qbytes * m->dim, b->pool, b->stream)) != cudaSuccess) {
    cudaFreeAsync(alt, b->stream);
    return solver_fail(CB_ERR_NOMEM, "cb_batch_add: gradient buffer: %s", cudaGetErrorString(e));
  }
  if ((e = ensure_work<T>(b, sid, (int)ngroups)) != cudaSuccess) {
    cudaFreeAsync(alt, b->stream);
    if (gq) cudaFreeAsync(gq, b->stream);
    return solver_fail(CB_ERR_NOMEM, "cb_batch_add: work list: %s", cudaGetErrorString(e));
  }
  BSlot sl;
  sl.used = true;
  sl.dim = m->dim;
  sl.N = m->N;
  sl.var = var;
  sl.sid = sid;
  sl.epb = epb;
  sl.nelem = m->nelem;
  sl.start = b->steps;
  sl.target = nsteps;
  sl.ngroups = (int)ngroups;
  sl.qbytes = qbytes;
  sl.Q = Q;
  sl.alt = alt;
  sl.gq = gq;
  BDesc<T> &d = record<T>(sl);
  d.Q[0] = (T *)Q;
  d.Q[1] = (T *)alt;
  d.rhs = (T *)rhs;
  d.vgeo = (const T *)(var_affine(var) ? m->aff : m->vgeo);
  d.sgeo = (const T *)m->sgeo;
  d.D = (const T *)m->D;
  d.nbr = m->nbr;
  d.status = b->status + slot;
  d.gq = (T *)gq;
  d.start = b->steps;
  d.target = nsteps;
  d.dt = dt;
  for (int k = 0; k < 5; ++k) d.qref[k] = qref ? T(qref[k]) : T(0);
  BList &L = b->list[sid];
  sl.pos = L.tail;
  if ((e = launch_admit<T>(b, slot, sl, sl.pos, sl.pos + sl.ngroups, true)) != cudaSuccess) {
    cudaFreeAsync(alt, b->stream);
    if (gq) cudaFreeAsync(gq, b->stream);
    return solver_fail(CB_ERR_CUDA, "cb_batch_add: %s", cudaGetErrorString(e));
  }
  L.tail = sl.pos + sl.ngroups;
  L.live += sl.ngroups;
  b->slots[slot] = sl;
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
  L.live -= sl.ngroups;
  const int ntail = L.live == 0 ? 0 : sl.pos + sl.ngroups == L.tail ? sl.pos : L.tail;
  const int blocks = std::max(1, std::min(1024, (sl.ngroups + 255) / 256));
  k_batch_invalidate<<<blocks, 256, 0, b->stream>>>(b->hdr, sl.sid, sl.pos, sl.ngroups, ntail);
  if ((e = cudaGetLastError()) != cudaSuccess)
    return solver_fail(CB_ERR_CUDA, "cb_batch_release: %s", cudaGetErrorString(e));
  L.tail = ntail;
  cudaFreeAsync(sl.alt, b->stream);
  if (sl.gq) cudaFreeAsync(sl.gq, b->stream);
  sl = BSlot{};
  return CB_OK;
}

}  // namespace

namespace {
// Wait for the mesh's set-up (once) and report its validation.
int mesh_check(const cb_mesh *m) {
  if (m->state < 0) {
    const cudaError_t e = cudaEventSynchronize(m->ready);
    if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "mesh set-up: %s", cudaGetErrorString(e));
    const unsigned h = m->hstat[0];
    m->affine = m->hstat[1] == 0;
    m->state = (h & ST_BC) ? CB_ERR_BC : (h & ST_MESH) ? CB_ERR_MESH : CB_OK;
  }
  if (m->state == CB_ERR_BC) return solver_fail(CB_ERR_BC, "cb_mesh: invalid boundary condition code");
  if (m->state == CB_ERR_MESH) return solver_fail(CB_ERR_MESH, "cb_mesh: vmaps do not describe a conforming mesh");
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
  if (((uintptr_t)vgeo | (uintptr_t)sgeo) & 15)
    return solver_fail(CB_ERR_ARG, "cb_mesh_create: vgeo and sgeo must be 16-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  cb_mesh *m = new cb_mesh();
  m->dim = dim;
  m->N = N;
  m->prec = precision;
  m->nelem = nelem;
  const int Nq = N + 1, nvg = dim == 2 ? 8 : 14, nsg = dim == 2 ? 4 : 5;
  const int64_t Np = dim == 2 ? (int64_t)Nq * Nq : (int64_t)Nq * Nq * Nq, Nfp = dim == 2 ? Nq : (int64_t)Nq * Nq;
  cudaError_t e = cudaMalloc((void **)&m->nbr, sizeof(int32_t) * 2 * dim * nelem);
  if (e == cudaSuccess) e = cudaMalloc((void **)&m->dstat, 2 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaMallocHost((void **)&m->hstat, 2 * sizeof(unsigned));
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&m->ready, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    cb_mesh_destroy(m);
    return solver_fail(CB_ERR_NOMEM, "cb_mesh_create: %s", cudaGetErrorString(e));
  }
  unsigned *status = m->dstat;
  cudaMemsetAsync(status, 0, 2 * sizeof(unsigned), st);
  const Ops<double> *o = dim == 2 ? get_ops<2, double>(N) : get_ops<3, double>(N);
  e = o->build_nbr(m->nbr, vmapM, vmapP, elemtobndy, nelem, status, st);
  if (e == cudaSuccess && precision == 32) {
    const int64_t nv = Np * nvg * nelem, nsv = nsg * Nfp * 2 * dim * nelem, nd = (int64_t)Nq * Nq;
    // each array starts on a 16-byte boundary (bulk copies of element slabs)
    const int64_t nvp = (nv + 3) & ~int64_t(3), nsp = (nsv + 3) & ~int64_t(3);
    e = cudaMalloc(&m->owned, sizeof(float) * (nvp + nsp + nd));
    if (e == cudaSuccess) {
      float *g = (float *)m->owned;
      if ((e = round_to_f32(g, vgeo, nv, st)) == cudaSuccess &&
          (e = round_to_f32(g + nvp, sgeo, nsv, st)) == cudaSuccess)
        e = round_to_f32(g + nvp + nsp, D, nd, st);
      m->vgeo = g;
      m->sgeo = g + nvp;
      m->D = g + nvp + nsp;
    }
  } else {
    m->vgeo = vgeo;
    m->sgeo = sgeo;
    m->D = D;
  }
  // affine-element records (status bit 31 set: some element is not affine)
  const size_t wsz = precision == 64 ? 8 : 4;
  const int aw = dim * dim + 1 + 2 * dim * (dim + 1);
  const int64_t gs = (int64_t)((wsz * aw + 15) & ~size_t(15)) / wsz, woff = (int64_t)((wsz * Nq + 15) & ~size_t(15)) / wsz;
  double wl[16] = {};
  lgl_weights(N, wl);
  if (e == cudaSuccess) e = cudaMalloc(&m->aff, wsz * (woff + gs * nelem));
  if (e == cudaSuccess) {
    WTab wt{};
    for (int i = 0; i < Nq; ++i) wt.w[i] = wl[i];
    const int blocks = (int)std::min<int64_t>(nelem, 4096);
    if (precision == 64)
      k_affine<double><<<blocks, 128, 0, st>>>(dim, Nq, nelem, vgeo, sgeo, wt, (double *)m->aff,
                                               (double *)m->aff + woff, (int)gs, AFFINE_TOL, status + 1);
    else
      k_affine<float><<<blocks, 128, 0, st>>>(dim, Nq, nelem, vgeo, sgeo, wt, (float *)m->aff,
                                              (float *)m->aff + woff, (int)gs, AFFINE_TOL, status + 1);
    e = cudaGetLastError();
  }
  // the status words are read at the first use of the mesh (no wait here)
  if (e == cudaSuccess) e = cudaMemcpyAsync(m->hstat, status, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaEventRecord(m->ready, st);
  if (e != cudaSuccess) {
    cb_mesh_destroy(m);
    return solver_fail(CB_ERR_CUDA, "cb_mesh_create: %s", cudaGetErrorString(e));
  }
  *out = m;
  return CB_OK;
}

int cb_mesh_affine(const cb_mesh *m, int *affine) {
  if (!m || !affine) return solver_fail(CB_ERR_ARG, "cb_mesh_affine: null argument");
  const int rc = mesh_check(m);
  if (rc) return rc;
  *affine = m->affine ? 1 : 0;
  return CB_OK;
}

int cb_mesh_destroy(cb_mesh *m) {
  if (!m) return CB_OK;
  if (m->ready) cudaEventSynchronize(m->ready);
  cudaFree(m->nbr);
  cudaFree(m->owned);
  cudaFree(m->aff);
  cudaFree(m->dstat);
  if (m->hstat) cudaFreeHost(m->hstat);
  if (m->ready) cudaEventDestroy(m->ready);
  delete m;
  return CB_OK;
}

int cb_batch_create(cb_batch **out, int precision, int max_instances, const cb_phys *phys, cb_stream_t stream) {
  if (!out || !phys) return solver_fail(CB_ERR_ARG, "cb_batch_create: null argument");
  *out = nullptr;
  if (precision != 32 && precision != 64) return solver_fail(CB_ERR_ARG, "precision must be 32 or 64");
  if (max_instances <= 0 || max_instances > (1 << 20))
    return solver_fail(CB_ERR_ARG, "cb_batch_create: max_instances must be 1..%d", 1 << 20);
  if (!(phys->visc >= 0.0)) return solver_fail(CB_ERR_ARG, "cb_batch_create: visc must be >= 0");
  cb_batch *b = new cb_batch();
  b->prec = precision;
  b->cap = max_instances;
  b->phys = *phys;
  b->visc = phys->visc > 0.0;
  // FP64 batches default to the per-node geometry: the affine-element stage
  // uses each element's first-node metric for all of its nodes, which
  // differs from the per-node arrays in the last bits, and over hundreds of
  // steps that moves an FP64 result ~1e-11 away from the oracle (measured
  // on the vortex ensemble: 1.4e-11 after 500 steps, 3e-15 per-node); in
  // FP32 the difference is far below the form's own rounding
  b->affine = precision == 32;
  b->slots.resize(max_instances);
  for (int dim = 2; dim <= 3; ++dim)
    for (int N = 1; b_order_ok(dim, N); ++N)
      b->var[dim - 2][N] = b->visc ? VAR_VISC
                                   : precision == 64 ? b_default_var<double>(dim, N) : b_default_var<float>(dim, N);
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
  const size_t db = precision == 64 ? sizeof(BDesc<double>) : sizeof(BDesc<float>);
  if ((e = cudaMalloc((void **)&b->status, sizeof(unsigned) * max_instances)) != cudaSuccess ||
      (e = cudaMalloc((void **)&b->hdr, sizeof(BHdr))) != cudaSuccess ||
      (e = cudaMalloc(&b->desc, db * max_instances)) != cudaSuccess ||
      (b->visc && (e = cudaMalloc(&b->gqtab, sizeof(void *) * max_instances)) != cudaSuccess))
    return bail("tables");
  BHdr h0{};
  h0.desc = b->desc;
  h0.gq = b->gqtab;
  if ((e = cudaMemsetAsync(b->status, 0, sizeof(unsigned) * max_instances, b->stream)) != cudaSuccess ||
      (e = cudaMemsetAsync(b->desc, 0, db * max_instances, b->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(b->hdr, &h0, sizeof h0, cudaMemcpyHostToDevice, b->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(b->stream)) != cudaSuccess)
    return bail("tables");
  *out = b;
  return CB_OK;
}

int cb_batch_set_variant(cb_batch *b, int dim, int N, int variant) {
  if (!b || (dim != 2 && dim != 3) || !b_order_ok(dim, N))
    return solver_fail(CB_ERR_ARG, "cb_batch_set_variant: bad arguments");
  if (b->visc && variant != VAR_VISC)
    return solver_fail(CB_ERR_UNSUPPORTED, "cb_batch_set_variant: viscous batches run variant %d only", VAR_VISC);
  if (!(b->prec == 64 ? b_var_ok<double>(dim, N, variant) : b_var_ok<float>(dim, N, variant)))
    return solver_fail(CB_ERR_UNSUPPORTED, "cb_batch_set_variant: variant %d is not built for dim %d N %d",
                       variant, dim, N);
  b->var[dim - 2][N] = variant;
  b->var_set[dim - 2][N] = true;
  return CB_OK;
}

int cb_batch_set_concurrent(cb_batch *b, int on) {
  if (!b) return solver_fail(CB_ERR_ARG, "cb_batch_set_concurrent: null handle");
  if (b->concurrent != (on != 0)) {
    b->concurrent = on != 0;
    drop_graph(b);  // re-built at the next run
  }
  return CB_OK;
}

int cb_batch_set_affine(cb_batch *b, int on) {
  if (!b) return solver_fail(CB_ERR_ARG, "cb_batch_set_affine: null handle");
  b->affine = on != 0;
  return CB_OK;
}

int cb_batch_get_variant(const cb_batch *b, int dim, int N, int *variant) {
  if (!b || !variant || (dim != 2 && dim != 3) || !b_order_ok(dim, N))
    return solver_fail(CB_ERR_ARG, "cb_batch_get_variant: bad arguments");
  *variant = b->var[dim - 2][N];
  return CB_OK;
}

}  // extern "C"

namespace {
template <typename T>
int variant_info(int dim, int N, int variant, int64_t *info) {
  const int sid = shape_id(dim, N, variant);
  BKernels<T> &k = b_kernels<T>();
  if (!k.fn[sid]) return solver_fail(CB_ERR_UNSUPPORTED, "cb_batch_variant_info: variant %d is not built", variant);
  const cudaError_t e = b_prepare<T>(sid);
  if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "cb_batch_variant_info: %s", cudaGetErrorString(e));
  const int Nq = N + 1, Np = dim == 2 ? Nq * Nq : Nq * Nq * Nq;
  info[0] = k.epb[sid];
  info[1] = k.threads[sid];
  info[2] = ((int64_t)k.epb[sid] * Np + k.threads[sid] - 1) / k.threads[sid];
  info[3] = k.ahead[sid];
  info[4] = k.grid[sid] / num_sms();
  info[5] = (int64_t)k.smem[sid];
  return CB_OK;
}
}  // namespace

extern "C" {

int cb_batch_variant_info(const cb_batch *b, int dim, int N, int variant, int64_t *info) {
  if (!b || !info || (dim != 2 && dim != 3) || !b_order_ok(dim, N) || variant < 0 || variant >= NVAR)
    return solver_fail(CB_ERR_ARG, "cb_batch_variant_info: bad arguments");
  return b->prec == 64 ? variant_info<double>(dim, N, variant, info) : variant_info<float>(dim, N, variant, info);
}

int cb_batch_add(cb_batch *b, const cb_mesh *m, void *Q, void *rhs, double dt, int64_t nsteps, const double *qref,
                 int *slot) {
  if (!b || !m || !Q || !rhs || !slot || nsteps < 0 || !std::isfinite(dt))
    return solver_fail(CB_ERR_ARG, "cb_batch_add: bad arguments");
  if (m->prec != b->prec) return solver_fail(CB_ERR_ARG, "cb_batch_add: mesh precision differs from the batch's");
  if (((uintptr_t)Q | (uintptr_t)rhs) & 15)
    return solver_fail(CB_ERR_ARG, "cb_batch_add: Q and rhs must be 16-byte aligned");
  if (const int rc = mesh_check(m)) return rc;
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

int cb_batch_slot_variant(const cb_batch *b, int slot, int *variant) {
  if (!b || !variant || slot < 0 || slot >= b->cap || !b->slots[slot].used)
    return solver_fail(CB_ERR_ARG, "cb_batch_slot_variant: slot is not in use");
  *variant = b->slots[slot].var;
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

int cb_batch_status_async(cb_batch *b, unsigned *out_host) {
  if (!b || !out_host) return solver_fail(CB_ERR_ARG, "cb_batch_status_async: null argument");
  const cudaError_t e =
      cudaMemcpyAsync(out_host, b->status, sizeof(unsigned) * b->cap, cudaMemcpyDeviceToHost, b->stream);
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "cb_batch_status_async: %s", cudaGetErrorString(e));
}

int cb_batch_destroy(cb_batch *b) {
  if (!b) return CB_OK;
  if (b->stream) cudaStreamSynchronize(b->stream);
  drop_graph(b);
  for (BSlot &s : b->slots) {
    if (s.used && s.alt) cudaFreeAsync(s.alt, b->stream);
    if (s.used && s.gq) cudaFreeAsync(s.gq, b->stream);
  }
  for (BList &L : b->list)
    if (L.buf) cudaFreeAsync(L.buf, b->stream);
  if (b->stream) cudaStreamSynchronize(b->stream);
  cudaFree(b->status);
  cudaFree(b->desc);
  cudaFree(b->gqtab);
  cudaFree(b->hdr);
  if (b->pool) cudaMemPoolDestroy(b->pool);
  if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
  delete b;
  return CB_OK;
}

}  // extern "C"
