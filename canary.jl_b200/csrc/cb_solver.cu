// Fused, graph-captured LSRK(5,4) solver behind cb_solver_* / cb_lsrk_run.
//
// Inviscid form: one k_stage launch per RK stage reads Q from one buffer and
// writes the next state into the other (neighbour traces must see the state
// at the start of the stage), so the state ping-pongs between the caller's Q
// and a solver-owned twin.  Two steps (ten stages) return to the caller's
// buffer and are captured as one CUDA graph; an odd final step is launched
// directly and copied back.
// Viscous (LDG Navier–Stokes) form: for orders whose element groups fit two
// nodes per thread, two fused passes per stage (gradient, then inviscid +
// viscous residual and update) that ping-pong like the inviscid form; above
// that, the reference sequence of passes per stage (volume, face, gradient,
// divergence, update) on a single buffer, captured one step per graph.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/canary_b200.h"
#include "cb_batch.cuh"
#include "cb_ops.h"

using namespace cb;

namespace cb {
int solver_fail(int code, const char *fmt, ...);
}

struct cb_solver {
  int dim = 0, N = 0, prec = 64, device = 0;
  int64_t nelem = 0;
  void *Q = nullptr, *rhs = nullptr, *Qalt = nullptr;
  const void *vgeo = nullptr, *sgeo = nullptr, *D = nullptr;
  void *owned_geo = nullptr;  // FP32 copies of vgeo | sgeo | D (precision 32)
  const int64_t *vmapM = nullptr, *vmapP = nullptr, *bnd = nullptr;
  int32_t *nbr = nullptr;
  void *gradQ = nullptr, *rhs_gradQ = nullptr;
  cb_phys phys{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  unsigned *status = nullptr;
  double *part = nullptr;
  int part_blocks = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  double graph_dt = NAN;
  double qref[5] = {0, 0, 0, 0, 0};  // stored state = Q - qref
  int64_t nghost = 0;  // ghost elements after the nelem own ones in Q and the twin
  int cur = 0;         // stage API: the current state is in Q (0) or in the twin (1)
  int kernel = 0;      // stage kernel choice (cb_solver_set_kernel)
  int64_t nsplit = -1;  // elements 0 .. nsplit - 1 read no ghost (cb_solver_set_split); -1: not set
};

namespace {

const double RKA[5] = {0.0, -567301805773.0 / 1357537059087.0, -2404267990393.0 / 2016746695238.0,
                       -3550918686646.0 / 2091501179385.0, -1275806237668.0 / 842570457699.0};
const double RKB[5] = {1432997174477.0 / 9575080441755.0, 5161836677717.0 / 13612068292357.0,
                       1720146321549.0 / 2090206949498.0, 3134564353537.0 / 4481467310338.0,
                       2277821191437.0 / 14882151754819.0};

template <typename T>
const Ops<T> *ops(const cb_solver *s) {
  return s->dim == 2 ? get_ops<2, T>(s->N) : get_ops<3, T>(s->N);
}
// viscous form through the two fused passes
bool fused_visc(const cb_solver *s) {
  return s->phys.visc > 0 && (s->prec == 64 ? ops<double>(s)->ns_pass != nullptr : ops<float>(s)->ns_pass != nullptr);
}
// the state ping-pongs between Q and Qalt (two steps per graph)
bool pingpong(const cb_solver *s) { return s->phys.visc <= 0 || fused_visc(s); }

template <typename T>
cudaError_t enqueue_step(cb_solver *s, double dt, bool from_user) {
  const Ops<T> *o = ops<T>(s);
  const PhysT<T> p(Phys{s->phys.gamma, s->phys.R_gas, s->phys.c_p, s->phys.c_v, s->phys.gravity,
                        s->phys.Pr, s->phys.lambda, s->phys.visc});
  const T *vg = (const T *)s->vgeo, *sg = (const T *)s->sgeo, *D = (const T *)s->D;
  cudaError_t e = cudaSuccess;
  if (fused_visc(s)) {
    T *a = (T *)(from_user ? s->Q : s->Qalt), *b = (T *)(from_user ? s->Qalt : s->Q);
    BDesc<T> I{};
    I.rhs = (T *)s->rhs;
    I.vgeo = vg;
    I.sgeo = sg;
    I.D = D;
    I.nbr = s->nbr;
    I.status = s->status;
    I.dt = dt;
    for (int k = 0; k < 5; ++k) I.qref[k] = T(s->qref[k]);
    for (int st = 0; st < 5 && e == cudaSuccess; ++st) {
      I.Q[0] = a;
      I.Q[1] = b;
      if ((e = o->ns_pass(0, I, (T *)s->gradQ, s->nelem, p, T(0), T(0), s->stream, s->kernel)) != cudaSuccess) break;
      e = o->ns_pass(1, I, (T *)s->gradQ, s->nelem, p, T(RKA[(st + 1) % 5]), T(RKB[st] * dt), s->stream, s->kernel);
      T *t = a;
      a = b;
      b = t;
    }
    return e;
  }
  if (s->phys.visc > 0) {
    T *Q = (T *)s->Q, *rhs = (T *)s->rhs, *gQ = (T *)s->gradQ, *rg = (T *)s->rhs_gradQ;
    for (int st = 0; st < 5 && e == cudaSuccess; ++st) {
      if ((e = o->volumerhs(rhs, Q, vg, D, s->nelem, p, s->stream)) != cudaSuccess) break;
      if ((e = o->fluxrhs(rhs, Q, sg, vg, s->nelem, s->vmapM, s->vmapP, s->bnd, p, s->status, s->stream)) != cudaSuccess) break;
      if ((e = o->volume_grad(rg, Q, vg, D, s->nelem, p, s->stream)) != cudaSuccess) break;
      if ((e = o->flux_grad(rg, Q, sg, vg, s->nelem, s->vmapM, s->vmapP, s->bnd, p, s->status, s->stream)) != cudaSuccess) break;
      if ((e = o->update_gradQ(gQ, rg, vg, s->nelem, o->Np, s->stream)) != cudaSuccess) break;
      if ((e = o->volume_div(rg, gQ, Q, vg, D, s->nelem, p, s->stream)) != cudaSuccess) break;
      if ((e = o->flux_div(rg, gQ, Q, sg, s->nelem, s->vmapM, s->vmapP, s->bnd, p, s->status, s->stream)) != cudaSuccess) break;
      e = o->update(rhs, rg, Q, vg, s->nelem, o->Np, T(RKA[(st + 1) % 5]), T(RKB[st]), T(dt), T(s->phys.visc), s->stream);
    }
    return e;
  }
  T *a = (T *)(from_user ? s->Q : s->Qalt), *b = (T *)(from_user ? s->Qalt : s->Q);
  Offs<T, 5> q5;
  for (int k = 0; k < 5; ++k) q5.v[k] = T(s->qref[k]);
  for (int st = 0; st < 5 && e == cudaSuccess; ++st) {
    e = o->stage_k(a, b, (T *)s->rhs, vg, sg, s->nbr, D, s->nelem, p, q5, T(RKA[(st + 1) % 5]),
                   T(RKB[st] * dt), s->status, s->stream, 0, s->kernel, 0);
    T *t = a;
    a = b;
    b = t;
  }
  return e;
}

cudaError_t enqueue(cb_solver *s, double dt, bool from_user) {
  return s->prec == 64 ? enqueue_step<double>(s, dt, from_user) : enqueue_step<float>(s, dt, from_user);
}

void drop_graph(cb_solver *s) {
  if (s->exec) cudaGraphExecDestroy(s->exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->exec = nullptr;
  s->graph = nullptr;
  s->graph_dt = NAN;
}

int capture(cb_solver *s, double dt) {
  drop_graph(s);
  cudaError_t e = cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e));
  cudaError_t e1 = enqueue(s, dt, true);
  if (pingpong(s) && e1 == cudaSuccess) e1 = enqueue(s, dt, false);  // two steps
  e = cudaStreamEndCapture(s->stream, &s->graph);
  if (e1 != cudaSuccess || e != cudaSuccess) {
    drop_graph(s);
    return solver_fail(CB_ERR_CUDA, "capture: %s", cudaGetErrorString(e1 != cudaSuccess ? e1 : e));
  }
  e = cudaGraphInstantiate(&s->exec, s->graph, 0);
  if (e != cudaSuccess) {
    drop_graph(s);
    return solver_fail(CB_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
  }
  s->graph_dt = dt;
  return CB_OK;
}

int solver_create(cb_solver **out, int dim, int N, int precision, int64_t nelem, int64_t nghost, void *Q,
                  void *rhs, const double *vgeo, const double *sgeo, const int64_t *vmapM, const int64_t *vmapP,
                  const int64_t *elemtobndy, const double *D, const cb_phys *phys, cb_stream_t stream);

// state bytes of the nelem own elements
size_t state_bytes(const cb_solver *s) {
  const int Nq = s->N + 1;
  const int64_t Np = s->dim == 2 ? (int64_t)Nq * Nq : (int64_t)Nq * Nq * Nq;
  return (s->prec == 64 ? 8 : 4) * (size_t)Np * (s->dim == 2 ? 4 : 5) * s->nelem;
}

// bring the state back into the caller's Q after an odd number of stages
cudaError_t settle(cb_solver *s) {
  if (!s->cur) return cudaSuccess;
  s->cur = 0;
  return cudaMemcpyAsync(s->Q, s->Qalt, state_bytes(s), cudaMemcpyDeviceToDevice, s->stream);
}

// one pass of an RK stage: pass 0 the viscous gradient of the current state
// (nothing for the inviscid form), pass 1 the stage from the current buffer
// into the other
template <typename T>
cudaError_t enqueue_pass(cb_solver *s, int st, double dt, int pass) {
  const Ops<T> *o = ops<T>(s);
  const PhysT<T> p(Phys{s->phys.gamma, s->phys.R_gas, s->phys.c_p, s->phys.c_v, s->phys.gravity,
                        s->phys.Pr, s->phys.lambda, s->phys.visc});
  T *a = (T *)(s->cur ? s->Qalt : s->Q), *b = (T *)(s->cur ? s->Q : s->Qalt);
  if (fused_visc(s)) {
    BDesc<T> I{};
    I.Q[0] = a;
    I.Q[1] = b;
    I.rhs = (T *)s->rhs;
    I.vgeo = (const T *)s->vgeo;
    I.sgeo = (const T *)s->sgeo;
    I.D = (const T *)s->D;
    I.nbr = s->nbr;
    I.status = s->status;
    I.dt = dt;
    for (int k = 0; k < 5; ++k) I.qref[k] = T(s->qref[k]);
    return pass == 0 ? o->ns_pass(0, I, (T *)s->gradQ, s->nelem, p, T(0), T(0), s->stream, s->kernel)
                     : o->ns_pass(1, I, (T *)s->gradQ, s->nelem, p, T(RKA[(st + 1) % 5]), T(RKB[st] * dt), s->stream,
                                  s->kernel);
  }
  if (pass == 0) return cudaSuccess;
  Offs<T, 5> q5;
  for (int k = 0; k < 5; ++k) q5.v[k] = T(s->qref[k]);
  return o->stage_k(a, b, (T *)s->rhs, (const T *)s->vgeo, (const T *)s->sgeo, s->nbr, (const T *)s->D, s->nelem,
                    p, q5, T(RKA[(st + 1) % 5]), T(RKB[st] * dt), s->status, s->stream, 0, s->kernel, 0);
}

// Copy whole elements: gather `n` elements listed in `idx` (device int64) of
// `src` into the contiguous `dst`.
template <typename T>
__global__ void k_pack(const T *__restrict__ src, const int64_t *__restrict__ idx, int64_t n, int64_t ew,
                       T *__restrict__ dst) {
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * ew; t += (int64_t)gridDim.x * blockDim.x)
    dst[t] = src[idx[t / ew] * ew + t % ew];
}

// Face traces of a partitioned solve.  Entry i of `codes` is (element << 3) |
// face; an entry carries the Nfp face-node values of W components (the
// state's fields, or state field x direction for the gradient), each
// component at element offset Np·c.  Pack reads own elements (0 .. nown - 1)
// into buf[(i·W + c)·Nfp + fn]; unpack writes ghost slots (element nown + g
// for code g << 3 | face).  An entry out of range is skipped and raises
// ST_MESH.
template <int DIM, typename T>
__global__ void k_faces(bool pack, T *__restrict__ arr, const int64_t *__restrict__ codes, int64_t n, int Nq,
                        int W, int64_t nown, int64_t nghost, T *__restrict__ buf, unsigned *status) {
  const int Nfp = DIM == 2 ? Nq : Nq * Nq, Np = Nfp * Nq;
  const int64_t per = (int64_t)W * Nfp;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n * per; t += (int64_t)gridDim.x * blockDim.x) {
    const int64_t i = t / per;
    const int c = (int)((t % per) / Nfp), fn = (int)(t % Nfp);
    const int64_t code = codes[i], e = code >> 3;
    const int f = (int)(code & 7);
    if (e < 0 || f >= 2 * DIM || e >= (pack ? nown : nghost)) {
      if (c == 0 && fn == 0) atomicOr(status, ST_MESH);
      continue;
    }
    const int64_t el = pack ? e : nown + e;
    T *a = arr + face_node_rt<DIM>(Nq, f, fn) + (int64_t)Np * (c + (int64_t)W * el);
    if (pack) buf[t] = *a;
    else *a = buf[t];
  }
}

template <typename T>
cudaError_t launch_faces(const cb_solver *s, bool pack, int what, const int64_t *codes, int64_t n, void *buf) {
  const int Nq = s->N + 1, Nfp = s->dim == 2 ? Nq : Nq * Nq;
  const int W = (s->dim == 2 ? 4 : 5) * (what ? s->dim : 1);
  T *arr = (T *)(what ? s->gradQ : (s->cur ? s->Qalt : s->Q));
  const int64_t total = n * W * Nfp;
  const int grid = (int)std::min<int64_t>((total + 255) / 256, 148 * 16);
  if (s->dim == 2)
    k_faces<2, T><<<grid, 256, 0, s->stream>>>(pack, arr, codes, n, Nq, W, s->nelem, s->nghost, (T *)buf, s->status);
  else
    k_faces<3, T><<<grid, 256, 0, s->stream>>>(pack, arr, codes, n, Nq, W, s->nelem, s->nghost, (T *)buf, s->status);
  return cudaGetLastError();
}

int faces(cb_solver *s, bool pack, int what, const int64_t *codes, int64_t n, void *buf) {
  const char *who = pack ? "cb_solver_pack_faces" : "cb_solver_unpack_faces";
  if (!s || n < 0 || (n && (!codes || !buf)) || what < 0 || what > 1 || (what == 1 && !s->gradQ))
    return solver_fail(CB_ERR_ARG, "%s: bad arguments", who);
  if (!n) return CB_OK;
  const cudaError_t e = s->prec == 64 ? launch_faces<double>(s, pack, what, codes, n, buf)
                                      : launch_faces<float>(s, pack, what, codes, n, buf);
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "%s: %s", who, cudaGetErrorString(e));
}

}  // namespace

extern "C" {

int cb_solver_pack_faces(cb_solver *s, int what, const int64_t *codes, int64_t n, void *buf) {
  return faces(s, true, what, codes, n, buf);
}

int cb_solver_unpack_faces(cb_solver *s, int what, const int64_t *codes, int64_t n, void *buf) {
  return faces(s, false, what, codes, n, buf);
}

int cb_solver_set_split(cb_solver *s, int64_t ninterior) {
  if (!s || ninterior < 0 || ninterior > s->nelem)
    return solver_fail(CB_ERR_ARG, "cb_solver_set_split: the split must be within 0..nelem");
  if (s->phys.visc > 0)
    return solver_fail(CB_ERR_UNSUPPORTED, "cb_solver_set_split: the inviscid form only");
  const void *Qa = s->Q, *Qb = s->Qalt;
  const bool ok = s->prec == 64 ? ops<double>(s)->ranged(Qa, s->rhs, s->vgeo, s->sgeo) &&
                                      ops<double>(s)->ranged(Qb, s->rhs, s->vgeo, s->sgeo)
                                : ops<float>(s)->ranged(Qa, s->rhs, s->vgeo, s->sgeo) &&
                                      ops<float>(s)->ranged(Qb, s->rhs, s->vgeo, s->sgeo);
  if (!ok)
    return solver_fail(CB_ERR_UNSUPPORTED,
                       "cb_solver_set_split: this shape's stage does not run over element ranges");
  s->nsplit = ninterior;
  return CB_OK;
}

int cb_solver_stage_split(cb_solver *s, int stage, double dt, int half, void **next_in) {
  if (!s || stage < 0 || stage > 4 || half < 0 || half > 1)
    return solver_fail(CB_ERR_ARG, "cb_solver_stage_split: bad arguments");
  if (s->nsplit < 0) return solver_fail(CB_ERR_ARG, "cb_solver_stage_split: no split set (cb_solver_set_split)");
  const int64_t lo = half ? s->nsplit : 0, hi = half ? s->nelem : s->nsplit;
  cudaError_t e = cudaSuccess;
  if (hi > lo) {
    void *a = s->cur ? s->Qalt : s->Q, *b = s->cur ? s->Q : s->Qalt;
    const Phys ph{s->phys.gamma, s->phys.R_gas, s->phys.c_p, s->phys.c_v, s->phys.gravity, s->phys.Pr,
                  s->phys.lambda, s->phys.visc};
    if (s->prec == 64) {
      Offs<double, 5> q5;
      for (int k = 0; k < 5; ++k) q5.v[k] = s->qref[k];
      e = ops<double>(s)->stage_k((const double *)a, (double *)b, (double *)s->rhs, (const double *)s->vgeo,
                                  (const double *)s->sgeo, s->nbr, (const double *)s->D, hi, PhysT<double>(ph), q5,
                                  RKA[(stage + 1) % 5], RKB[stage] * dt, s->status, s->stream, 0, s->kernel, lo);
    } else {
      Offs<float, 5> q5;
      for (int k = 0; k < 5; ++k) q5.v[k] = (float)s->qref[k];
      e = ops<float>(s)->stage_k((const float *)a, (float *)b, (float *)s->rhs, (const float *)s->vgeo,
                                 (const float *)s->sgeo, s->nbr, (const float *)s->D, hi, PhysT<float>(ph), q5,
                                 (float)RKA[(stage + 1) % 5], (float)(RKB[stage] * dt), s->status, s->stream, 0,
                                 s->kernel, lo);
    }
  }
  if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "cb_solver_stage_split: %s", cudaGetErrorString(e));
  if (half == 1) s->cur ^= 1;
  if (next_in) *next_in = s->cur ? s->Qalt : s->Q;
  return CB_OK;
}

int cb_solver_create(cb_solver **out, int dim, int N, int precision, int64_t nelem, void *Q,
                     void *rhs, const double *vgeo, const double *sgeo, const int64_t *vmapM,
                     const int64_t *vmapP, const int64_t *elemtobndy, const double *D,
                     const cb_phys *phys, cb_stream_t stream) {
  return solver_create(out, dim, N, precision, nelem, 0, Q, rhs, vgeo, sgeo, vmapM, vmapP, elemtobndy, D, phys,
                       stream);
}

int cb_solver_create_ghosted(cb_solver **out, int dim, int N, int precision, int64_t nelem, int64_t nghost,
                             void *Q, void *rhs, const double *vgeo, const double *sgeo, const int64_t *vmapM,
                             const int64_t *vmapP, const int64_t *elemtobndy, const double *D,
                             const cb_phys *phys, cb_stream_t stream) {
  if (nghost < 0) return solver_fail(CB_ERR_ARG, "cb_solver_create_ghosted: nghost must be >= 0");
  // the gravity source reads the neighbour's height from vgeo, which holds
  // the own elements only
  if (nghost > 0 && phys && phys->gravity != 0.0)
    return solver_fail(CB_ERR_UNSUPPORTED, "cb_solver_create_ghosted: ghost elements with gravity != 0");
  return solver_create(out, dim, N, precision, nelem, nghost, Q, rhs, vgeo, sgeo, vmapM, vmapP, elemtobndy, D,
                       phys, stream);
}

int cb_solver_stage_pass(cb_solver *s, int stage, double dt, int pass, void **next_in) {
  if (!s || stage < 0 || stage > 4 || pass < 0 || pass > 1)
    return solver_fail(CB_ERR_ARG, "cb_solver_stage_pass: bad arguments");
  if (!pingpong(s)) return solver_fail(CB_ERR_UNSUPPORTED, "cb_solver_stage: this viscous order has no stage form");
  const cudaError_t e =
      s->prec == 64 ? enqueue_pass<double>(s, stage, dt, pass) : enqueue_pass<float>(s, stage, dt, pass);
  if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "cb_solver_stage: %s", cudaGetErrorString(e));
  if (pass == 1) s->cur ^= 1;
  if (next_in) *next_in = s->cur ? s->Qalt : s->Q;
  return CB_OK;
}

int cb_solver_stage(cb_solver *s, int stage, double dt, void **next_in) {
  const int rc = cb_solver_stage_pass(s, stage, dt, 0, nullptr);
  return rc ? rc : cb_solver_stage_pass(s, stage, dt, 1, next_in);
}

int cb_solver_current(const cb_solver *s, void **state) {
  if (!s || !state) return solver_fail(CB_ERR_ARG, "cb_solver_current: null argument");
  *state = s->cur ? s->Qalt : s->Q;
  return CB_OK;
}

int cb_solver_settle(cb_solver *s) {
  if (!s) return solver_fail(CB_ERR_ARG, "cb_solver_settle: null solver");
  const cudaError_t e = settle(s);
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "cb_solver_settle: %s", cudaGetErrorString(e));
}

int cb_solver_pack(cb_solver *s, int what, const int64_t *elems, int64_t n, void *buf) {
  if (!s || n < 0 || (n && (!elems || !buf)) || what < 0 || what > 1 || (what == 1 && !s->gradQ))
    return solver_fail(CB_ERR_ARG, "cb_solver_pack: bad arguments");
  if (!n) return CB_OK;
  const int Nq = s->N + 1;
  const int64_t ew = (s->dim == 2 ? (int64_t)Nq * Nq * 4 : (int64_t)Nq * Nq * Nq * 5) * (what ? s->dim : 1);
  const int grid = (int)std::min<int64_t>((n * ew + 255) / 256, 148 * 16);
  const void *src = what ? s->gradQ : (s->cur ? s->Qalt : s->Q);
  if (s->prec == 64)
    k_pack<double><<<grid, 256, 0, s->stream>>>((const double *)src, elems, n, ew, (double *)buf);
  else
    k_pack<float><<<grid, 256, 0, s->stream>>>((const float *)src, elems, n, ew, (float *)buf);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "cb_solver_pack: %s", cudaGetErrorString(e));
}

int cb_solver_unpack(cb_solver *s, int what, const void *buf, int64_t first, int64_t n) {
  if (!s || what < 0 || what > 1 || (what == 1 && !s->gradQ))
    return solver_fail(CB_ERR_ARG, "cb_solver_unpack: bad arguments");
  if (first < 0 || n < 0 || first + n > s->nghost || (n && !buf))
    return solver_fail(CB_ERR_ARG, "cb_solver_unpack: ghost range outside 0..%lld", (long long)s->nghost);
  if (!n) return CB_OK;
  const size_t ew = state_bytes(s) / (size_t)s->nelem * (what ? s->dim : 1);
  char *dst = (char *)(what ? s->gradQ : (s->cur ? s->Qalt : s->Q)) + ew * (size_t)(s->nelem + first);
  const cudaError_t e = cudaMemcpyAsync(dst, buf, ew * (size_t)n, cudaMemcpyDeviceToDevice, s->stream);
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "cb_solver_unpack: %s", cudaGetErrorString(e));
}

}  // extern "C"

namespace {

int solver_create(cb_solver **out, int dim, int N, int precision, int64_t nelem, int64_t nghost, void *Q,
                  void *rhs, const double *vgeo, const double *sgeo, const int64_t *vmapM, const int64_t *vmapP,
                  const int64_t *elemtobndy, const double *D, const cb_phys *phys, cb_stream_t stream) {
  if (!out || !Q || !rhs || !vgeo || !sgeo || !vmapM || !vmapP || !elemtobndy || !D || !phys)
    return solver_fail(CB_ERR_ARG, "cb_solver_create: null pointer argument");
  if (dim != 2 && dim != 3) return solver_fail(CB_ERR_ARG, "dim must be 2 or 3");
  if (precision != 32 && precision != 64) return solver_fail(CB_ERR_ARG, "precision must be 32 or 64");
  if (nelem <= 0) return solver_fail(CB_ERR_ARG, "nelem must be positive");
  if (N < 1 || N > MAXN) return solver_fail(CB_ERR_UNSUPPORTED, "order N=%d outside 1..%d", N, MAXN);
  *out = nullptr;
  cb_solver *s = new cb_solver();
  s->dim = dim;
  s->N = N;
  s->prec = precision;
  s->nelem = nelem;
  s->Q = Q;
  s->rhs = rhs;
  s->vmapM = vmapM;
  s->vmapP = vmapP;
  s->bnd = elemtobndy;
  s->phys = *phys;
  s->nghost = nghost;
  cudaGetDevice(&s->device);
  const int Nq = N + 1;
  const int64_t Np = dim == 2 ? (int64_t)Nq * Nq : (int64_t)Nq * Nq * Nq;
  const int64_t Nfp = dim == 2 ? Nq : (int64_t)Nq * Nq;
  const int ns = dim == 2 ? 4 : 5, nvg = dim == 2 ? 8 : 14, nsg = dim == 2 ? 4 : 5, nface = 2 * dim;
  const size_t w = precision == 64 ? 8 : 4;
  cudaError_t e = cudaSuccess;
  auto bail = [&](int code, const char *what) {
    cb_solver_destroy(s);
    return solver_fail(code, "cb_solver_create: %s: %s", what, cudaGetErrorString(e));
  };
  if (stream) {
    s->stream = (cudaStream_t)stream;
  } else {
    // graph capture is not allowed on the legacy default stream; a blocking
    // stream stays ordered with work the caller put on stream 0
    if ((e = cudaStreamCreate(&s->stream)) != cudaSuccess) return bail(CB_ERR_CUDA, "stream");
    s->own_stream = true;
  }
  if ((e = cudaMalloc(&s->status, sizeof(unsigned))) != cudaSuccess) return bail(CB_ERR_NOMEM, "status");
  cudaMemsetAsync(s->status, 0, sizeof(unsigned), s->stream);
  s->part_blocks = 296;
  if ((e = cudaMalloc(&s->part, sizeof(double) * 4 * ns * s->part_blocks)) != cudaSuccess)
    return bail(CB_ERR_NOMEM, "partials");
  if (phys->visc > 0 && nghost > 0 && !fused_visc(s)) {
    cb_solver_destroy(s);
    return solver_fail(CB_ERR_UNSUPPORTED, "cb_solver_create_ghosted: this viscous order has no stage form");
  }
  if (phys->visc > 0) {
    const size_t gbytes = w * (size_t)Np * ns * dim * (nelem + nghost);
    if ((e = cudaMalloc(&s->gradQ, gbytes)) != cudaSuccess) return bail(CB_ERR_NOMEM, "gradQ");
    cudaMemsetAsync(s->gradQ, 0, gbytes, s->stream);
    if (!fused_visc(s)) {
      if ((e = cudaMalloc(&s->rhs_gradQ, gbytes)) != cudaSuccess) return bail(CB_ERR_NOMEM, "rhs_gradQ");
      cudaMemsetAsync(s->rhs_gradQ, 0, gbytes, s->stream);
    }
  }
  if (pingpong(s)) {
    if ((e = cudaMalloc(&s->Qalt, w * (size_t)Np * ns * (nelem + nghost))) != cudaSuccess)
      return bail(CB_ERR_NOMEM, "state twin");
    if ((e = cudaMalloc(&s->nbr, sizeof(int32_t) * nface * nelem)) != cudaSuccess) return bail(CB_ERR_NOMEM, "neighbours");
  }
  if (precision == 64) {
    s->vgeo = vgeo;
    s->sgeo = sgeo;
    s->D = D;
  } else {
    const int64_t nv = Np * nvg * nelem, ns_ = nsg * Nfp * nface * nelem, nd = (int64_t)Nq * Nq;
    // each array starts on a 16-byte boundary (the pipelined stages copy
    // element slabs with bulk copies)
    const int64_t nvp = (nv + 3) & ~int64_t(3), nsp = (ns_ + 3) & ~int64_t(3);
    if ((e = cudaMalloc(&s->owned_geo, sizeof(float) * (nvp + nsp + nd))) != cudaSuccess)
      return bail(CB_ERR_NOMEM, "fp32 geometry");
    float *g = (float *)s->owned_geo;
    round_to_f32(g, vgeo, nv, s->stream);
    round_to_f32(g + nvp, sgeo, ns_, s->stream);
    round_to_f32(g + nvp + nsp, D, nd, s->stream);
    s->vgeo = g;
    s->sgeo = g + nvp;
    s->D = g + nvp + nsp;
  }
  e = precision == 64 ? ops<double>(s)->prepare() : ops<float>(s)->prepare();
  if (e != cudaSuccess) return bail(CB_ERR_CUDA, "kernel attributes");
  if (pingpong(s)) {
    const Ops<double> *o = ops<double>(s);
    if ((e = o->build_nbr_ghost(s->nbr, vmapM, vmapP, elemtobndy, nelem, nelem + nghost, s->status, s->stream)) !=
        cudaSuccess)
      return bail(CB_ERR_CUDA, "neighbour table");
  }
  unsigned h = 0;
  if ((e = cudaMemcpyAsync(&h, s->status, sizeof h, cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s->stream)) != cudaSuccess)
    return bail(CB_ERR_CUDA, "setup");
  if (h & ST_BC) {
    cb_solver_destroy(s);
    return solver_fail(CB_ERR_BC, "invalid boundary condition code (only 0 and 1 are defined)");
  }
  if (h & ST_MESH) {
    cb_solver_destroy(s);
    return solver_fail(CB_ERR_MESH, "vmapM/vmapP do not describe a conforming mesh with orientation 1");
  }
  *out = s;
  return CB_OK;
}

}  // namespace

extern "C" {

int cb_lsrk_run(cb_solver *s, int64_t nsteps, double dt) {
  if (!s) return solver_fail(CB_ERR_ARG, "null solver");
  if (nsteps < 0) return solver_fail(CB_ERR_ARG, "nsteps must be >= 0");
  if (nsteps == 0) return CB_OK;
  cudaError_t e0 = settle(s);  // a state left in the twin by the stage API
  if (e0 != cudaSuccess) return solver_fail(CB_ERR_CUDA, "state copy: %s", cudaGetErrorString(e0));
  const int64_t per_graph = pingpong(s) ? 2 : 1;
  const int64_t reps = nsteps / per_graph, rem = nsteps % per_graph;
  cudaError_t e;
  if (reps > 0) {
    if (!s->exec || s->graph_dt != dt) {
      int rc = capture(s, dt);
      if (rc) return rc;
    }
    for (int64_t r = 0; r < reps; ++r)
      if ((e = cudaGraphLaunch(s->exec, s->stream)) != cudaSuccess)
        return solver_fail(CB_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
  }
  if (rem) {
    if ((e = enqueue(s, dt, true)) != cudaSuccess)
      return solver_fail(CB_ERR_CUDA, "step launch: %s", cudaGetErrorString(e));
    const int Nq = s->N + 1;
    const int64_t Np = s->dim == 2 ? (int64_t)Nq * Nq : (int64_t)Nq * Nq * Nq;
    const size_t bytes = (s->prec == 64 ? 8 : 4) * (size_t)Np * (s->dim == 2 ? 4 : 5) * s->nelem;
    if ((e = cudaMemcpyAsync(s->Q, s->Qalt, bytes, cudaMemcpyDeviceToDevice, s->stream)) != cudaSuccess)
      return solver_fail(CB_ERR_CUDA, "state copy: %s", cudaGetErrorString(e));
  }
  return CB_OK;
}

int cb_solver_sums(cb_solver *s, double *out_host) {
  if (!s || !out_host) return solver_fail(CB_ERR_ARG, "null argument");
  const int ns = s->dim == 2 ? 4 : 5, Nq = s->N + 1;
  const int Np = s->dim == 2 ? Nq * Nq : Nq * Nq * Nq;
  Offs<double, 5> q5;
  for (int k = 0; k < 5; ++k) q5.v[k] = s->qref[k];
  const void *Qc = s->cur ? s->Qalt : s->Q;  // the current state
  cudaError_t e = s->prec == 64
                      ? ops<double>(s)->cons_sums((const double *)Qc, (const double *)s->vgeo, s->nelem, Np, q5, s->part, s->part_blocks, s->stream)
                      : ops<float>(s)->cons_sums((const float *)Qc, (const float *)s->vgeo, s->nelem, Np, q5, s->part, s->part_blocks, s->stream);
  if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "sums launch: %s", cudaGetErrorString(e));
  std::string buf(sizeof(double) * 4 * ns * s->part_blocks, '\0');
  double *h = (double *)&buf[0];
  unsigned st = 0;
  if ((e = cudaMemcpyAsync(h, s->part, buf.size(), cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(&st, s->status, sizeof st, cudaMemcpyDeviceToHost, s->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s->stream)) != cudaSuccess)
    return solver_fail(CB_ERR_CUDA, "sums: %s", cudaGetErrorString(e));
  for (int q = 0; q < 2 * ns; ++q) {
    double sum = 0.0, comp = 0.0;
    for (int b = 0; b < s->part_blocks; ++b) {
      const double v = h[b * 4 * ns + 2 * q], c = h[b * 4 * ns + 2 * q + 1];
      const double t = sum + v;
      if (std::fabs(sum) >= std::fabs(v)) comp += (sum - t) + v;
      else comp += (v - t) + sum;
      sum = t;
      comp += c;
    }
    // q = 2*s + k  (k = 0: Σ MJ Q, k = 1: Σ MJ Q²) -> out[k*ns + s]
    out_host[(q % 2) * ns + q / 2] = sum + comp;
  }
  if (st & ST_TIMEOUT)
    return solver_fail(CB_ERR_TIMEOUT, "a bounded device wait gave up: a stage stored nothing, the state is stale");
  if (st & ST_NONFINITE) return solver_fail(CB_ERR_NONFINITE, "the state became non-finite");
  if (st & ST_BC) return solver_fail(CB_ERR_BC, "invalid boundary condition code");
  return CB_OK;
}

int cb_solver_set_offset(cb_solver *s, const double *qref) {
  if (!s || !qref) return solver_fail(CB_ERR_ARG, "null argument");
  if (s->phys.visc > 0 && !fused_visc(s)) {
    for (int k = 0; k < (s->dim == 2 ? 4 : 5); ++k)
      if (qref[k] != 0.0)
        return solver_fail(CB_ERR_UNSUPPORTED, "state offsets: the viscous form of this order has none");
    return CB_OK;
  }
  for (int k = 0; k < (s->dim == 2 ? 4 : 5); ++k) s->qref[k] = qref[k];
  drop_graph(s);
  return CB_OK;
}

int cb_solver_set_kernel(cb_solver *s, int kernel) {
  if (!s || kernel < 0 || kernel > 4) return solver_fail(CB_ERR_ARG, "cb_solver_set_kernel: bad arguments");
  if (kernel == 4) {
    const bool lean = s->prec == 64 ? ops<double>(s)->lean : ops<float>(s)->lean;
    if (!lean || s->phys.visc > 0)
      return solver_fail(CB_ERR_UNSUPPORTED, "cb_solver_set_kernel: the lean stage is not built for this shape");
  }
  if (kernel == 2) {
    const bool mma = s->prec == 64 ? ops<double>(s)->mma : ops<float>(s)->mma;
    if (!mma || s->phys.visc > 0)
      return solver_fail(CB_ERR_UNSUPPORTED,
                         "cb_solver_set_kernel: the tensor-core stage is built for the inviscid 3-D N=7 form");
  }
  if (kernel != s->kernel) drop_graph(s);
  s->kernel = kernel;
  return CB_OK;
}

int cb_solver_get_kernel(const cb_solver *s, int *kernel) {
  if (!s || !kernel) return solver_fail(CB_ERR_ARG, "cb_solver_get_kernel: null argument");
  const int def = s->prec == 64 ? ops<double>(s)->default_kernel : ops<float>(s)->default_kernel;
  *kernel = s->kernel ? s->kernel : (s->phys.visc > 0 ? 1 : def);
  return CB_OK;
}

int cb_solver_reset_status(cb_solver *s) {
  if (!s) return solver_fail(CB_ERR_ARG, "cb_solver_reset_status: null solver");
  const cudaError_t e = cudaMemsetAsync(s->status, 0, sizeof(unsigned), s->stream);
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "cb_solver_reset_status: %s", cudaGetErrorString(e));
}

int cb_solver_test_timeout(cb_solver *s) {
  if (!s) return solver_fail(CB_ERR_ARG, "cb_solver_test_timeout: null solver");
  if (s->phys.visc > 0)
    return solver_fail(CB_ERR_UNSUPPORTED, "cb_solver_test_timeout: the inviscid pipelined stage only");
  const PhysT<double> p64(Phys{s->phys.gamma, s->phys.R_gas, s->phys.c_p, s->phys.c_v, s->phys.gravity, s->phys.Pr,
                               s->phys.lambda, s->phys.visc});
  const PhysT<float> p32(Phys{s->phys.gamma, s->phys.R_gas, s->phys.c_p, s->phys.c_v, s->phys.gravity, s->phys.Pr,
                              s->phys.lambda, s->phys.visc});
  void *a = s->cur ? s->Qalt : s->Q, *b = s->cur ? s->Q : s->Qalt;
  cudaError_t e;
  if (s->prec == 64) {
    Offs<double, 5> q5;
    for (int k = 0; k < 5; ++k) q5.v[k] = s->qref[k];
    e = ops<double>(s)->stage_k((const double *)a, (double *)b, (double *)s->rhs, (const double *)s->vgeo,
                                (const double *)s->sgeo, s->nbr, (const double *)s->D, s->nelem, p64, q5, RKA[1],
                                RKB[0], s->status, s->stream, 1, s->kernel, 0);
  } else {
    Offs<float, 5> q5;
    for (int k = 0; k < 5; ++k) q5.v[k] = (float)s->qref[k];
    e = ops<float>(s)->stage_k((const float *)a, (float *)b, (float *)s->rhs, (const float *)s->vgeo,
                               (const float *)s->sgeo, s->nbr, (const float *)s->D, s->nelem, p32, q5,
                               (float)RKA[1], (float)RKB[0], s->status, s->stream, 1, s->kernel, 0);
  }
  if (e == cudaErrorNotSupported)  // returned by the launcher, not by CUDA
    return solver_fail(CB_ERR_UNSUPPORTED, "cb_solver_test_timeout: this shape does not run the pipelined stage");
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "cb_solver_test_timeout: %s", cudaGetErrorString(e));
}

int cb_solver_status_async(cb_solver *s, unsigned *out_host) {
  if (!s || !out_host) return solver_fail(CB_ERR_ARG, "cb_solver_status_async: null argument");
  const cudaError_t e = cudaMemcpyAsync(out_host, s->status, sizeof(unsigned), cudaMemcpyDeviceToHost, s->stream);
  return e == cudaSuccess ? CB_OK : solver_fail(CB_ERR_CUDA, "cb_solver_status_async: %s", cudaGetErrorString(e));
}

int cb_solver_destroy(cb_solver *s) {
  if (!s) return CB_OK;
  if (s->stream) cudaStreamSynchronize(s->stream);
  drop_graph(s);
  cudaFree(s->Qalt);
  cudaFree(s->nbr);
  cudaFree(s->gradQ);
  cudaFree(s->rhs_gradQ);
  cudaFree(s->owned_geo);
  cudaFree(s->status);
  cudaFree(s->part);
  if (s->own_stream && s->stream) cudaStreamDestroy(s->stream);
  delete s;
  return CB_OK;
}

}  // extern "C"
