// cb_lsrk_stage_noalloc: one fused LSRK(5,4) stage that allocates nothing.
//
// Some callers cannot allocate device memory themselves or through this
// library: code that runs inside a host framework which owns every device
// allocation (a memory-pool-managed runtime, an embedding that forbids
// cudaMalloc after start-up), or code on a path where an allocation would
// synchronise the device.  For them this entry point performs the same work
// as cb_volumerhs + cb_fluxrhs + cb_updatesolution (visc = 0) in one fused
// pass, with all of its scratch — the copy of the stage's input state that
// neighbour traces are read from, the compact face-neighbour table and a
// sticky status word — in a fixed file-scope device array instead of memory
// from cudaMalloc.  cb_noalloc_status reads (and clears) the sticky word
// without allocating either.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/canary_b200.h"
#include "cb_ops.h"

namespace cb {
int solver_fail(int code, const char *fmt, ...);
}
using namespace cb;

namespace {

constexpr size_t SCRATCH_BYTES = (size_t)CB_NOALLOC_SCRATCH_BYTES;
constexpr size_t ALIGN = 256;

// Every GPU that loads the library holds this array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 128;  // devices whose scratch address is cached
std::mutex g_mu;
void *g_addr[MAX_DEVICES] = {nullptr};

size_t up(size_t b) { return (b + ALIGN - 1) / ALIGN * ALIGN; }

// Scratch layout: [sticky status word | face-neighbour table | stage-input state].
// The status word is never cleared by a stage call (the array starts zeroed
// when the library's device code is loaded); cb_noalloc_status clears it.
constexpr size_t OFF_NBR = ALIGN;

// Device address of the scratch array for the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device, with that device current, and kept for the life of the
// process: after cudaDeviceReset (or any reset of the primary context) the
// cached address is stale, so a process that resets a device must not call
// the allocation-free entry points again.
int scratch_address(void **out, const char *who) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "%s: cudaGetDevice: %s", who, cudaGetErrorString(e));
  if (dev < 0 || dev >= MAX_DEVICES)
    return solver_fail(CB_ERR_UNSUPPORTED, "%s: device %d is beyond the %d devices this library tracks", who, dev,
                       MAX_DEVICES);
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return solver_fail(CB_ERR_CUDA, "%s: cudaGetSymbolAddress: %s", who, cudaGetErrorString(e));
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return CB_OK;
}

}  // namespace

extern "C" int cb_lsrk_stage_noalloc(int dim, int N, double *Q, double *rhs, const double *vgeo,
                                     const double *sgeo, const int64_t *vmapM, const int64_t *vmapP,
                                     const int64_t *elemtobndy, const double *D, int64_t nelem,
                                     const cb_phys *phys, double rka, double rkb, double dt,
                                     unsigned *status, cb_stream_t stream) {
  if (!Q || !rhs || !vgeo || !sgeo || !vmapM || !vmapP || !elemtobndy || !D || !phys)
    return solver_fail(CB_ERR_ARG, "cb_lsrk_stage_noalloc: null pointer argument");
  if (dim != 2 && dim != 3) return solver_fail(CB_ERR_ARG, "cb_lsrk_stage_noalloc: dim must be 2 or 3");
  if (nelem < 0) return solver_fail(CB_ERR_ARG, "cb_lsrk_stage_noalloc: nelem must be >= 0");
  const Ops<double> *o = dim == 2 ? get_ops<2, double>(N) : get_ops<3, double>(N);
  if (!o) return solver_fail(CB_ERR_UNSUPPORTED, "cb_lsrk_stage_noalloc: order N=%d outside 1..%d", N, MAXN);
  if (nelem == 0) return CB_OK;
  const int ns = dim == 2 ? 4 : 5, nface = 2 * dim;
  // reject before any size arithmetic can wrap: the neighbour table and the
  // state copy together take this many bytes per element, plus two padded
  // boundaries
  const size_t per_elem = sizeof(double) * (size_t)o->Np * ns + sizeof(int32_t) * (size_t)nface;
  const size_t max_elems = (SCRATCH_BYTES - OFF_NBR - 2 * ALIGN) / per_elem;
  const size_t qbytes = (size_t)nelem <= max_elems ? sizeof(double) * (size_t)o->Np * ns * (size_t)nelem : 0;
  const size_t nbytes = sizeof(int32_t) * (size_t)nface * ((size_t)nelem <= max_elems ? (size_t)nelem : 0);
  const size_t need = OFF_NBR + up(nbytes) + up(qbytes);
  if ((size_t)nelem > max_elems || need > SCRATCH_BYTES)
    return solver_fail(CB_ERR_ARG,
                       "cb_lsrk_stage_noalloc: nelem=%lld at dim=%d, N=%d exceeds the %zu elements that "
                       "the static scratch of %zu bytes holds (use cb_solver_create for larger meshes)",
                       (long long)nelem, dim, N, max_elems, SCRATCH_BYTES);
  void *base = nullptr;
  int rc = scratch_address(&base, "cb_lsrk_stage_noalloc");
  if (rc) return rc;
  unsigned char *b = (unsigned char *)base;
  unsigned *sticky = (unsigned *)b;
  int32_t *nbr = (int32_t *)(b + OFF_NBR);
  double *Qin = (double *)(b + OFF_NBR + up(nbytes));
  unsigned *st = status ? status : sticky;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if ((e = o->prepare()) != cudaSuccess ||
      (e = o->build_nbr(nbr, vmapM, vmapP, elemtobndy, nelem, st, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(Qin, Q, qbytes, cudaMemcpyDeviceToDevice, s)) != cudaSuccess)
    return solver_fail(CB_ERR_CUDA, "cb_lsrk_stage_noalloc: %s", cudaGetErrorString(e));
  Offs<double, 5> q0;
  for (int k = 0; k < 5; ++k) q0.v[k] = 0.0;
  const PhysT<double> p(Phys{phys->gamma, phys->R_gas, phys->c_p, phys->c_v, phys->gravity, phys->Pr,
                             phys->lambda, phys->visc});
  e = o->stage(Qin, Q, rhs, vgeo, sgeo, nbr, D, nelem, p, q0, rka, rkb * dt, st, s);
  if (e != cudaSuccess) return solver_fail(CB_ERR_CUDA, "cb_lsrk_stage_noalloc: %s", cudaGetErrorString(e));
  return CB_OK;
}

extern "C" int cb_noalloc_status(cb_stream_t stream, unsigned *bits) {
  void *base = nullptr;
  int rc = scratch_address(&base, "cb_noalloc_status");
  if (rc) return rc;
  unsigned h = 0;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if ((e = cudaMemcpyAsync(&h, base, sizeof h, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(base, 0, sizeof h, s)) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return solver_fail(CB_ERR_CUDA, "cb_noalloc_status: %s", cudaGetErrorString(e));
  if (bits) *bits = h;
  if (h & ST_BC) return solver_fail(CB_ERR_BC, "invalid boundary condition code (only 0 and 1 are defined)");
  if (h & ST_MESH) return solver_fail(CB_ERR_MESH, "vmapM/vmapP do not describe a conforming mesh");
  if (h & ST_NONFINITE) return solver_fail(CB_ERR_NONFINITE, "non-finite state");
  if (h & ST_TIMEOUT) return solver_fail(CB_ERR_TIMEOUT, "a bounded device wait gave up");
  return CB_OK;
}
