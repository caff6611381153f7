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
// status word — in a fixed file-scope device array instead of memory from
// cudaMalloc.
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

std::mutex g_mu;
void *g_addr[128] = {nullptr};

size_t up(size_t b) { return (b + ALIGN - 1) / ALIGN * ALIGN; }

// Device address of the scratch array for the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// once per device, with that device current.
int scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 128)
    return solver_fail(CB_ERR_CUDA, "cb_lsrk_stage_noalloc: cudaGetDevice: %s", cudaGetErrorString(e));
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return solver_fail(CB_ERR_CUDA, "cb_lsrk_stage_noalloc: cudaGetSymbolAddress: %s",
                         cudaGetErrorString(e));
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
  const size_t qbytes = sizeof(double) * (size_t)o->Np * ns * (size_t)nelem;
  const size_t nbytes = sizeof(int32_t) * (size_t)nface * (size_t)nelem;
  const size_t need = up(sizeof(unsigned)) + up(nbytes) + up(qbytes);
  if (need > SCRATCH_BYTES)
    return solver_fail(CB_ERR_ARG,
                       "cb_lsrk_stage_noalloc: nelem=%lld at dim=%d, N=%d needs %zu bytes of scratch; "
                       "the static scratch holds %zu bytes (use cb_solver_create for larger meshes)",
                       (long long)nelem, dim, N, need, SCRATCH_BYTES);
  void *base = nullptr;
  int rc = scratch_address(&base);
  if (rc) return rc;
  unsigned char *b = (unsigned char *)base;
  unsigned *own_status = (unsigned *)b;
  int32_t *nbr = (int32_t *)(b + up(sizeof(unsigned)));
  double *Qin = (double *)(b + up(sizeof(unsigned)) + up(nbytes));
  unsigned *st = status ? status : own_status;
  cudaStream_t s = (cudaStream_t)stream;
  cudaError_t e;
  if ((e = cudaMemsetAsync(own_status, 0, sizeof(unsigned), s)) != cudaSuccess ||
      (e = o->prepare()) != cudaSuccess ||
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
