// C-ABI entry points (include/canary_b200.h): argument checks, dispatch on
// (dim, order, precision), error reporting, and the fused LSRK solver.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/canary_b200.h"
#include "cb_ops.h"

namespace cb {

__global__ void k_round_f32_impl(float *__restrict__ dst, const double *__restrict__ src, int64_t n) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (float)src[i];
}

cudaError_t round_to_f32(float *dst, const double *src, int64_t n, cudaStream_t st) {
  int grid = (int)((n + 255) / 256);
  if (grid > 148 * 16) grid = 148 * 16;
  if (grid < 1) grid = 1;
  k_round_f32_impl<<<grid, 256, 0, st>>>(dst, src, n);
  return cudaGetLastError();
}

}  // namespace cb

using namespace cb;

namespace {

thread_local std::string g_err;

int fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char *where) {
  return fail(CB_ERR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

// One sticky status word per device for the stateless entry points.
std::mutex g_mu;
unsigned *g_status[128] = {nullptr};

unsigned *device_status_word(int *rc) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= 128) {
    *rc = cuda_fail(e, "cudaGetDevice");
    return nullptr;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_status[dev]) {
    unsigned *p = nullptr;
    e = cudaMalloc(&p, sizeof(unsigned));
    if (e != cudaSuccess) {
      *rc = cuda_fail(e, "cudaMalloc(status)");
      return nullptr;
    }
    cudaMemset(p, 0, sizeof(unsigned));
    g_status[dev] = p;
  }
  *rc = CB_OK;
  return g_status[dev];
}

template <typename T>
const Ops<T> *ops_for(int dim, int N, int *rc) {
  const Ops<T> *o = nullptr;
  if (dim == 2) o = get_ops<2, T>(N);
  else if (dim == 3) o = get_ops<3, T>(N);
  else {
    *rc = fail(CB_ERR_ARG, "dim must be 2 or 3 (got %d)", dim);
    return nullptr;
  }
  if (!o) {
    *rc = fail(CB_ERR_UNSUPPORTED, "polynomial order N=%d is outside the compiled range 1..%d", N, MAXN);
    return nullptr;
  }
  *rc = CB_OK;
  return o;
}

Phys to_phys(const cb_phys *p) {
  Phys q;
  q.gamma = p->gamma;
  q.R_gas = p->R_gas;
  q.c_p = p->c_p;
  q.c_v = p->c_v;
  q.gravity = p->gravity;
  q.Pr = p->Pr;
  q.lambda = p->lambda;
  q.visc = p->visc;
  return q;
}

#define CHECK_PTR(p) \
  if (!(p)) return fail(CB_ERR_ARG, "%s: null pointer argument " #p, __func__)
#define CHECK_NELEM(n) \
  if ((n) < 0) return fail(CB_ERR_ARG, "%s: nelem must be >= 0", __func__)

template <typename T>
int volumerhs_impl(int dim, int N, T *rhs, const T *Q, const T *vgeo, const T *D, int64_t nelem,
                   const cb_phys *phys, cudaStream_t st) {
  CHECK_PTR(rhs); CHECK_PTR(Q); CHECK_PTR(vgeo); CHECK_PTR(D); CHECK_PTR(phys); CHECK_NELEM(nelem);
  int rc;
  const Ops<T> *o = ops_for<T>(dim, N, &rc);
  if (!o) return rc;
  if (nelem == 0) return CB_OK;
  cudaError_t e = o->volumerhs(rhs, Q, vgeo, D, nelem, PhysT<T>(to_phys(phys)), st);
  return e == cudaSuccess ? CB_OK : cuda_fail(e, "volumerhs launch");
}

template <typename T>
int fluxrhs_impl(int dim, int N, T *rhs, const T *Q, const T *sgeo, const T *vgeo, int64_t nelem,
                 const int64_t *vmapM, const int64_t *vmapP, const int64_t *bnd,
                 const cb_phys *phys, cudaStream_t st) {
  CHECK_PTR(rhs); CHECK_PTR(Q); CHECK_PTR(sgeo); CHECK_PTR(vgeo); CHECK_PTR(vmapM);
  CHECK_PTR(vmapP); CHECK_PTR(bnd); CHECK_PTR(phys); CHECK_NELEM(nelem);
  int rc;
  const Ops<T> *o = ops_for<T>(dim, N, &rc);
  if (!o) return rc;
  unsigned *status = device_status_word(&rc);
  if (!status) return rc;
  if (nelem == 0) return CB_OK;
  cudaError_t e = o->fluxrhs(rhs, Q, sgeo, vgeo, nelem, vmapM, vmapP, bnd, PhysT<T>(to_phys(phys)),
                             status, st);
  return e == cudaSuccess ? CB_OK : cuda_fail(e, "fluxrhs launch");
}

template <typename T>
int update_impl(int dim, int N, T *rhs, const T *rg, T *Q, const T *vgeo, int64_t nelem, double rka,
                double rkb, double dt, double visc, cudaStream_t st) {
  CHECK_PTR(rhs); CHECK_PTR(Q); CHECK_PTR(vgeo); CHECK_NELEM(nelem);
  int rc;
  const Ops<T> *o = ops_for<T>(dim, N, &rc);
  if (!o) return rc;
  if (nelem == 0) return CB_OK;
  cudaError_t e = o->update(rhs, rg, Q, vgeo, nelem, o->Np, T(rka), T(rkb), T(dt), T(visc), st);
  return e == cudaSuccess ? CB_OK : cuda_fail(e, "updatesolution launch");
}

}  // namespace

namespace cb {
int solver_fail(int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}
}  // namespace cb

// ====================================================================== API
extern "C" {

int cb_version(void) { return 1; }

const char *cb_last_error(void) { return g_err.c_str(); }

int cb_max_order(int dim) { return (dim == 2 || dim == 3) ? MAXN : 0; }

int cb_device_status(cb_stream_t stream) {
  int rc;
  unsigned *status = device_status_word(&rc);
  if (!status) return rc;
  cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return cuda_fail(e, "cudaStreamSynchronize");
  unsigned h = 0;
  e = cudaMemcpy(&h, status, sizeof h, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "read status");
  cudaMemset(status, 0, sizeof(unsigned));
  if (h & ST_BC) return fail(CB_ERR_BC, "invalid boundary condition code (only 0 and 1 are defined)");
  if (h & ST_MESH) return fail(CB_ERR_MESH, "vmapP points outside the mesh (those faces were skipped)");
  if (h & ST_NONFINITE) return fail(CB_ERR_NONFINITE, "non-finite state");
  if (h & ST_TIMEOUT) return fail(CB_ERR_TIMEOUT, "a bounded device wait gave up (that stage stored nothing)");
  return CB_OK;
}

int cb_volumerhs(int dim, int N, double *rhs, const double *Q, const double *vgeo, const double *D,
                 int64_t nelem, const cb_phys *phys, cb_stream_t stream) {
  return volumerhs_impl<double>(dim, N, rhs, Q, vgeo, D, nelem, phys, (cudaStream_t)stream);
}
int cb_volumerhs_f32(int dim, int N, float *rhs, const float *Q, const float *vgeo, const float *D,
                     int64_t nelem, const cb_phys *phys, cb_stream_t stream) {
  return volumerhs_impl<float>(dim, N, rhs, Q, vgeo, D, nelem, phys, (cudaStream_t)stream);
}

int cb_fluxrhs(int dim, int N, double *rhs, const double *Q, const double *sgeo, const double *vgeo,
               int64_t nelem, const int64_t *vmapM, const int64_t *vmapP, const int64_t *elemtobndy,
               const cb_phys *phys, cb_stream_t stream) {
  return fluxrhs_impl<double>(dim, N, rhs, Q, sgeo, vgeo, nelem, vmapM, vmapP, elemtobndy, phys,
                              (cudaStream_t)stream);
}
int cb_fluxrhs_f32(int dim, int N, float *rhs, const float *Q, const float *sgeo, const float *vgeo,
                   int64_t nelem, const int64_t *vmapM, const int64_t *vmapP,
                   const int64_t *elemtobndy, const cb_phys *phys, cb_stream_t stream) {
  return fluxrhs_impl<float>(dim, N, rhs, Q, sgeo, vgeo, nelem, vmapM, vmapP, elemtobndy, phys,
                             (cudaStream_t)stream);
}

int cb_updatesolution(int dim, int N, double *rhs, const double *rhs_gradQ, double *Q,
                      const double *vgeo, int64_t nelem, double rka, double rkb, double dt,
                      double visc, cb_stream_t stream) {
  return update_impl<double>(dim, N, rhs, rhs_gradQ, Q, vgeo, nelem, rka, rkb, dt, visc,
                             (cudaStream_t)stream);
}
int cb_updatesolution_f32(int dim, int N, float *rhs, const float *rhs_gradQ, float *Q,
                          const float *vgeo, int64_t nelem, double rka, double rkb, double dt,
                          double visc, cb_stream_t stream) {
  return update_impl<float>(dim, N, rhs, rhs_gradQ, Q, vgeo, nelem, rka, rkb, dt, visc,
                            (cudaStream_t)stream);
}

int cb_volume_grad(int dim, int N, double *rhs, const double *Q, const double *vgeo, const double *D,
                   int64_t nelem, const cb_phys *phys, cb_stream_t stream) {
  CHECK_PTR(rhs); CHECK_PTR(Q); CHECK_PTR(vgeo); CHECK_PTR(D); CHECK_PTR(phys); CHECK_NELEM(nelem);
  int rc;
  const Ops<double> *o = ops_for<double>(dim, N, &rc);
  if (!o) return rc;
  if (nelem == 0) return CB_OK;
  cudaError_t e = o->volume_grad(rhs, Q, vgeo, D, nelem, PhysT<double>(to_phys(phys)), (cudaStream_t)stream);
  return e == cudaSuccess ? CB_OK : cuda_fail(e, "volume_grad launch");
}

int cb_flux_grad(int dim, int N, double *rhs, const double *Q, const double *sgeo,
                 const double *vgeo, int64_t nelem, const int64_t *vmapM, const int64_t *vmapP,
                 const int64_t *elemtobndy, const cb_phys *phys, cb_stream_t stream) {
  CHECK_PTR(rhs); CHECK_PTR(Q); CHECK_PTR(sgeo); CHECK_PTR(vgeo); CHECK_PTR(vmapM);
  CHECK_PTR(vmapP); CHECK_PTR(elemtobndy); CHECK_PTR(phys); CHECK_NELEM(nelem);
  int rc;
  const Ops<double> *o = ops_for<double>(dim, N, &rc);
  if (!o) return rc;
  unsigned *status = device_status_word(&rc);
  if (!status) return rc;
  if (nelem == 0) return CB_OK;
  cudaError_t e = o->flux_grad(rhs, Q, sgeo, vgeo, nelem, vmapM, vmapP, elemtobndy,
                               PhysT<double>(to_phys(phys)), status, (cudaStream_t)stream);
  return e == cudaSuccess ? CB_OK : cuda_fail(e, "flux_grad launch");
}

int cb_update_gradQ(int dim, int N, double *gradQ, const double *rhs, const double *vgeo,
                    int64_t nelem, cb_stream_t stream) {
  CHECK_PTR(gradQ); CHECK_PTR(rhs); CHECK_PTR(vgeo); CHECK_NELEM(nelem);
  int rc;
  const Ops<double> *o = ops_for<double>(dim, N, &rc);
  if (!o) return rc;
  if (nelem == 0) return CB_OK;
  cudaError_t e = o->update_gradQ(gradQ, rhs, vgeo, nelem, o->Np, (cudaStream_t)stream);
  return e == cudaSuccess ? CB_OK : cuda_fail(e, "update_gradQ launch");
}

int cb_volume_div(int dim, int N, double *rhs, const double *gradQ, const double *Q,
                  const double *vgeo, const double *D, int64_t nelem, const cb_phys *phys,
                  cb_stream_t stream) {
  CHECK_PTR(rhs); CHECK_PTR(gradQ); CHECK_PTR(Q); CHECK_PTR(vgeo); CHECK_PTR(D); CHECK_PTR(phys);
  CHECK_NELEM(nelem);
  int rc;
  const Ops<double> *o = ops_for<double>(dim, N, &rc);
  if (!o) return rc;
  if (nelem == 0) return CB_OK;
  cudaError_t e = o->volume_div(rhs, gradQ, Q, vgeo, D, nelem, PhysT<double>(to_phys(phys)),
                                (cudaStream_t)stream);
  return e == cudaSuccess ? CB_OK : cuda_fail(e, "volume_div launch");
}

int cb_flux_div(int dim, int N, double *rhs, const double *gradQ, const double *Q,
                const double *sgeo, int64_t nelem, const int64_t *vmapM, const int64_t *vmapP,
                const int64_t *elemtobndy, const cb_phys *phys, cb_stream_t stream) {
  CHECK_PTR(rhs); CHECK_PTR(gradQ); CHECK_PTR(Q); CHECK_PTR(sgeo); CHECK_PTR(vmapM);
  CHECK_PTR(vmapP); CHECK_PTR(elemtobndy); CHECK_PTR(phys); CHECK_NELEM(nelem);
  int rc;
  const Ops<double> *o = ops_for<double>(dim, N, &rc);
  if (!o) return rc;
  unsigned *status = device_status_word(&rc);
  if (!status) return rc;
  if (nelem == 0) return CB_OK;
  cudaError_t e = o->flux_div(rhs, gradQ, Q, sgeo, nelem, vmapM, vmapP, elemtobndy,
                              PhysT<double>(to_phys(phys)), status, (cudaStream_t)stream);
  return e == cudaSuccess ? CB_OK : cuda_fail(e, "flux_div launch");
}

}  // extern "C"
