/*
 * CPU oracle for the nodal-DG right-hand side and LSRK(5,4) hot path of
 * CliMA/Canary.jl.
 *
 * THIS IS TEST INFRASTRUCTURE. It is a plain-C restatement of the reference's
 * Julia CPU code path, used only as the parity checker by tests/, by
 * __graft_entry__.smoke() and as the timed CPU baseline arm of bench.py.  The
 * product (canary.jl_b200/) never links, imports or calls it.
 *
 * Parity status: the setup layer (quadrature, operators, brick mesh, Hilbert
 * partition, connectivity, mappings, metric terms) is pinned against the
 * known-answer tests of the reference (test/test_operators.jl,
 * test/test_mesh.jl, test/test_metric.jl).  The RHS / flux / LSRK / LDG
 * kernels have no golden vectors in the reference (its tests never execute
 * the examples) and are pinned by analytic properties instead (free-stream
 * preservation, conservation, convergence to the exact isentropic vortex).
 *
 * Conventions: every array is column-major exactly as in the Julia source,
 * index arrays (vmapM, vmapP, elemtoelem, ...) hold the reference's 1-based
 * Int64 values.  Build with -ffp-contract=off so that each floating-point
 * operation rounds exactly as Julia's scalar code does.
 */
#ifndef CANARY_ORACLE_H
#define CANARY_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Physical constants of the set3c / nse formulations
 * (examples/3d_kernels/euler3d_set3c.jl:113-118, examples/2d_kernels/nse2d.jl:121-128).
 * The pressure law is P = (R_gas/c_v) (E - |U|^2/(2 rho) - rho g z). */
typedef struct or_phys {
  double gamma, R_gas, c_p, c_v, gravity, Pr, lambda, visc;
} or_phys;

/* ---- src/GaussQuadrature/quadrature.jl ---- */
int or_legendre_coefs(int n, double *a, double *b);
int or_custom_gauss_rule(double lo, double hi, int n, double *a, double *b,
                         char endpt, int maxits, double *x, double *w,
                         int *err_iter);
int or_legendre(int n, char endpt, double *x, double *w);

/* ---- src/operators.jl ---- */
int or_lglpoints(int N, double *r, double *w);
int or_lgpoints(int N, double *r, double *w);
void or_baryweights(int n, const double *r, double *wb);
void or_spectralderivative(int n, const double *r, double *D);
void or_interpolationmatrix(int nsrc, const double *rsrc, int ndst,
                            const double *rdst, double *I);

/* ---- src/mesh.jl ---- */
void or_hilbertcode(int n, const uint64_t *Y, int bits, uint64_t *H);
void or_centroidtocode(int d, int nvert, int64_t nelem,
                       const double *elemtocoord, uint64_t *code);
int or_vertsortandorder(int nv, const int64_t *v, int64_t *sorted, int *o,
                        int *flips);
int64_t or_brickmesh(int d, const double *x, const int64_t *nx,
                     const int *periodic, int64_t part, int64_t numparts,
                     const int64_t *boundary, int64_t *elemtovert,
                     double *elemtocoord, int64_t *elemtobndy,
                     int64_t *faceconnections, int64_t *nfc);
int or_partition(int d, int64_t nelem, int64_t *elemtovert,
                 double *elemtocoord, int64_t *elemtobndy,
                 int64_t *faceconnections, int64_t *nfc);
int or_connectmesh(int d, int64_t nelem, const int64_t *elemtovert,
                   const int64_t *elemtobndy_in,
                   const int64_t *faceconnections, int64_t nfc,
                   int64_t *elemtoelem, int64_t *elemtoface,
                   int64_t *elemtoordr, int64_t *elemtobndy);
int or_mappings(int d, int N, int64_t nelem, const int64_t *elemtoelem,
                const int64_t *elemtoface, const int64_t *elemtoordr,
                int64_t *vmapM, int64_t *vmapP);

/* ---- src/metric.jl ---- */
void or_creategrid(int d, int Nq, int64_t nelem, const double *e2c,
                   const double *r, double *x, double *y, double *z);
void or_computemetric1d(int Nq, int64_t nelem, const double *x, double *J,
                        double *xix, double *sJ, double *nx, const double *D);
void or_computemetric2d(int Nq, int64_t nelem, const double *x,
                        const double *y, double *J, double *xix, double *etax,
                        double *xiy, double *etay, double *sJ, double *nx,
                        double *ny, const double *D);
void or_computemetric3d(int Nq, int64_t nelem, const double *x,
                        const double *y, const double *z, double *J,
                        double *xix, double *etax, double *zetax, double *xiy,
                        double *etay, double *zetay, double *xiz,
                        double *etaz, double *zetaz, double *sJ, double *nx,
                        double *ny, double *nz, const double *D);

/* computegeometry of the set3c drivers (euler3d_set3c.jl:210-248,
 * euler2d_set3c.jl:171-208).  warp: 0 none, 1 = x_i += a sin(x)sin(y)[sin(z)]. */
int or_computegeometry(int d, int N, int64_t nelem, const double *elemtocoord,
                       const int64_t *vmapM, int warp, double warp_amp,
                       double *vgeo, double *sgeo);

/* ---- set3c Euler kernels (CPU methods) ---- */
void or_volumerhs(int d, int N, double *rhs, const double *Q,
                  const double *vgeo, const double *D, int64_t nelem,
                  const or_phys *p, int nthreads);
int or_fluxrhs(int d, int N, double *rhs, const double *Q, const double *sgeo,
               const double *vgeo, int64_t nelem, const int64_t *vmapM,
               const int64_t *vmapP, const int64_t *elemtobndy,
               const or_phys *p, int nthreads);
void or_updatesolution(int d, int N, double *rhs, const double *rhs_gradQ,
                       double *Q, const double *vgeo, int64_t nelem,
                       double rka, double rkb, double dt, double visc,
                       int nthreads);

/* ---- nse LDG viscous passes (nse2d.jl:396-814, nse3d.jl:475-995) ---- */
void or_volume_grad(int d, int N, double *rhs, const double *Q,
                    const double *vgeo, const double *D, int64_t nelem,
                    const or_phys *p, int nthreads);
int or_flux_grad(int d, int N, double *rhs, const double *Q,
                 const double *sgeo, const double *vgeo, int64_t nelem,
                 const int64_t *vmapM, const int64_t *vmapP,
                 const int64_t *elemtobndy, const or_phys *p, int nthreads);
void or_update_gradQ(int d, int N, double *gradQ, const double *rhs,
                     const double *vgeo, int64_t nelem, int nthreads);
void or_volume_div(int d, int N, double *rhs, const double *gradQ,
                   const double *Q, const double *vgeo, const double *D,
                   int64_t nelem, const or_phys *p, int nthreads);
int or_flux_div(int d, int N, double *rhs, const double *gradQ,
                const double *Q, const double *sgeo, int64_t nelem,
                const int64_t *vmapM, const int64_t *vmapP,
                const int64_t *elemtobndy, const or_phys *p, int nthreads);

/* ---- lowstorageRK (euler3d_set3c.jl:1361-1523, nse2d.jl:1728-1890) ---- */
int or_lowstorageRK(int d, int N, int64_t nelem, const double *vgeo,
                    const double *sgeo, double *Q, double *rhs,
                    const double *D, double dt, int64_t nsteps,
                    const int64_t *vmapM, const int64_t *vmapP,
                    const int64_t *elemtobndy, const or_phys *p,
                    int nthreads);

/* L2energysquared (euler3d_set3c.jl:1252-1264). */
double or_L2energysquared(int d, int N, int nstate, const double *Q,
                          const double *vgeo, int64_t nelem);

#ifdef __cplusplus
}
#endif
#endif
