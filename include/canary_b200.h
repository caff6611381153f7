/*
 * canary_b200 — C-ABI of the B200 (sm_100a) nodal-DG hot path of
 * CliMA/Canary.jl: volume RHS, Rusanov face flux, LDG Navier–Stokes passes
 * and the Carpenter–Kennedy LSRK(5,4) update.
 *
 * Every array argument is a DEVICE pointer owned by the caller and uses the
 * reference's column-major Julia layout unchanged:
 *
 *   Q, rhs       (Np, nstate, nelem)          state order 3-D (U,V,W,ρ,E),
 *                                              2-D (U,V,ρ,E)
 *   gradQ        (Np, nstate, dim, nelem)
 *   vgeo         (Np, nvgeo, nelem)           3-D (ξx,ηx,ζx,ξy,ηy,ζy,ξz,ηz,ζz,
 *                                              MJ,MJI,x,y,z); 2-D (ξx,ηx,ξy,ηy,
 *                                              MJ,MJI,x,y)
 *   sgeo         (nsgeo, Nfp, nface, nelem)   3-D (nx,ny,nz,sMJ,vMJI);
 *                                              2-D (nx,ny,sMJ,vMJI)
 *   vmapM/vmapP  (Nfp, nface, nelem) int64, 1-based node ids (mesh.jl:973)
 *   elemtobndy   (nface, nelem) int64, 0 = connected face, 1 = wall
 *   D            (Nq, Nq) spectral derivative matrix (operators.jl:84)
 *
 * with Nq = N+1, Np = Nq^dim, Nfp = Nq^(dim-1), nface = 2 dim.  Calls are
 * asynchronous on `stream` (0 = legacy default stream) and return a status
 * code; they never synchronise the device except where stated.
 *
 * The `_f32` twins take single-precision arrays of the same layouts.
 */
#ifndef CANARY_B200_H
#define CANARY_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *cb_stream_t; /* == cudaStream_t */

/* Status codes. */
enum {
  CB_OK = 0,
  CB_ERR_ARG = 1,         /* bad dimension, order, size or null pointer   */
  CB_ERR_UNSUPPORTED = 2, /* (dim, N) outside the compiled range          */
  CB_ERR_BC = 3,          /* boundary code other than 0 or 1              */
  CB_ERR_CUDA = 4,        /* a CUDA runtime call failed                   */
  CB_ERR_MESH = 5,        /* vmapM/vmapP do not describe a conforming mesh*/
  CB_ERR_NONFINITE = 6,   /* the state became NaN or Inf                  */
  CB_ERR_TIMEOUT = 7,     /* a bounded device wait gave up                */
  CB_ERR_NOMEM = 8        /* allocation failed                            */
};

/* Physical constants of the set3c / nse formulations.  Reference values:
 * euler3d_set3c.jl:113-118 (γ=7/5, R_gas=287.17, c_p=1004.67, c_v=717.5,
 * gravity=10) and nse2d.jl:127-128 (Pr=71/10, λ=-2/3).  The pressure law is
 * P = (R_gas/c_v)(E - |U|²/(2ρ) - ρ g x_dim); `visc` multiplies the viscous
 * residual as the `visc` argument of nse()/updatesolution! does. */
typedef struct cb_phys {
  double gamma;
  double R_gas;
  double c_p;
  double c_v;
  double gravity;
  double Pr;
  double lambda;
  double visc;
} cb_phys;

/* Library identification and error reporting. */
int cb_version(void);
/* Message of the last failing call on this host thread ("" if none). */
const char *cb_last_error(void);
/* Synchronises `stream` and returns (and clears) the sticky device-side
 * status raised by kernels since the last call: CB_ERR_BC when a face with a
 * boundary code other than 0/1 was met (that face is skipped, as no valid
 * flux exists), CB_ERR_NONFINITE, or CB_OK. */
int cb_device_status(cb_stream_t stream);
/* Largest polynomial order compiled for `dim` (orders 1..max are built). */
int cb_max_order(int dim);

/* ---------------------------------------------------------------------- */
/* Per-function drop-ins of the reference's kernels (stateless).          */
/* ---------------------------------------------------------------------- */

/* rhs += volume integral (and the -MJ ρ g buoyancy source).
 * Replaces volumerhs!(Val(dim), Val(N), d_rhsC::CuArray, d_QC, d_vgeoC, d_D,
 * elems): euler2d_set3c.jl:975-980 / euler3d_set3c.jl:1227-1232 (CPU
 * semantics euler3d_set3c.jl:253-339). */
int cb_volumerhs(int dim, int N, double *rhs, const double *Q,
                 const double *vgeo, const double *D, int64_t nelem,
                 const cb_phys *phys, cb_stream_t stream);
int cb_volumerhs_f32(int dim, int N, float *rhs, const float *Q,
                     const float *vgeo, const float *D, int64_t nelem,
                     const cb_phys *phys, cb_stream_t stream);

/* rhs -= sMJ · Rusanov flux at every face node of every element.
 * Replaces fluxrhs!(Val(dim), Val(N), d_rhsL::CuArray, d_QL, d_sgeo, d_vgeoL,
 * elems, d_vmapM, d_vmapP, d_elemtobndy): euler2d_set3c.jl:982-988 /
 * euler3d_set3c.jl:1234-1240 (CPU semantics euler3d_set3c.jl:342-458). */
int cb_fluxrhs(int dim, int N, double *rhs, const double *Q,
               const double *sgeo, const double *vgeo, int64_t nelem,
               const int64_t *vmapM, const int64_t *vmapP,
               const int64_t *elemtobndy, const cb_phys *phys,
               cb_stream_t stream);
int cb_fluxrhs_f32(int dim, int N, float *rhs, const float *Q,
                   const float *sgeo, const float *vgeo, int64_t nelem,
                   const int64_t *vmapM, const int64_t *vmapP,
                   const int64_t *elemtobndy, const cb_phys *phys,
                   cb_stream_t stream);

/* rhs += visc·rhs_gradQ[:,:,1,:] (skipped when rhs_gradQ is NULL);
 * Q += rkb·dt·rhs·MJI; rhs *= rka.
 * Replaces updatesolution!(Val(dim), Val(N), d_rhsL::CuArray, d_rhs_gradQL,
 * d_QL, d_vgeoL, elems, rka, rkb, dt, visc): euler3d_set3c.jl:862-872 /
 * nse2d.jl:806-814 (GPU form euler2d_set3c.jl:990-996). */
int cb_updatesolution(int dim, int N, double *rhs, const double *rhs_gradQ,
                      double *Q, const double *vgeo, int64_t nelem, double rka,
                      double rkb, double dt, double visc, cb_stream_t stream);
int cb_updatesolution_f32(int dim, int N, float *rhs, const float *rhs_gradQ,
                          float *Q, const float *vgeo, int64_t nelem,
                          double rka, double rkb, double dt, double visc,
                          cb_stream_t stream);

/* LDG Navier–Stokes passes (nse2d.jl:396-778, nse3d.jl:475-970).
 * volume_grad! zeroes rhs (Np,nstate,dim,nelem) and writes -Dᵀ(MJ ξ·q̂) of the
 * primitives q̂ = (u,v,[w],ρ,T); flux_grad! adds the central trace term;
 * update_gradQ! scales by MJI; volume_div!/flux_div! build the divergence of
 * the viscous stress / heat flux into rhs[:,:,1,:]. */
int cb_volume_grad(int dim, int N, double *rhs, const double *Q,
                   const double *vgeo, const double *D, int64_t nelem,
                   const cb_phys *phys, cb_stream_t stream);
int cb_flux_grad(int dim, int N, double *rhs, const double *Q,
                 const double *sgeo, const double *vgeo, int64_t nelem,
                 const int64_t *vmapM, const int64_t *vmapP,
                 const int64_t *elemtobndy, const cb_phys *phys,
                 cb_stream_t stream);
int cb_update_gradQ(int dim, int N, double *gradQ, const double *rhs,
                    const double *vgeo, int64_t nelem, cb_stream_t stream);
int cb_volume_div(int dim, int N, double *rhs, const double *gradQ,
                  const double *Q, const double *vgeo, const double *D,
                  int64_t nelem, const cb_phys *phys, cb_stream_t stream);
int cb_flux_div(int dim, int N, double *rhs, const double *gradQ,
                const double *Q, const double *sgeo, int64_t nelem,
                const int64_t *vmapM, const int64_t *vmapP,
                const int64_t *elemtobndy, const cb_phys *phys,
                cb_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Fused, graph-captured LSRK(5,4) driver (drop-in for lowstorageRK).      */
/* ---------------------------------------------------------------------- */

/* Opaque solver bound to one mesh and one caller-owned state.
 * Replaces lowstorageRK(Val(dim), Val(N), mesh, vgeo, sgeo, Q, rhs, D, dt,
 * nsteps, tout, vmapM, vmapP, mpicomm, iplot, visc; ArrType=CuArray):
 * euler3d_set3c.jl:1361-1523, nse2d.jl:1728-1890.
 *
 * precision = 64: Q/rhs are double and vgeo/sgeo/D are used as given.
 * precision = 32: Q/rhs are float; vgeo/sgeo/D are the FP64 arrays, rounded
 *                 once into solver-owned FP32 copies.
 * The solver owns its scratch (a second state buffer for the double-buffered
 * stage, compact int32 face-neighbour tables built from vmapM/vmapP, the
 * gradient arrays of the viscous form and the captured CUDA graph). */
typedef struct cb_solver cb_solver;

int cb_solver_create(cb_solver **out, int dim, int N, int precision,
                     int64_t nelem, void *Q, void *rhs, const double *vgeo,
                     const double *sgeo, const int64_t *vmapM,
                     const int64_t *vmapP, const int64_t *elemtobndy,
                     const double *D, const cb_phys *phys,
                     cb_stream_t stream);
/* Advance Q and the residual carry rhs by nsteps LSRK(5,4) steps of size dt.
 * Asynchronous; the first call for a given dt captures one step into a CUDA
 * graph that later calls replay. */
int cb_lsrk_run(cb_solver *s, int64_t nsteps, double dt);
/* Per-field constants qref[nstate] (host array) for the stored state: the
 * state array then holds Q - qref and the kernels add qref back when they form
 * fluxes.  Used by the FP32 form so that the per-stage rounding of the update
 * is relative to the deviation from a reference state (e.g. the free stream)
 * rather than to the full state; FP64 solvers leave it at zero.  Inviscid
 * form only.  The conservation sums below are reported for the full Q. */
int cb_solver_set_offset(cb_solver *s, const double *qref);
/* Compensated (Neumaier) FP64 sums over all nodes of MJ·Q[:,s,:] and
 * MJ·Q[:,s,:]² for every state field s: out[2*nstate]; synchronises. */
int cb_solver_sums(cb_solver *s, double *out_host);
/* Enqueue on the solver's stream a copy of its status bits (bit 2:
 * non-finite state) into *out_host (page-locked memory for an asynchronous
 * copy); the value is valid once the stream has reached the copy. */
int cb_solver_status_async(cb_solver *s, unsigned *out_host);
/* Stage kernel: 0 = the default for the shape, 1 = the CUDA-core stages
 * (pipelined bulk-copy staging where the plan fits), 2 = the tensor-core
 * stage of the inviscid form (D contraction on the FP64 tensor pipe as 8x8x4
 * DMMA tiles, for FP32 solvers on the FP32 fluxes converted to FP64, the sum
 * rounded once; built for 3-D N=7, CB_ERR_UNSUPPORTED elsewhere), 3 = the
 * unpipelined grouped stages (the inviscid k_stage; for the fused viscous
 * form the grouped passes instead of the pipelined ones), 4 = the lean
 * pipelined stage of the inviscid form (only the state staged in shared
 * memory, the geometry and carry read from L2; bit-identical to 1).  The
 * default is the fastest on B200 for the shape.  All agree with the oracle
 * to round-off; changing it re-captures the step graph at the next run.
 * cb_solver_get_kernel reports the kernel the solver runs (1 to 4). */
int cb_solver_set_kernel(cb_solver *s, int kernel);
int cb_solver_get_kernel(const cb_solver *s, int *kernel);
/* Clear the solver's sticky status bits (stream-ordered). */
int cb_solver_reset_status(cb_solver *s);
/* Test hook of the bounded waits (no counterpart in the reference): enqueue
 * one inviscid stage of the pipelined kernel in which each block's first
 * state copy is never issued and the mbarrier waits give up after a short
 * poll limit.  Every block then stores nothing, sets status bit 8
 * (reported as CB_ERR_TIMEOUT by cb_solver_sums), lets its issued copies
 * land and exits; the state and the residual carry are left unchanged.
 * CB_ERR_UNSUPPORTED for shapes that do not run the pipelined stage. */
int cb_solver_test_timeout(cb_solver *s);
int cb_solver_destroy(cb_solver *s);

/* Element-partitioned solve (one rank per GPU, the reference's partition
 * into contiguous ranges of the Hilbert element order, src/mesh.jl:499-580,
 * with the ghost exchange of its drivers once per RK stage,
 * euler2d_set2c.jl:529-594 / :707-735).  A ghosted solver advances its nelem
 * own elements; Q and the twin (and, viscous, the gradient buffer) hold
 * nghost ghost elements after them, which vmapP may name (elements nelem ..
 * nelem + nghost - 1).  Before every stage the caller fills the ghosts of the
 * state the stage reads: cb_solver_pack (what = 0) gathers own elements of
 * the current state for a neighbour rank, cb_solver_unpack (what = 0) stores
 * received elements into its ghost range [first, first + n).  The viscous
 * form (the orders with fused passes) also exchanges the gradient (what = 1)
 * between the stage's gradient pass and its stage pass
 * (cb_solver_stage_pass, pass 0 then 1); cb_solver_stage runs both passes.
 * A stage goes from the current state into the other buffer and returns the
 * new current buffer; cb_solver_settle copies a state left in the twin back
 * into Q (cb_lsrk_run and cb_solver_sums handle it themselves). */
int cb_solver_create_ghosted(cb_solver **out, int dim, int N, int precision,
                             int64_t nelem, int64_t nghost, void *Q, void *rhs,
                             const double *vgeo, const double *sgeo,
                             const int64_t *vmapM, const int64_t *vmapP,
                             const int64_t *elemtobndy, const double *D,
                             const cb_phys *phys, cb_stream_t stream);
int cb_solver_stage(cb_solver *s, int stage, double dt, void **next_in);
int cb_solver_stage_pass(cb_solver *s, int stage, double dt, int pass, void **next_in);
int cb_solver_current(const cb_solver *s, void **state);
int cb_solver_settle(cb_solver *s);
int cb_solver_pack(cb_solver *s, int what, const int64_t *elems, int64_t n, void *buf);
int cb_solver_unpack(cb_solver *s, int what, const void *buf, int64_t first, int64_t n);
/* Face-trace exchange: the minimal message of the partitioned solve.  A
 * stage reads a ghost element only at the face nodes of the faces its own
 * elements touch, so a neighbour needs Nfp·nstate values per shared face
 * (Nfp·nstate·dim for the gradient) instead of whole elements.  codes
 * (device int64, n entries) are (element << 3) | face: own elements
 * 0 .. nelem-1 for pack, ghost slots 0 .. nghost-1 for unpack; buf holds
 * n x components x Nfp values in the solver's precision (component-major
 * per entry).  Entries out of range are skipped and raise CB_ERR_MESH in the
 * status.  Stream-ordered on the solver's stream. */
int cb_solver_pack_faces(cb_solver *s, int what, const int64_t *codes, int64_t n, void *buf);
int cb_solver_unpack_faces(cb_solver *s, int what, const int64_t *codes, int64_t n, void *buf);
/* Overlap of the ghost exchange with interior work (the reference runs
 * volumerhs! while MPI receives are in flight, euler2d_set2c.jl:707-731):
 * elements 0 .. ninterior-1 must read no ghost (the caller orders its own
 * elements interior first).  cb_solver_stage_split(half = 0) runs the
 * stage for those elements, half = 1 for the others (once the ghosts of the
 * state the stage reads are filled) and then makes the other buffer
 * current; a stage split this way equals cb_solver_stage bit for bit.
 * Inviscid form, shapes whose stage runs over element ranges (the pipelined,
 * lean and tensor-core stages); CB_ERR_UNSUPPORTED otherwise. */
int cb_solver_set_split(cb_solver *s, int64_t ninterior);
int cb_solver_stage_split(cb_solver *s, int stage, double dt, int half, void **next_in);

/* ---------------------------------------------------------------------- */
/* Device-side geometry.                                                   */
/* ---------------------------------------------------------------------- */

/* vgeo and sgeo of an element mesh computed on the device in FP64: the LGL
 * grid blended from the element corners (creategrid, metric.jl:11-107), the
 * optional warp x_c += warp_amp * prod_d sin(x_d) (0: none), the metric terms
 * (computemetric, metric.jl:155-208 in 2-D and the curl-invariant form of
 * metric.jl:230-400 in 3-D) and computegeometry's vgeo / sgeo assembly
 * (euler3d_set3c.jl:210-248).  Replaces the host setup of those arrays.
 * elemtocoord is (dim, 2^dim, nelem); r, w the LGL points and weights (Nq);
 * D the derivative matrix; all device pointers.  sgeo's vMJI entry is MJI at
 * the face node of the element itself (vmapM of a conforming mesh).  The sums
 * follow the reference's order without multiply-add contraction; results
 * agree with a host evaluation to the last bits of sin and hypot. */
int cb_computegeometry(int dim, int N, int64_t nelem, const double *elemtocoord,
                       double warp_amp, const double *r, const double *w,
                       const double *D, double *vgeo, double *sgeo,
                       cb_stream_t stream);

/* Cartesian brick mesh and its connectivity on the device: the set-up
 * sequence brickmesh -> partition -> connectmesh -> mappings of the
 * reference's drivers (src/mesh.jl:259-317, :499-580, :751-956, :973-1001;
 * euler3d_set3c.jl:1689-1708) for one rank, with the same element order
 * (Hilbert code of the centroids, ties by element number) and the same
 * arrays.  n[d] elements along dimension d between the coordinates x[d]
 * (device arrays of n[d] + 1 doubles); periodic[d]; boundary (2, dim)
 * column-major codes of the non-periodic ends (NULL: all 1).  Writes the
 * device arrays elemtocoord (dim, 2^dim, nelem), elemtobndy (2 dim, nelem),
 * vmapM and vmapP ((N+1)^(dim-1), 2 dim, nelem, 1-based), nelem = prod n.
 * Asynchronous on `stream` (its scratch comes from the stream-ordered
 * allocator). */
int cb_brickmesh(int dim, int N, const int64_t *n, const double *const *x,
                 const int *periodic, const int64_t *boundary,
                 double *elemtocoord, int64_t *elemtobndy, int64_t *vmapM,
                 int64_t *vmapP, cb_stream_t stream);

/* ---------------------------------------------------------------------- */
/* Batched LSRK(5,4) over many independent instances (ensembles, serving). */
/* ---------------------------------------------------------------------- */

/* The reference advances one mesh per lowstorageRK call
 * (euler2d_set3c.jl:1109-1282); a batch advances many independent instances
 * of uneven order and element count together, each with its own dt, step
 * count and state, with the same per-instance result as cb_lsrk_run (the
 * fused stage arithmetic is the same; results do not depend on what else is
 * in the batch).  Dim 2 with N 1..8 and dim 3 with N 1..7; Euler, or LDG
 * Navier-Stokes when the batch's visc > 0 (nse2d.jl / nse3d.jl viscous
 * passes, as cb_lsrk_run with visc > 0, fused into two passes per stage).
 *
 * A cb_mesh holds what instances on the same mesh share: the geometry (the
 * caller's FP64 arrays for precision 64, rounded FP32 copies for precision 32)
 * and the int32 face-neighbour table built from vmapM/vmapP/elemtobndy.  Its
 * set-up is enqueued on `stream` without waiting for it; the validation of
 * the vmaps (CB_ERR_MESH, CB_ERR_BC) is reported by the first cb_mesh_affine
 * or cb_batch_add that uses the mesh, which waits for the set-up once.  A
 * mesh must outlive the batch instances that use it. */
typedef struct cb_mesh cb_mesh;
int cb_mesh_create(cb_mesh **out, int dim, int N, int precision,
                   int64_t nelem, const double *vgeo, const double *sgeo,
                   const int64_t *vmapM, const int64_t *vmapP,
                   const int64_t *elemtobndy, const double *D,
                   cb_stream_t stream);
/* Whether every element of the mesh is affine: its metric terms, J (MJ / M),
 * unit normals and sJ (sMJ / sM) equal their values at the first node to a
 * relative 1e-10.  cb_mesh_create then also keeps one record per element
 * (metric, J, per face normal and sJ), and the pipelined batch stage forms
 * MJ, MJI and sMJ from the LGL weights as computegeometry does
 * (euler3d_set3c.jl:222-246) instead of reading the per-node geometry. */
int cb_mesh_affine(const cb_mesh *m, int *affine);
int cb_mesh_destroy(cb_mesh *m);

/* A batch of up to max_instances slots.  All calls are ordered on `stream`
 * (0: the batch makes its own) and asynchronous except cb_batch_status and
 * cb_batch_destroy.  visc >= 0; with visc > 0 every instance is advanced by
 * the LDG Navier-Stokes stage (a gradient pass writing a batch-owned
 * (Np, nstate, dim, nelem) buffer per instance, then the fused inviscid +
 * viscous stage), variant 1 only. */
typedef struct cb_batch cb_batch;
int cb_batch_create(cb_batch **out, int precision, int max_instances,
                    const cb_phys *phys, cb_stream_t stream);
/* Stage variant used for instances of (dim, N) admitted from now on:
 * 0 = pipelined bulk-copy staging at its default occupancy (where every slab
 * is a multiple of 16 bytes: all 2-D orders, 3-D odd orders), 1 / 2 = grouped
 * staging with about 256 / 512 nodes per block, 3 / 4 = pipelined staging
 * compiled for the other occupancies (2, 3 or 4 blocks per SM), 6 = pipelined
 * staging with copies two element groups ahead instead of one, 7 = pipelined
 * staging with twice the elements per group on twice the threads (shapes
 * whose default block has at most 256 threads), 8 = pipelined staging with
 * two nodes per thread on half the threads; 5 and 9 = the affine-element
 * stage (see cb_batch_set_affine; copies two groups ahead) with one and two
 * nodes per thread; 10 = the tensor-core stage (3-D N=7, as
 * cb_solver_set_kernel 2; the default there), 11 = the lean pipelined
 * stage (cb_solver_set_kernel 4).  An affine
 * variant (5, 9) runs on meshes that allow it and falls back to the shape's
 * default per-node variant elsewhere.  A variant
 * chosen here runs as chosen; without a choice the batch uses variant 5 in
 * place of its default pipelined variant where the affine stage applies.
 * Variants that are not built for (dim, N) give CB_ERR_UNSUPPORTED.  Chosen
 * by an autotuner; the per-node pipelined variants agree bit for bit among
 * themselves, as do the grouped ones and the affine ones, and the families
 * to round-off. */
int cb_batch_set_variant(cb_batch *b, int dim, int N, int variant);
int cb_batch_get_variant(const cb_batch *b, int dim, int N, int *variant);
/* Launch configuration of a stage variant of (dim, N) in this batch's
 * precision: info[0] elements per CTA,
 * info[1] threads per CTA, info[2] nodes per thread, info[3] element groups
 * staged ahead of the work (0: grouped staging, no copies in flight),
 * info[4] resident CTAs per SM, info[5] dynamic shared memory per CTA. */
int cb_batch_variant_info(const cb_batch *b, int dim, int N, int variant, int64_t *info);
/* Whether instances admitted from now on whose mesh is affine
 * (cb_mesh_affine), with gravity 0, may use the affine-element stage: an
 * affine variant chosen by cb_batch_set_variant, or variant 5 in place of a
 * default pipelined variant.  The stage reads no vgeo / sgeo and uses each
 * element's first-node metric for all its nodes, which agrees with the
 * per-node geometry to round-off per stage.  Default: on for precision 32,
 * off for precision 64 (over hundreds of FP64 steps that round-off reaches
 * ~1e-11 relative, above the 1e-12 oracle bar). */
int cb_batch_set_affine(cb_batch *b, int on);
/* How the step graph orders the shapes present: 1 (default) = one chain per
 * shape, the chains as concurrent graph branches (kernels of different
 * shapes share the SMs); 0 = one chain, each RK stage of every shape in
 * turn, so that each persistent stage kernel has the whole GPU.  Results do
 * not depend on it. */
int cb_batch_set_concurrent(cb_batch *b, int on);
/* Admit an instance: the caller's state Q and zeroed residual carry rhs
 * (layouts as above, precision of the batch) advance by nsteps steps of dt
 * during the following cb_batch_run calls.  qref (nstate doubles, or NULL for
 * zeros) are per-field offsets as in cb_solver_set_offset (Q holds Q - qref).
 * Writes the slot id.  The batch keeps a twin state buffer from its own
 * stream-ordered pool.  Q and rhs (and the mesh's vgeo and sgeo) must be
 * 16-byte aligned: the stage copies element slabs with bulk copies. */
int cb_batch_add(cb_batch *b, const cb_mesh *m, void *Q, void *rhs, double dt,
                 int64_t nsteps, const double *qref, int *slot);
/* Advance every admitted instance by nsteps steps, each stopping at its own
 * step count; one captured CUDA graph per step (5 stage launches per
 * dimension present, 2-D and 3-D in concurrent branches). */
int cb_batch_run(cb_batch *b, int64_t nsteps);
/* Steps taken and to take by a slot (host bookkeeping, no synchronisation). */
int cb_batch_info(const cb_batch *b, int slot, int64_t *done, int64_t *target);
/* Stage variant an admitted slot runs with (the variant in effect for its
 * (dim, N) when it was admitted, after the affine rules above). */
int cb_batch_slot_variant(const cb_batch *b, int slot, int *variant);
/* Retire a slot: the instance's current state is placed in its Q (stream-
 * ordered), the twin buffer returns to the pool and the slot is free. */
int cb_batch_release(cb_batch *b, int slot);
/* Per-slot sticky status bits (out_host[max_instances]; bit 2 = non-finite
 * state); synchronises. */
int cb_batch_status(cb_batch *b, unsigned *out_host);
/* The same copy enqueued on the batch stream without synchronising (for a
 * serving loop that polls an event after it). */
int cb_batch_status_async(cb_batch *b, unsigned *out_host);
int cb_batch_destroy(cb_batch *b);

/* ---------------------------------------------------------------------- */
/* Allocation-free stage (no counterpart in the reference).                */
/* ---------------------------------------------------------------------- */

/* Size of the file-scope device array that cb_lsrk_stage_noalloc uses as
 * scratch; every GPU that loads the library holds it until the process
 * exits. */
#define CB_NOALLOC_SCRATCH_BYTES (32u * 1024u * 1024u)

/* One LSRK(5,4) stage, FP64, for callers that cannot allocate device memory
 * (an embedding whose host runtime owns every device allocation, or a path
 * where an allocation's implicit synchronisation is not allowed).  It has no
 * counterpart in the reference.  Same result as cb_volumerhs, cb_fluxrhs and
 * cb_updatesolution(rhs_gradQ = NULL, visc = 0) called in that order with the
 * same rka, rkb, dt; Q and rhs are updated in place.
 *
 * It calls no cudaMalloc/cudaFree and no allocating library routine: its
 * scratch (a copy of the stage's input state, the face-neighbour table and a
 * status word) lives in a static device array of CB_NOALLOC_SCRATCH_BYTES.
 * A mesh whose scratch need (about 8·Np·nstate + 4·2·dim bytes per element)
 * exceeds it is rejected with CB_ERR_ARG before any device work.  The first
 * call on a device looks up the array's device address (once per device, with
 * that device current); make that first call before any stream capture.
 * Every call shares the one array, so calls that overlap on the GPU (other
 * streams, other host threads) race; serialise them.  Kernel-detected
 * problems (boundary code other than 0/1, vmaps that are not a conforming
 * mesh, non-finite state, a bounded wait that gave up) are OR-ed into *status
 * when status is a non-NULL device pointer (the caller clears it), and into a
 * sticky word inside the static array when status is NULL.  The address of
 * the array is looked up once per device and kept: a process that resets a
 * device (cudaDeviceReset) must not call these entry points afterwards. */
int cb_lsrk_stage_noalloc(int dim, int N, double *Q, double *rhs,
                          const double *vgeo, const double *sgeo,
                          const int64_t *vmapM, const int64_t *vmapP,
                          const int64_t *elemtobndy, const double *D,
                          int64_t nelem, const cb_phys *phys, double rka,
                          double rkb, double dt, unsigned *status,
                          cb_stream_t stream);
/* Reads and clears, on the current device, the sticky status word that
 * cb_lsrk_stage_noalloc calls with status == NULL raise; synchronises
 * `stream`.  Writes the raw bits to *bits (if non-NULL) and returns
 * CB_ERR_BC, CB_ERR_MESH, CB_ERR_NONFINITE, CB_ERR_TIMEOUT or CB_OK.
 * Allocates nothing. */
int cb_noalloc_status(cb_stream_t stream, unsigned *bits);

#ifdef __cplusplus
}
#endif
#endif
