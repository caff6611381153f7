// Host-side table of launchers for one (dim, precision, order).
#pragma once
#include "cb_dg.cuh"

namespace cb {

constexpr int MAXN = 10;  // orders 1..MAXN are compiled for dim 2 and 3

template <typename T>
struct BDesc;

template <typename T>
struct Ops {
  int Np, Nfp, epb, threads;
  size_t smem_stage;
  // sets the dynamic shared-memory limits of every kernel of this order
  cudaError_t (*prepare)();
  cudaError_t (*volumerhs)(T *, const T *, const T *, const T *, int64_t, const PhysT<T> &, cudaStream_t);
  cudaError_t (*fluxrhs)(T *, const T *, const T *, const T *, int64_t, const int64_t *,
                         const int64_t *, const int64_t *, const PhysT<T> &, unsigned *, cudaStream_t);
  cudaError_t (*stage)(const T *, T *, T *, const T *, const T *, const int32_t *, const T *, int64_t,
                       const PhysT<T> &, const Offs<T, 5> &, T, T, unsigned *, cudaStream_t);
  // the stage with, after the stream: the timeout test hook flag (each
  // block's first state copy withheld and a short wait limit;
  // cudaErrorNotSupported where no pipelined stage runs), the kernel choice
  // (0 the shape's default, 1 the CUDA-core stages, 2 the tensor-core stage;
  // cudaErrorNotSupported where the choice is not built) and the first
  // element of the launch (elements first .. nelem - 1)
  cudaError_t (*stage_k)(const T *, T *, T *, const T *, const T *, const int32_t *, const T *, int64_t,
                         const PhysT<T> &, const Offs<T, 5> &, T, T, unsigned *, cudaStream_t, int, int, int64_t);
  // whether stage_k takes a first element > 0 (an element range) for arrays
  // aligned like these: (Qin, rhs, vgeo, sgeo)
  bool (*ranged)(const void *, const void *, const void *, const void *);
  bool mma;          // whether the tensor-core stage is built for this shape
  bool mma_default;  // whether it is the shape's default stage kernel
  bool lean;         // whether the lean pipelined stage is built for this shape
  int default_kernel;  // the stage kernel choice 0 resolves to (1 to 4)
  cudaError_t (*build_nbr)(int32_t *, const int64_t *, const int64_t *, const int64_t *, int64_t,
                           unsigned *, cudaStream_t);
  // the same with neighbours allowed up to a total element count (ghosts)
  cudaError_t (*build_nbr_ghost)(int32_t *, const int64_t *, const int64_t *, const int64_t *, int64_t,
                                 int64_t, unsigned *, cudaStream_t);
  cudaError_t (*volume_grad)(T *, const T *, const T *, const T *, int64_t, const PhysT<T> &, cudaStream_t);
  cudaError_t (*flux_grad)(T *, const T *, const T *, const T *, int64_t, const int64_t *,
                           const int64_t *, const int64_t *, const PhysT<T> &, unsigned *, cudaStream_t);
  cudaError_t (*volume_div)(T *, const T *, const T *, const T *, const T *, int64_t, const PhysT<T> &,
                            cudaStream_t);
  cudaError_t (*flux_div)(T *, const T *, const T *, const T *, int64_t, const int64_t *, const int64_t *,
                          const int64_t *, const PhysT<T> &, unsigned *, cudaStream_t);
  // order-independent element-wise kernels
  cudaError_t (*update)(T *, const T *, T *, const T *, int64_t, int, T, T, T, T, cudaStream_t);
  cudaError_t (*update_gradQ)(T *, const T *, const T *, int64_t, int, cudaStream_t);
  cudaError_t (*cons_sums)(const T *, const T *, int64_t, int, const Offs<double, 5> &, double *, int,
                           cudaStream_t);
  // fused viscous passes over one mesh (pass 0: gradient, 1: stage + update);
  // nullptr for orders whose groups would need more than two nodes per thread
  // pass 0 (gradient) or 1 (stage) of the fused viscous form; the last
  // argument is the solver's kernel choice (3: the grouped stage pass)
  cudaError_t (*ns_pass)(int, const BDesc<T> &, T *, int64_t, const PhysT<T> &, T, T, cudaStream_t, int);
};

// Defined in cb_inst_<dim>d_<prec>.cu; nullptr when N is outside 1..MAXN.
template <int DIM, typename T>
const Ops<T> *get_ops(int N);

cudaError_t round_to_f32(float *dst, const double *src, int64_t n, cudaStream_t st);

}  // namespace cb
