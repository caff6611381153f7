// Batched stage kernels for dim 2, double (see cb_batch.cuh).
#include "cb_batch.cuh"

namespace cb {
template <>
void b_fill_dim<2, double>(BKernels<double> &k) {
  b_fill<2, 2, double>(k);
  b_fill<2, 3, double>(k);
  b_fill<2, 4, double>(k);
  b_fill<2, 5, double>(k);
  b_fill<2, 6, double>(k);
  b_fill<2, 7, double>(k);
  b_fill<2, 8, double>(k);
  b_fill<2, 9, double>(k);
}
}  // namespace cb
