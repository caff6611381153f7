// Batched stage kernels for dim 3, double (see cb_batch.cuh).
#include "cb_batch.cuh"

namespace cb {
template <>
void b_fill_dim<3, double>(BKernels<double> &k) {
  b_fill<3, 2, double>(k);
  b_fill<3, 3, double>(k);
  b_fill<3, 4, double>(k);
  b_fill<3, 5, double>(k);
  b_fill<3, 6, double>(k);
  b_fill<3, 7, double>(k);
  b_fill<3, 8, double>(k);
}
}  // namespace cb
