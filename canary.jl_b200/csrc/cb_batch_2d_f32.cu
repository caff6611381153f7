// Batched stage kernels for dim 2, float (see cb_batch.cuh).
#include "cb_batch.cuh"

namespace cb {
template <>
void b_fill_dim<2, float>(BKernels<float> &k) {
  b_fill<2, 2, float>(k);
  b_fill<2, 3, float>(k);
  b_fill<2, 4, float>(k);
  b_fill<2, 5, float>(k);
  b_fill<2, 6, float>(k);
  b_fill<2, 7, float>(k);
  b_fill<2, 8, float>(k);
  b_fill<2, 9, float>(k);
}
}  // namespace cb
