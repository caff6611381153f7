// Batched stage kernels for dim 3, float (see cb_batch.cuh).
#include "cb_batch.cuh"

namespace cb {
template <>
void b_fill_dim<3, float>(BKernels<float> &k) {
  b_fill<3, 2, float>(k);
  b_fill<3, 3, float>(k);
  b_fill<3, 4, float>(k);
  b_fill<3, 5, float>(k);
  b_fill<3, 6, float>(k);
  b_fill<3, 7, float>(k);
  b_fill<3, 8, float>(k);
}
}  // namespace cb
