// Kernel instantiations for dim 3, float.
#include "cb_batch.cuh"
#include "cb_ops.h"
#define DIM_ 3
#define T_ float
#include "cb_inst.inc"
