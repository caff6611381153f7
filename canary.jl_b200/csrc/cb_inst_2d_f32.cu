// Kernel instantiations for dim 2, float.
#include "cb_batch.cuh"
#include "cb_ops.h"
#define DIM_ 2
#define T_ float
#include "cb_inst.inc"
