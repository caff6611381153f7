// Kernel instantiations for dim 3, double.
#include "cb_batch.cuh"
#include "cb_ops.h"
#define DIM_ 3
#define T_ double
#include "cb_inst.inc"
