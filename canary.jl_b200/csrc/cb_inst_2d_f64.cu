// Kernel instantiations for dim 2, double.
#include "cb_batch.cuh"
#include "cb_ops.h"
#define DIM_ 2
#define T_ double
#include "cb_inst.inc"
