// Kernel instantiations (batched time step) for storage __nv_bfloat16 (scaled), compute float.
#include "launch.cuh"
BGK_INSTANTIATE_BATCH(__nv_bfloat16, float)
