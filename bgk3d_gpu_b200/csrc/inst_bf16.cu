// Kernel instantiations for storage __nv_bfloat16, compute float.
#include "launch.cuh"
BGK_INSTANTIATE(__nv_bfloat16, float)
