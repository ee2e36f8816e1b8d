// Kernel instantiations (reductions, outflow, initial state) for storage __nv_bfloat16 (scaled), compute float.
#include "launch.cuh"
BGK_INSTANTIATE_MISC(__nv_bfloat16, float)
