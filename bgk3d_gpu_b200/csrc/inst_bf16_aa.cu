// Kernel instantiations (in-place AA time steps) for storage __nv_bfloat16 (scaled), compute float.
#include "launch.cuh"
BGK_INSTANTIATE_AA(__nv_bfloat16, float)
