// Kernel instantiations (in-place AA time steps) for storage float, compute float.
#include "launch.cuh"
BGK_INSTANTIATE_AA(float, float)
