// Kernel instantiations for storage float, compute float.
#include "launch.cuh"
BGK_INSTANTIATE(float, float)
