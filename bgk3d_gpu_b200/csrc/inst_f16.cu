// Kernel instantiations for storage __half, compute float.
#include "launch.cuh"
BGK_INSTANTIATE(__half, float)
