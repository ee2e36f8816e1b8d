// Kernel instantiations (reductions, outflow, initial state) for storage float, compute float.
#include "launch.cuh"
BGK_INSTANTIATE_MISC(float, float)
