// Kernel instantiations (reductions, outflow, initial state) for storage __half (scaled), compute float.
#include "launch.cuh"
BGK_INSTANTIATE_MISC(__half, float)
