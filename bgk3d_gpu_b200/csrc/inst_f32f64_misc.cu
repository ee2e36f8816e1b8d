// Kernel instantiations (reductions, outflow, initial state) for storage float, compute double.
#include "launch.cuh"
BGK_INSTANTIATE_MISC(float, double)
