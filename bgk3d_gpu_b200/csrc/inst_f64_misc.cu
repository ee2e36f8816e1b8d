// Kernel instantiations (reductions, outflow, initial state) for storage double, compute double.
#include "launch.cuh"
BGK_INSTANTIATE_MISC(double, double)
