// Kernel instantiations for storage double, compute double.
#include "launch.cuh"
BGK_INSTANTIATE(double, double)
