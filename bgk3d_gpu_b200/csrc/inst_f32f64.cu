// Kernel instantiations for storage float, compute double.
#include "launch.cuh"
BGK_INSTANTIATE(float, double)
