// Kernel instantiations (in-place AA time steps) for storage double, compute double.
#include "launch.cuh"
BGK_INSTANTIATE_AA(double, double)
