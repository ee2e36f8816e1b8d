// Kernel instantiations (in-place AA time steps) for storage float, compute double.
#include "launch.cuh"
BGK_INSTANTIATE_AA(float, double)
