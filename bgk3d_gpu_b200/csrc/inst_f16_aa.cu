// Kernel instantiations (in-place AA time steps) for storage __half (scaled), compute float.
#include "launch.cuh"
BGK_INSTANTIATE_AA(__half, float)
