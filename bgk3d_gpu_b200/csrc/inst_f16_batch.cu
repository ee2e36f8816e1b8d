// Kernel instantiations (batched time step) for storage __half (scaled), compute float.
#include "launch.cuh"
BGK_INSTANTIATE_BATCH(__half, float)
