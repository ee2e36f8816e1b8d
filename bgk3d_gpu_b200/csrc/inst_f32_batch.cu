// Kernel instantiations (batched time step) for storage float, compute float.
#include "launch.cuh"
BGK_INSTANTIATE_BATCH(float, float)
