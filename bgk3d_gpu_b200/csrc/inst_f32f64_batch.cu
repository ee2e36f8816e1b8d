// Kernel instantiations (batched time step) for storage float, compute double.
#include "launch.cuh"
BGK_INSTANTIATE_BATCH(float, double)
