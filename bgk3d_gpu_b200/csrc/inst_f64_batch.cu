// Kernel instantiations (batched time step) for storage double, compute double.
#include "launch.cuh"
BGK_INSTANTIATE_BATCH(double, double)
