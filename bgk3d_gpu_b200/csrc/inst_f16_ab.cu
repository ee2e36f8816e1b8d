// Kernel instantiations (two-lattice time step) for storage __half (scaled), compute float.
#include "launch.cuh"
BGK_INSTANTIATE_AB(__half, float)
