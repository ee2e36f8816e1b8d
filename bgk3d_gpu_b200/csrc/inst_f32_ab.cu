// Kernel instantiations (two-lattice time step) for storage float, compute float.
#include "launch.cuh"
BGK_INSTANTIATE_AB(float, float)
