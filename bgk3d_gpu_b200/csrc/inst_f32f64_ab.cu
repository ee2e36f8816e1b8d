// Kernel instantiations (two-lattice time step) for storage float, compute double.
#include "launch.cuh"
BGK_INSTANTIATE_AB(float, double)
