// Kernel instantiations (two-lattice time step) for storage double, compute double.
#include "launch.cuh"
BGK_INSTANTIATE_AB(double, double)
