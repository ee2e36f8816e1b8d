// Kernel instantiations (two-lattice time step) for storage __nv_bfloat16 (scaled), compute float.
#include "launch.cuh"
BGK_INSTANTIATE_AB(__nv_bfloat16, float)
