"""bgk3d_gpu_b200: B200-native (sm_100a) D3Q19 BGK time-step hot path.

Native libraries (built by bgk3d_gpu_b200.build):
  libbgk3d_b200.so       C ABI of include/bgk3d_b200.h
  libbgk3d_dropin_*.so   the reference's own symbol names (include/bgk3d_dropin.h)
"""
from ._lib import (BC_CHANNEL, BC_DRIVEN, BC_INFLOW, BC_NONE, BC_PERIODIC, KIND_BF16, KIND_F16,
                   KIND_F32, KIND_F32_F64, KIND_F64, BGKError, lib, load_dropin, sweep_params)

__all__ = ["lib", "load_dropin", "sweep_params", "BGKError", "KIND_F64", "KIND_F32", "KIND_F16",
           "KIND_BF16", "KIND_F32_F64", "BC_NONE", "BC_DRIVEN", "BC_PERIODIC", "BC_CHANNEL",
           "BC_INFLOW"]
__version__ = "0.1.0"
