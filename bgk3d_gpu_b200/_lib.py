"""ctypes binding of libbgk3d_b200.so (include/bgk3d_b200.h).

The native library is the only compute path: if it is missing or cannot be
loaded, every entry point raises instead of falling back to anything else.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import (POINTER, Structure, c_char_p, c_double, c_float, c_int, c_longlong, c_size_t,
                    c_void_p)

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libbgk3d_b200.so")
DROPIN_SP_PATH = os.path.join(PKG, "libbgk3d_dropin_sp.so")
DROPIN_DP_PATH = os.path.join(PKG, "libbgk3d_dropin_dp.so")

BGK_OK = 0
BGK_ERR_ARG = -1
KIND_F64, KIND_F32, KIND_F16, KIND_BF16, KIND_F32_F64 = 0, 1, 2, 3, 4
BC_NONE, BC_DRIVEN, BC_PERIODIC, BC_CHANNEL, BC_INFLOW = -1, 0, 1, 2, 3
PATTERN_AB, PATTERN_AA = 0, 1

KIND_NAMES = {"f64": KIND_F64, "f32": KIND_F32, "f16": KIND_F16, "bf16": KIND_BF16, "f32_f64": KIND_F32_F64}
BC_NAMES = {"none": BC_NONE, "driven": BC_DRIVEN, "periodic": BC_PERIODIC, "channel": BC_CHANNEL,
            "inflow": BC_INFLOW}
# bytes per stored value of each kind
KIND_BYTES = {KIND_F64: 8, KIND_F32: 4, KIND_F16: 2, KIND_BF16: 2, KIND_F32_F64: 4}


class SweepParams(Structure):
    """Mirror of bgk_sweep_params (field order and types must match the header)."""
    _fields_ = [
        ("kind", c_int), ("bcase", c_int),
        ("l", c_int), ("m", c_int), ("n", c_int),
        ("nx", c_longlong), ("ny", c_longlong),
        ("omega", c_double), ("cte0", c_double), ("cte1", c_double),
        ("p0", c_double), ("p1", c_double), ("p2", c_double),
        ("rf", c_double), ("qf", c_double), ("tre", c_double),
        ("force_mode", c_int),
        ("fx", c_double), ("fy", c_double), ("fz", c_double),
        ("lid_force", c_double), ("u_inflow", c_double), ("inflow_cte1", c_double),
        ("scale", c_float),
        ("obs", c_void_p), ("obs_nx", c_int), ("obs_ny", c_int),
        ("imin", c_int), ("imax", c_int), ("jmin", c_int), ("jmax", c_int),
        ("kmin", c_int), ("kmax", c_int),
        ("fast", c_int),
        ("zhalo", c_int),
    ]


class BGKError(RuntimeError):
    pass


_lib = None


def lib() -> ctypes.CDLL:
    """Load (once) and return libbgk3d_b200.so; raises if it is not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise BGKError(f"{LIB_PATH} is missing: build it with bgk3d_gpu_b200.build.build() "
                       "(there is no fallback path)")
    L = ctypes.CDLL(LIB_PATH)
    P = POINTER(SweepParams)
    L.bgk_sweep_params_init.argtypes = [P, c_int, c_int, c_int, c_int, c_double]
    L.bgk_sweep_params_init.restype = None
    L.bgk_sweep.argtypes = [P, POINTER(c_void_p), POINTER(c_void_p), c_void_p]
    L.bgk_sweep.restype = c_int
    L.bgk_reduce_workspace_bytes.argtypes = [c_int, c_int, c_int]
    L.bgk_reduce_workspace_bytes.restype = c_size_t
    L.bgk_moments.argtypes = [P, POINTER(c_void_p), c_void_p, c_void_p, c_size_t, c_void_p]
    L.bgk_moments.restype = c_int
    L.bgk_dissipation_workspace_bytes.argtypes = [c_int, c_int, c_int]
    L.bgk_dissipation_workspace_bytes.restype = c_size_t
    L.bgk_dissipation.argtypes = [P, POINTER(c_void_p), c_double, c_void_p, c_void_p, c_size_t, c_void_p]
    L.bgk_dissipation.restype = c_int
    L.bgk_moments_noalloc.argtypes = [P, POINTER(c_void_p), c_void_p, c_void_p]
    L.bgk_moments_noalloc.restype = c_int
    L.bgk_moments_noalloc_max_bytes.argtypes = []
    L.bgk_moments_noalloc_max_bytes.restype = c_size_t
    L.bgk_sweep_moments_workspace_bytes.argtypes = [P]
    L.bgk_sweep_moments_workspace_bytes.restype = c_size_t
    L.bgk_sweep_moments.argtypes = [P, POINTER(c_void_p), POINTER(c_void_p), c_void_p, c_void_p, c_size_t,
                                    c_void_p]
    L.bgk_sweep_moments.restype = c_int
    L.bgk_draglift.argtypes = [P, POINTER(c_void_p), c_int, c_int, c_int, c_int, c_int, c_int,
                               c_void_p, c_void_p, c_size_t, c_void_p]
    L.bgk_draglift.restype = c_int
    L.bgk_profile.argtypes = [P, POINTER(c_void_p), c_int, c_int, c_int, c_void_p, c_void_p]
    L.bgk_profile.restype = c_int
    L.bgk_probe.argtypes = [P, POINTER(c_void_p), c_int, c_int, c_int, c_void_p, c_void_p]
    L.bgk_probe.restype = c_int
    L.bgk_slice.argtypes = [P, POINTER(c_void_p), c_int, c_int, c_void_p, c_void_p]
    L.bgk_slice.restype = c_int
    L.bgk_device_sync.argtypes = []
    L.bgk_device_sync.restype = c_int
    L.bgk_last_error.argtypes = []
    L.bgk_last_error.restype = c_char_p
    L.bgk_version.argtypes = []
    L.bgk_version.restype = c_char_p
    L.bgk_set_obstacle_split.argtypes = [c_int]
    L.bgk_set_obstacle_split.restype = c_int
    L.bgk_set_pair_kernels.argtypes = [c_int]
    L.bgk_set_pair_kernels.restype = c_int
    L.bgk_abi_struct_size.argtypes = [c_int]
    L.bgk_abi_struct_size.restype = c_size_t
    L.bgk_abi_field_offset.argtypes = [c_int, c_int]
    L.bgk_abi_field_offset.restype = c_longlong
    _bind_lattice(L)
    _lib = L
    return L


def _bind_lattice(L: ctypes.CDLL) -> None:
    """Bind the lattice / batch / server entry points when the library has them."""
    if not hasattr(L, "bgk_lattice_create"):
        return
    from . import _lattice_abi
    _lattice_abi.bind(L)


def check(rc: int, what: str = "") -> None:
    if rc != BGK_OK:
        msg = lib().bgk_last_error().decode(errors="replace")
        raise BGKError(f"{what} failed ({rc}): {msg}")


def ptr_array(ptrs) -> ctypes.Array:
    arr = (c_void_p * 19)()
    for d, p in enumerate(ptrs):
        arr[d] = p
    return arr


def sweep_params(kind: int, l: int, m: int, n: int, omega: float, **kw) -> SweepParams:
    p = SweepParams()
    lib().bgk_sweep_params_init(ctypes.byref(p), int(kind), int(l), int(m), int(n), float(omega))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown sweep parameter {k}")
        setattr(p, k, v)
    return p


def load_dropin(double: bool) -> ctypes.CDLL:
    """Load the reference-named drop-in library (real_t = double or float)."""
    path = DROPIN_DP_PATH if double else DROPIN_SP_PATH
    if not os.path.exists(path):
        raise BGKError(f"{path} is missing: build it with bgk3d_gpu_b200.build.build()")
    lib()  # dependency first
    D = ctypes.CDLL(path)
    real = c_double if double else c_float
    D.col_mc_gpu.argtypes = [c_void_p] * 37 + [c_int] * 5 + [real] * 12
    D.col_mc_gpu.restype = None
    pa = POINTER(c_void_p)
    D.bcond_periodic_gpu.argtypes = [pa, c_int, c_int, c_int, c_int, c_int]
    D.bcond_channel_gpu.argtypes = [pa, c_int, c_int, c_int, c_int, c_int]
    D.bcond_driven_gpu.argtypes = [pa, c_int, c_int, c_int, c_int, c_int, real]
    D.bcond_inflow_gpu.argtypes = [pa, c_int, c_int, c_int, c_int, c_int] + [real] * 7
    D.bcond_obs_gpu.argtypes = [pa, c_void_p] + [c_int] * 13
    D.gpu_device_sync.argtypes = []
    D.bgk_dropin_track_moments.argtypes = [c_int]
    D.bgk_dropin_track_moments.restype = None
    D.bgk_dropin_moments.argtypes = [c_void_p, c_void_p]
    D.bgk_dropin_moments.restype = c_int
    D.bgk_dropin_moments_ptr.argtypes = []
    D.bgk_dropin_moments_ptr.restype = c_void_p
    D.bgk_dropin_moments_to.argtypes = [c_void_p]
    D.bgk_dropin_moments_to.restype = None
    for f in ("bcond_periodic_gpu", "bcond_channel_gpu", "bcond_driven_gpu", "bcond_inflow_gpu",
              "bcond_obs_gpu", "gpu_device_sync", "bgk_dropin_reset", "bgk_dropin_track_moments"):
        getattr(D, f).restype = None
    return D
