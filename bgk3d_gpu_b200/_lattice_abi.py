"""ctypes signatures of the library-owned lattice entry points (include/bgk3d_lattice.h)."""
from __future__ import annotations

import ctypes

from ctypes import (POINTER, Structure, c_double, c_float, c_int, c_longlong, c_size_t, c_void_p)


class LatticeDesc(Structure):
    """Mirror of bgk_lattice_desc."""
    _fields_ = [
        ("kind", c_int), ("bcase", c_int), ("pattern", c_int),
        ("l", c_int), ("m", c_int), ("n", c_int),
        ("omega", c_double),
        ("force_mode", c_int), ("fx", c_double), ("fy", c_double), ("fz", c_double),
        ("lid_force", c_double), ("u_inflow", c_double),
        ("scale", c_float),
        ("fast", c_int),
    ]


def bind_batch(L) -> None:
    from ctypes import POINTER as P_
    L.bgk_batch_create.argtypes = [P_(c_void_p), c_int, P_(c_void_p)]
    L.bgk_batch_create.restype = c_int
    L.bgk_batch_destroy.argtypes = [c_void_p]
    L.bgk_batch_destroy.restype = c_int
    L.bgk_batch_resync.argtypes = [c_void_p]
    L.bgk_batch_resync.restype = c_int
    L.bgk_batch_step.argtypes = [c_void_p, c_int, c_void_p]
    L.bgk_batch_step.restype = c_int
    L.bgk_batch_set_config.argtypes = [c_void_p, c_int, c_int]
    L.bgk_batch_set_config.restype = c_int
    L.bgk_batch_set_chunk.argtypes = [c_void_p, c_int]
    L.bgk_batch_set_chunk.restype = c_int
    L.bgk_batch_get_chunk.argtypes = [c_void_p, P_(c_int)]
    L.bgk_batch_get_chunk.restype = c_int
    L.bgk_batch_set_solo.argtypes = [c_void_p, c_longlong]
    L.bgk_batch_set_solo.restype = c_int
    L.bgk_batch_get_solo.argtypes = [c_void_p]
    L.bgk_batch_get_solo.restype = c_longlong
    L.bgk_batch_groups.argtypes = [c_void_p]
    L.bgk_batch_groups.restype = c_int
    L.bgk_batch_get_config.argtypes = [c_void_p, P_(c_int), P_(c_int)]
    L.bgk_batch_get_config.restype = c_int
    L.bgk_batch_tune.argtypes = [c_void_p, c_int, c_void_p, P_(c_int)]
    L.bgk_batch_tune.restype = c_int
    L.bgk_batch_nodes.argtypes = [c_void_p]
    L.bgk_batch_nodes.restype = c_longlong
    L.bgk_batch_tiles.argtypes = [c_void_p]
    L.bgk_batch_tiles.restype = c_longlong


def bind(L) -> None:
    bind_batch(L)
    D = POINTER(LatticeDesc)
    L.bgk_lattice_desc_init.argtypes = [D, c_int, c_int, c_int, c_int, c_int, c_double]
    L.bgk_lattice_desc_init.restype = None
    L.bgk_lattice_device_bytes.argtypes = [D]
    L.bgk_lattice_device_bytes.restype = c_size_t
    L.bgk_lattice_create.argtypes = [D, POINTER(c_void_p)]
    L.bgk_lattice_create.restype = c_int
    L.bgk_lattice_destroy.argtypes = [c_void_p]
    L.bgk_lattice_destroy.restype = c_int
    L.bgk_lattice_destroy_async.argtypes = [c_void_p, c_void_p]
    L.bgk_lattice_destroy_async.restype = c_int
    L.bgk_lattice_set_obstacle.argtypes = [c_void_p, c_void_p]
    L.bgk_lattice_set_obstacle.restype = c_int
    L.bgk_lattice_save.argtypes = [c_void_p, ctypes.c_char_p, c_int, c_int, c_void_p]
    L.bgk_lattice_save.restype = c_int
    L.bgk_lattice_restore.argtypes = [c_void_p, ctypes.c_char_p, ctypes.POINTER(c_int), c_void_p]
    L.bgk_lattice_restore.restype = c_int
    L.bgk_io_set_subrecord_limit.argtypes = [ctypes.c_longlong]
    L.bgk_io_set_subrecord_limit.restype = ctypes.c_longlong
    L.bgk_lattice_profile.argtypes = [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]
    L.bgk_lattice_profile.restype = c_int
    L.bgk_lattice_probe.argtypes = [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p]
    L.bgk_lattice_probe.restype = c_int
    L.bgk_lattice_slice.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p]
    L.bgk_lattice_slice.restype = c_int
    L.bgk_lattice_uses_tma.argtypes = [c_void_p]
    L.bgk_lattice_uses_tma.restype = c_int
    L.bgk_set_tma_kernels.argtypes = [c_int]
    L.bgk_set_tma_kernels.restype = c_int
    L.bgk_lattice_status.argtypes = [c_void_p]
    L.bgk_lattice_status.restype = c_int
    L.bgk_lattice_set_sphere.argtypes = [c_void_p, c_double, c_double, c_double, c_double]
    L.bgk_lattice_set_sphere.restype = c_int
    L.bgk_lattice_set_zhalo.argtypes = [c_void_p, c_int]
    L.bgk_lattice_set_zhalo.restype = c_int
    L.bgk_lattice_plane.argtypes = [c_void_p, c_int, c_int, POINTER(c_void_p), POINTER(c_size_t)]
    L.bgk_lattice_plane.restype = c_int
    L.bgk_set_retained_bytes.argtypes = [c_size_t]
    L.bgk_set_retained_bytes.restype = c_int
    L.bgk_trim_memory.argtypes = []
    L.bgk_trim_memory.restype = c_int
    L.bgk_lattice_init.argtypes = [c_void_p, c_int, c_void_p, c_void_p]
    L.bgk_lattice_init.restype = c_int
    L.bgk_lattice_load.argtypes = [c_void_p, c_void_p, c_void_p]
    L.bgk_lattice_load.restype = c_int
    L.bgk_lattice_store.argtypes = [c_void_p, c_void_p, c_void_p]
    L.bgk_lattice_store.restype = c_int
    L.bgk_lattice_step.argtypes = [c_void_p, c_int, c_void_p]
    L.bgk_lattice_step.restype = c_int
    L.bgk_lattice_prepare.argtypes = [c_void_p]
    L.bgk_lattice_prepare.restype = c_int
    L.bgk_lattice_step_moments.argtypes = [c_void_p, c_int, c_int, c_void_p, c_void_p]
    L.bgk_lattice_step_moments.restype = c_int
    L.bgk_lattice_set_omega.argtypes = [c_void_p, c_double]
    L.bgk_lattice_set_omega.restype = c_int
    L.bgk_lattice_moments.argtypes = [c_void_p, c_void_p, c_void_p]
    L.bgk_lattice_moments.restype = c_int
    L.bgk_lattice_dissipation.argtypes = [c_void_p, c_double, c_void_p, c_void_p]
    L.bgk_lattice_dissipation.restype = c_int
    L.bgk_lattice_draglift.argtypes = [c_void_p] + [c_int] * 6 + [c_void_p, c_void_p]
    L.bgk_lattice_draglift.restype = c_int
    L.bgk_lattice_steps.argtypes = [c_void_p]
    L.bgk_lattice_steps.restype = c_longlong
    L.bgk_lattice_arrays.argtypes = [c_void_p, POINTER(c_void_p), POINTER(c_longlong), POINTER(c_longlong)]
    L.bgk_lattice_arrays.restype = c_int
