"""CPU checks of the boundary: the shared libraries load, export every symbol
the headers in include/ declare, and reject invalid arguments before touching
the device."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "bgk3d_gpu_b200")


def declared(header):
    txt = open(os.path.join(ROOT, "include", header)).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    names = re.findall(r"\b([a-z_][a-z0-9_]*)\s*\(", txt)
    skip = {"if", "defined", "sizeof", "return"}
    return sorted({n for n in names if n not in skip and not n.startswith("__")})


def exported(path):
    import subprocess
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    return {line.split()[-1] for line in out.splitlines() if " T " in line}


@pytest.fixture(scope="module")
def built():
    from bgk3d_gpu_b200 import build
    return build.build()


def test_main_library_exports_header(built):
    syms = exported(os.path.join(PKG, "libbgk3d_b200.so"))
    missing = [n for n in declared("bgk3d_b200.h") if n not in syms]
    assert not missing, missing
    for h in ("bgk3d_lattice.h",):
        if os.path.exists(os.path.join(ROOT, "include", h)):
            missing = [n for n in declared(h) if n not in syms]
            assert not missing, (h, missing)


@pytest.mark.parametrize("lib", ["libbgk3d_dropin_sp.so", "libbgk3d_dropin_dp.so"])
def test_dropin_library_exports_reference_names(built, lib):
    syms = exported(os.path.join(PKG, lib))
    want = declared("bgk3d_dropin.h")
    assert {"col_mc_gpu", "bcond_periodic_gpu", "bcond_channel_gpu", "bcond_driven_gpu",
            "bcond_inflow_gpu", "bcond_obs_gpu", "gpu_device_sync"} <= set(want)
    missing = [n for n in want if n not in syms]
    assert not missing, missing
    ctypes.CDLL(os.path.join(PKG, lib))


def test_invalid_arguments_rejected_without_device(built):
    from bgk3d_gpu_b200 import _lib
    L = _lib.lib()
    dummy = _lib.ptr_array([1] * 19)
    cases = [dict(kind=9), dict(bcase=7), dict(l=0), dict(nx=3), dict(kind=2, scale=3.0)]
    for kw in cases:
        p = _lib.sweep_params(1, 8, 8, 8, 1.0)
        for k, v in kw.items():
            setattr(p, k, v)
        rc = L.bgk_sweep(ctypes.byref(p), dummy, dummy, None)
        assert rc == _lib.BGK_ERR_ARG if hasattr(_lib, "BGK_ERR_ARG") else rc == -1, kw
        assert L.bgk_last_error().decode()
    # obstacle touching a face
    import numpy as np
    obs = np.zeros(8 * 8 * 8, np.int32)
    p = _lib.sweep_params(1, 8, 8, 8, 1.0, obs=obs.ctypes.data, imin=1, imax=3, jmin=2, jmax=3,
                          kmin=2, kmax=3)
    assert L.bgk_sweep(ctypes.byref(p), dummy, dummy, None) == -1
    assert "inside" in L.bgk_last_error().decode()


def test_workspace_query(built):
    from bgk3d_gpu_b200 import _lib
    L = _lib.lib()
    assert L.bgk_reduce_workspace_bytes(256, 256, 256) >= 5 * 8
    assert L.bgk_version().decode().startswith("bgk3d_b200")


def test_struct_mirrors_match_the_library():
    """The ctypes mirrors of bgk_sweep_params and bgk_lattice_desc have the
    size the library was compiled with (a field added on one side only
    would shift every field after it).  A pure host call: no GPU needed."""
    import ctypes
    from bgk3d_gpu_b200._lib import SweepParams, lib
    from bgk3d_gpu_b200._lattice_abi import LatticeDesc
    L = lib()
    assert L.bgk_abi_struct_size(0) == ctypes.sizeof(SweepParams)
    assert L.bgk_abi_struct_size(1) == ctypes.sizeof(LatticeDesc)
    assert L.bgk_abi_struct_size(7) == 0


def test_struct_mirror_fields_sit_where_the_library_has_them():
    """Every field of the ctypes mirrors, in declaration order, at the byte
    offset the library was compiled with: two swapped fields of equal total
    size, or a field moved into a padding hole, would pass the size check
    and shift the values the kernels read."""
    from bgk3d_gpu_b200._lib import SweepParams, lib
    from bgk3d_gpu_b200._lattice_abi import LatticeDesc
    L = lib()
    for which, mirror in ((0, SweepParams), (1, LatticeDesc)):
        fields = [getattr(mirror, name) for name, _ in mirror._fields_]
        for idx, f in enumerate(fields):
            assert L.bgk_abi_field_offset(which, idx) == f.offset, (mirror.__name__, mirror._fields_[idx][0])
        assert L.bgk_abi_field_offset(which, len(fields)) == -1
    assert L.bgk_abi_field_offset(5, 0) == -1
