"""CPU oracle (test infrastructure only): Python side of oracle/bgk_oracle.cpp.

Holds a lattice exactly as the reference does -- 19 "a" arrays and 18 "b"
arrays (pop 19 in place), each (0:l+1+ipad, 0:m+1+jpad, 0:n+1) with i fastest
(SRC/alloca.F90:153-191) -- and advances it the way SRC/bgk3d.F90:169-179
does: boundaries (SRC/boundaries.F90:31-47), col_MC, pointer swap
(SRC/col_MC.F90:539-596).  Only tests/, __graft_entry__.smoke() and bench.py's
CPU baseline use this module; the product path never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_double, c_float, c_int, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

KIND_F64, KIND_F32, KIND_F16, KIND_BF16, KIND_F32_F64 = 0, 1, 2, 3, 4
BC_DRIVEN, BC_PERIODIC, BC_CHANNEL, BC_INFLOW = 0, 1, 2, 3
# numpy dtype used to hold each storage kind (16-bit kinds as raw bits)
STORAGE_DTYPE = {KIND_F64: np.float64, KIND_F32: np.float32, KIND_F16: np.uint16,
                 KIND_BF16: np.uint16, KIND_F32_F64: np.float32}
COMPUTE_DTYPE = {KIND_F64: np.float64, KIND_F32: np.float32, KIND_F16: np.float32,
                 KIND_BF16: np.float32, KIND_F32_F64: np.float64}

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        pp = POINTER(c_void_p)
        fp = POINTER(c_float)
        dp = POINTER(c_double)
        L.orc_bcond.argtypes = [c_int, c_int, pp, c_int, c_int, c_int, c_int, c_int, c_double,
                                c_double, c_double, fp]
        L.orc_bcond_obs.argtypes = [c_int, pp, c_void_p] + [c_int] * 11 + [fp]
        L.orc_col_mc.argtypes = [c_int, pp, pp, c_int, c_int, c_int, c_int, c_int, c_double,
                                 c_double, c_int, c_double, c_double, c_double, fp, c_int]
        L.orc_diagno.argtypes = [c_int, pp, c_int, c_int, c_int, c_int, c_int, c_void_p, c_double,
                                 fp, dp]
        L.orc_draglift.argtypes = [c_int, pp, c_void_p] + [c_int] * 11 + [fp, dp]
        L.orc_profile.argtypes = [c_int, pp] + [c_int] * 8 + [c_double, fp, dp]
        L.orc_probe.argtypes = [c_int, pp] + [c_int] * 5 + [c_double, fp, dp]
        L.orc_slice.argtypes = [c_int, pp] + [c_int] * 7 + [fp, fp]
        L.orc_dissipation.argtypes = [c_int, pp] + [c_int] * 5 + [c_void_p] + [c_double] * 9 + [fp, dp]
        L.orc_enstrophy.argtypes = [c_int, pp] + [c_int] * 5 + [c_void_p, c_double, c_int, fp, dp]
        L.orc_init.argtypes = [c_int, pp] + [c_int] * 6 + [dp] + [c_double] * 6 + [fp]
        L.orc_float_to_half.argtypes = [c_float]
        L.orc_float_to_half.restype = ctypes.c_uint16
        L.orc_half_to_float.argtypes = [ctypes.c_uint16]
        L.orc_half_to_float.restype = c_float
        L.orc_float_to_bf16.argtypes = [c_float]
        L.orc_float_to_bf16.restype = ctypes.c_uint16
        L.orc_bf16_to_float.argtypes = [ctypes.c_uint16]
        L.orc_bf16_to_float.restype = c_float
        L.orc_max_threads.restype = c_int
        _lib = L
    return _lib


def _ptrs(planes) -> ctypes.Array:
    arr = (c_void_p * 19)()
    for d, p in enumerate(planes):
        arr[d] = p.ctypes.data
    return arr


def omega_from_visc(svisc: float, kind: int) -> float:
    """SRC/hencol.F90:31, omega = 2/(6 nu + 1), evaluated in the compute type."""
    C = COMPUTE_DTYPE[kind]
    nu = C(svisc)
    return float(C(C(2.0) / (C(6.0) * nu + C(1.0))))


class OracleLattice:
    """Reference-layout lattice advanced by the C restatement."""

    def __init__(self, l, m, n, kind=KIND_F64, ipad=0, jpad=0, scale=1.0, nthreads=None):
        self.l, self.m, self.n, self.kind = l, m, n, kind
        self.nx, self.ny, self.nz = l + 2 + ipad, m + 2 + jpad, n + 2
        dt = STORAGE_DTYPE[kind]
        self.a = [np.zeros((self.nz, self.ny, self.nx), dt) for _ in range(19)]
        self.b = [np.zeros((self.nz, self.ny, self.nx), dt) for _ in range(18)]
        self.scale = (c_float * 2)(scale, 1.0 / scale)
        self.nthreads = nthreads or max(1, lib().orc_max_threads())
        self.obs = None
        self.bbox = None

    # -- state ------------------------------------------------------------
    def set_state(self, arr19: np.ndarray) -> None:
        """arr19: (19, nz, ny, nx) in the storage dtype (copied)."""
        for d in range(19):
            self.a[d][...] = arr19[d]
        for d in range(18):
            self.b[d][...] = arr19[d]

    def state(self) -> np.ndarray:
        return np.stack([p.copy() for p in self.a])

    def set_obstacle(self, obs: np.ndarray) -> None:
        """obs: int32 (n, m, l) [k, j, i] with 1 = solid; bbox computed here."""
        self.obs = np.ascontiguousarray(obs, dtype=np.int32)
        ks, js, is_ = np.nonzero(self.obs == 1)
        if len(is_) == 0:
            self.bbox = None
        else:
            self.bbox = (int(is_.min()) + 1, int(is_.max()) + 1, int(js.min()) + 1,
                         int(js.max()) + 1, int(ks.min()) + 1, int(ks.max()) + 1)

    # -- one reference time step -----------------------------------------
    def bcond(self, bcase, force=0.0, u_inflow=0.0, inflow_cte1=0.0):
        rc = lib().orc_bcond(self.kind, bcase, _ptrs(self.a), self.l, self.m, self.n, self.nx,
                             self.ny, force, u_inflow, inflow_cte1, self.scale)
        assert rc == 0

    def bcond_obs(self):
        if self.obs is None or self.bbox is None:
            return
        rc = lib().orc_bcond_obs(self.kind, _ptrs(self.a), self.obs.ctypes.data, self.l, self.m,
                                 self.n, self.nx, self.ny, *self.bbox, self.scale)
        assert rc == 0

    def col_mc(self, omega, cte1=1.0, force_mode=0, fx=0.0, fy=0.0, fz=0.0):
        bptr = list(self.b) + [self.a[18]]
        rc = lib().orc_col_mc(self.kind, _ptrs(self.a), _ptrs(bptr), self.l, self.m, self.n,
                              self.nx, self.ny, omega, cte1, force_mode, fx, fy, fz, self.scale,
                              self.nthreads)
        assert rc == 0

    def swap(self):
        for d in range(18):
            self.a[d], self.b[d] = self.b[d], self.a[d]

    def step(self, bcase, omega, nsteps=1, force=0.0, u_inflow=0.0, inflow_cte1=0.0, cte1=1.0,
             force_mode=0, fx=0.0, fy=0.0, fz=0.0):
        for _ in range(nsteps):
            if bcase is not None and bcase >= 0:
                self.bcond(bcase, force, u_inflow, inflow_cte1)
            self.bcond_obs()
            self.col_mc(omega, cte1, force_mode, fx, fy, fz)
            self.swap()

    # -- diagnostics -------------------------------------------------------
    def diagno(self, cte1=1.0, fluid_only=True) -> np.ndarray:
        out = (c_double * 5)()
        obs = self.obs.ctypes.data if (fluid_only and self.obs is not None) else None
        rc = lib().orc_diagno(self.kind, _ptrs(self.a), self.l, self.m, self.n, self.nx, self.ny,
                              obs, cte1, self.scale, out)
        assert rc == 0
        return np.array(out[:])

    def dissipation(self, svisc, cte1=1.0, p0=1.0 / 3.0, p1=1.0 / 18.0, p2=1.0 / 36.0, rf=3.0, qf=1.5,
                    tre=3.0, fluid_only=True) -> np.ndarray:
        """SRC/dissipation.F90:136-338 on the current a arrays, halo as stored
        (call bcond first for the reference's boundary values): {sum 0.5 vsq,
        sum 2 nu Ptotal, sum vx2, sum vy2, sum vz2}."""
        out = (c_double * 5)()
        obs = self.obs.ctypes.data if (fluid_only and self.obs is not None) else None
        rc = lib().orc_dissipation(self.kind, _ptrs(self.a), self.l, self.m, self.n, self.nx, self.ny, obs,
                                   svisc, 1.0 - cte1, cte1, p0, p1, p2, rf, qf, tre, self.scale, out)
        assert rc == 0
        return np.array(out[:])

    def enstrophy(self, periodic=(True, True, True), cte1=1.0) -> np.ndarray:
        """{sum 0.5 |curl u|^2, nodes counted} with central differences of the
        node velocities (SRC/vtk_om.xy.binary.F90:49-87); periodic axes wrap,
        other axes leave out their two face layers."""
        out = (c_double * 2)()
        obs = self.obs.ctypes.data if self.obs is not None else None
        bits = sum(1 << a for a, p in enumerate(periodic) if p)
        rc = lib().orc_enstrophy(self.kind, _ptrs(self.a), self.l, self.m, self.n, self.nx, self.ny, obs, cte1,
                                 bits, self.scale, out)
        assert rc == 0
        return np.array(out[:])

    def init(self, flow: int, params=(1.0, 0.0, 0.0, 0.0), rf=3.0, qf=1.5, tre=3.0, p0=1.0 / 3.0,
             p1=1.0 / 18.0, p2=1.0 / 36.0) -> None:
        """Initial populations over the whole box: flow 0 uniform, 1 Taylor-Green,
        2 Kida (benchmark forms), 3 the reference's TGV3D form, 4 its default
        periodic 2-D Taylor-Green form (SRC/init.F90:113-201)."""
        prm = (c_double * 4)(*([float(v) for v in params] + [0.0] * (4 - len(params))))
        rc = lib().orc_init(self.kind, _ptrs(self.a), self.l, self.m, self.n, self.nx, self.ny, flow, prm,
                            rf, qf, tre, p0, p1, p2, self.scale)
        assert rc == 0
        for d in range(18):
            self.b[d][...] = self.a[d]

    def draglift(self, box) -> np.ndarray:
        out = (c_double * 3)()
        rc = lib().orc_draglift(self.kind, _ptrs(self.a), self.obs.ctypes.data, self.l, self.m,
                                self.n, self.nx, self.ny, *box, self.scale, out)
        assert rc == 0
        return np.array(out[:])

    def profile(self, axis: int, c1: int, c2: int, cte1: float = 1.0) -> np.ndarray:
        """(len, 4) (u_x, u_y, u_z, rho) along a grid line (SRC/prof_k.F90:47-77)."""
        ln = (self.l, self.m, self.n)[axis]
        out = np.zeros((ln, 4))
        rc = lib().orc_profile(self.kind, _ptrs(self.a), self.l, self.m, self.n, self.nx, self.ny, axis, c1, c2,
                               cte1, self.scale, out.ctypes.data_as(POINTER(c_double)))
        assert rc == 0
        return out

    def probe(self, i: int, j: int, k: int, cte1: float = 1.0) -> np.ndarray:
        """(u_x, u_y, u_z, rho) at one node (SRC/probe.F90:50-78)."""
        out = np.zeros(4)
        rc = lib().orc_probe(self.kind, _ptrs(self.a), self.nx, self.ny, i, j, k, cte1, self.scale,
                             out.ctypes.data_as(POINTER(c_double)))
        assert rc == 0
        return out

    def slice(self, plane: int, index: int) -> np.ndarray:
        """(n2, n1, 3) float32 velocity of a VTK slice (SRC/vtk_xy.binary.F90:78-97)."""
        n1 = self.m if plane == 2 else self.l
        n2 = self.m if plane == 0 else self.n
        out = np.zeros((n2, n1, 3), np.float32)
        rc = lib().orc_slice(self.kind, _ptrs(self.a), self.l, self.m, self.n, self.nx, self.ny, plane, index,
                             self.scale, out.ctypes.data_as(POINTER(c_float)))
        assert rc == 0
        return out

    def fluid_mask(self) -> np.ndarray:
        """(n, m, l) bool mask of the nodes whose values are defined."""
        if self.obs is None:
            return np.ones((self.n, self.m, self.l), bool)
        return self.obs != 1

    def interior(self, d=None) -> np.ndarray:
        """Interior (1..l,1..m,1..n) view of the current a arrays: (19, n, m, l)."""
        st = np.stack(self.a)
        return st[:, 1:self.n + 1, 1:self.m + 1, 1:self.l + 1]
