"""Python host side of the library: a reference-layout lattice on the device
(memory from torch), advanced through the C ABI of libbgk3d_b200.so.

`DeviceLattice` mirrors the reference's driver loop for one case
(SRC/bgk3d.F90:169-179: boundaries -> col_MC -> pointer swap) with the
boundary fused into the sweep, and its diagnostics (SRC/diagno.F90,
SRC/draglift.F90) as FP64 device reductions.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch

from . import _lib
from ._lib import BC_NAMES, KIND_NAMES, check, lib, ptr_array, sweep_params

TORCH_DTYPE = {0: torch.float64, 1: torch.float32, 2: torch.float16, 3: torch.bfloat16,
               4: torch.float32}


def _kind(k) -> int:
    return KIND_NAMES[k] if isinstance(k, str) else int(k)


def _bcase(b) -> int:
    return BC_NAMES[b] if isinstance(b, str) else int(b)


class DeviceLattice:
    """19 'a' + 18 'b' device arrays in the reference layout, pop 19 in place."""

    def __init__(self, l, m, n, kind="f32", bcase="periodic", omega=1.0, ipad=0, jpad=0,
                 device="cuda", scale=1.0, lid_force=0.0, u_inflow=0.0, inflow_cte1=0.0,
                 force_mode=0, force=(0.0, 0.0, 0.0), cte1=1.0, fast=False):
        self.l, self.m, self.n = l, m, n
        self.kind, self.bcase = _kind(kind), _bcase(bcase)
        self.nx, self.ny, self.nz = l + 2 + ipad, m + 2 + jpad, n + 2
        self.device = torch.device(device)
        dt = TORCH_DTYPE[self.kind]
        self.A = torch.zeros((19, self.nz, self.ny, self.nx), dtype=dt, device=self.device)
        self.B = torch.zeros((18, self.nz, self.ny, self.nx), dtype=dt, device=self.device)
        self._a = [self.A[d] for d in range(19)]
        self._b = [self.B[d] for d in range(18)]
        self.obs = None
        self.params = sweep_params(self.kind, l, m, n, omega, bcase=self.bcase, nx=self.nx,
                                   ny=self.ny, scale=scale, lid_force=lid_force, u_inflow=u_inflow,
                                   inflow_cte1=inflow_cte1, force_mode=force_mode,
                                   fx=force[0], fy=force[1], fz=force[2], cte1=cte1,
                                   cte0=1.0 - cte1, fast=1 if fast else 0)
        self._ws = None
        self._out = torch.zeros(8, dtype=torch.float64, device=self.device)
        self.steps_done = 0

    # ------------------------------------------------------------ state I/O
    def upload(self, state: np.ndarray) -> None:
        """state: (19, nz, ny, nx) in the storage representation (uint16 bits for 16-bit kinds)."""
        t = torch.from_numpy(np.ascontiguousarray(state))
        if self.kind in (2, 3):
            t = t.view(torch.int16).view(TORCH_DTYPE[self.kind])
        for d in range(19):
            self._a[d].copy_(t[d].to(self.device))
        for d in range(18):
            self._b[d].copy_(t[d].to(self.device))

    def download(self) -> np.ndarray:
        """Current (post-collision) state, (19, nz, ny, nx), storage representation."""
        st = torch.stack([p for p in self._a]).cpu()
        if self.kind in (2, 3):
            return st.view(torch.int16).numpy().view(np.uint16)
        return st.numpy()

    def set_obstacle(self, obs: np.ndarray) -> None:
        """obs: int32 (n, m, l) [k, j, i], 1 = solid (SRC/build.obs.F90 convention)."""
        obs = np.ascontiguousarray(obs, np.int32)
        self.obs = torch.from_numpy(obs).to(self.device)
        ks, js, is_ = np.nonzero(obs == 1)
        p = self.params
        p.obs = self.obs.data_ptr()
        p.obs_nx, p.obs_ny = self.l, self.m
        if len(is_):
            p.imin, p.imax = int(is_.min()) + 1, int(is_.max()) + 1
            p.jmin, p.jmax = int(js.min()) + 1, int(js.max()) + 1
            p.kmin, p.kmax = int(ks.min()) + 1, int(ks.max()) + 1
        else:
            p.imin, p.imax, p.jmin, p.jmax, p.kmin, p.kmax = 1, 0, 1, 0, 1, 0

    # ------------------------------------------------------------ time loop
    def _ptrs(self):
        return (ptr_array([t.data_ptr() for t in self._a]),
                ptr_array([t.data_ptr() for t in self._b] + [self._a[18].data_ptr()]))

    def sweep(self, stream=None) -> None:
        """One fused time step (boundaries + stream + collide) and the a<->b swap."""
        a, b = self._ptrs()
        st = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        check(lib().bgk_sweep(ctypes.byref(self.params), a, b, st), "bgk_sweep")
        for d in range(18):
            self._a[d], self._b[d] = self._b[d], self._a[d]
        self.steps_done += 1

    def step(self, nsteps=1) -> None:
        for _ in range(nsteps):
            self.sweep()

    # ---------------------------------------------------------- diagnostics
    def _workspace(self):
        if self._ws is None:
            nb = lib().bgk_reduce_workspace_bytes(self.l, self.m, self.n)
            self._ws = torch.empty(max(nb, 1 << 16), dtype=torch.uint8, device=self.device)
        return self._ws

    def moments(self) -> np.ndarray:
        """FP64 sums over fluid nodes: rho, u_x, u_y, u_z, 0.5|u|^2 (SRC/diagno.F90)."""
        ws = self._workspace()
        a, _ = self._ptrs()
        st = torch.cuda.current_stream(self.device).cuda_stream
        check(lib().bgk_moments(ctypes.byref(self.params), a, self._out.data_ptr(), ws.data_ptr(),
                                ws.numel(), st), "bgk_moments")
        return self._out[:5].cpu().numpy().copy()

    def dissipation(self, nu: float) -> np.ndarray:
        """FP64 turbulence diagnostics (SRC/dissipation.F90 and the enstrophy):
        sum 0.5|u|^2, sum 2 nu Pi:Pi, sum u_x^2, u_y^2, u_z^2, sum 0.5|w|^2 and
        the number of nodes in that last sum (bgk_dissipation)."""
        nb = lib().bgk_dissipation_workspace_bytes(self.l, self.m, self.n)
        ws = torch.empty(max(nb, 1 << 16), dtype=torch.uint8, device=self.device)
        a, _ = self._ptrs()
        st = torch.cuda.current_stream(self.device).cuda_stream
        check(lib().bgk_dissipation(ctypes.byref(self.params), a, float(nu), self._out.data_ptr(), ws.data_ptr(),
                                    ws.numel(), st), "bgk_dissipation")
        return self._out[:7].cpu().numpy().copy()

    def draglift(self, box) -> np.ndarray:
        """FP64 momentum-exchange force (Fx, Fy, Fz) over the box (is, ie, js, je, ks, ke)."""
        ws = self._workspace()
        a, _ = self._ptrs()
        st = torch.cuda.current_stream(self.device).cuda_stream
        check(lib().bgk_draglift(ctypes.byref(self.params), a, *[int(v) for v in box],
                                 self._out.data_ptr(), ws.data_ptr(), ws.numel(), st),
              "bgk_draglift")
        return self._out[:3].cpu().numpy().copy()

    def _diag_call(self, fn, *args, n_out: int, dtype):
        out = torch.empty(n_out, dtype=dtype, device=self.device)
        a, _ = self._ptrs()
        st = torch.cuda.current_stream(self.device).cuda_stream
        check(getattr(lib(), fn)(ctypes.byref(self.params), a, *args, out.data_ptr(), st), fn)
        return out.cpu().numpy()

    def profile(self, axis: int, c1: int, c2: int) -> np.ndarray:
        """(len, 5): position (t - 0.5), u_x, u_y, u_z, rho along a grid line (bgk_profile)."""
        ln = (self.l, self.m, self.n)[axis] if axis in (0, 1, 2) else 1   # the library rejects bad axes
        v = self._diag_call("bgk_profile", axis, c1, c2, n_out=4 * ln, dtype=torch.float64).reshape(ln, 4)
        return np.column_stack([np.arange(1, ln + 1) - 0.5, v])

    def probe(self, i: int, j: int, k: int) -> np.ndarray:
        """(u_x, u_y, u_z, rho) at one node (bgk_probe)."""
        return self._diag_call("bgk_probe", i, j, k, n_out=4, dtype=torch.float64)

    def slice(self, plane: int, index: int) -> np.ndarray:
        """(n2, n1, 3) float32 velocity over a plane (bgk_slice)."""
        n1 = self.m if plane == 2 else self.l
        n2 = self.m if plane == 0 else self.n    # (the library rejects planes other than 0, 1, 2)
        return self._diag_call("bgk_slice", plane, index, n_out=3 * n1 * n2, dtype=torch.float32).reshape(n2, n1, 3)


class Lattice:
    """A library-owned lattice (bgk_lattice_*): padded aligned layout, AB or
    in-place AA pattern, CUDA-graph replay of long step runs.  Host transfers
    use the reference layout (19, n+2, m+2, l+2) in the storage representation."""

    def __init__(self, l, m, n, kind="f32", bcase="periodic", omega=1.0, pattern="ab",
                 lid_force=0.0, u_inflow=0.0, force_mode=0, force=(0.0, 0.0, 0.0), scale=1.0,
                 device=None, fast=False):
        from ._lattice_abi import LatticeDesc
        self.L = lib()
        self.l, self.m, self.n = l, m, n
        self.kind, self.bcase = _kind(kind), _bcase(bcase)
        self.device = torch.device(device or "cuda")
        d = LatticeDesc()
        self.L.bgk_lattice_desc_init(ctypes.byref(d), self.kind, self.bcase, l, m, n, float(omega))
        d.pattern = 1 if pattern in ("aa", 1) else 0
        d.lid_force, d.u_inflow, d.force_mode = lid_force, u_inflow, force_mode
        d.fx, d.fy, d.fz = force
        d.scale = scale
        d.fast = 1 if fast else 0
        self.desc = d
        h = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            check(self.L.bgk_lattice_create(ctypes.byref(d), ctypes.byref(h)), "bgk_lattice_create")
        self.h = h
        self._out = torch.zeros(8, dtype=torch.float64, device=self.device)

    def close(self, stream=None):
        """Free the lattice; with a torch stream, stream-ordered after the work
        queued on it (every use of the lattice must be on that stream)."""
        if getattr(self, "h", None):
            if stream is None:
                self.L.bgk_lattice_destroy(self.h)
            else:
                self.L.bgk_lattice_destroy_async(self.h, stream.cuda_stream)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def device_bytes(self) -> int:
        return int(self.L.bgk_lattice_device_bytes(ctypes.byref(self.desc)))

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def set_obstacle(self, obs: np.ndarray | None) -> None:
        if obs is None:
            check(self.L.bgk_lattice_set_obstacle(self.h, None), "set_obstacle")
            return
        o = np.ascontiguousarray(obs, np.int32)
        check(self.L.bgk_lattice_set_obstacle(self.h, o.ctypes.data), "set_obstacle")

    def set_zhalo(self, flags: int) -> None:
        """z faces that read the halo planes as stored (bgk_lattice_set_zhalo):
        bit 0 the face k = 1, bit 1 the face k = n (z-slab decomposition)."""
        check(self.L.bgk_lattice_set_zhalo(self.h, int(flags)), "bgk_lattice_set_zhalo")

    def plane(self, pop: int, k: int) -> torch.Tensor:
        """Plane k of population pop of the current state as a device tensor
        view (storage representation; bgk_lattice_plane).  Valid until the next step."""
        ptr, nb = ctypes.c_void_p(), ctypes.c_size_t()
        check(self.L.bgk_lattice_plane(self.h, int(pop), int(k), ctypes.byref(ptr), ctypes.byref(nb)),
              "bgk_lattice_plane")
        return _device_bytes(ptr.value, nb.value, self.device)

    def set_sphere(self, center, r2: float) -> None:
        """Solid sphere obstacle built on the device (bgk_lattice_set_sphere)."""
        check(self.L.bgk_lattice_set_sphere(self.h, float(center[0]), float(center[1]), float(center[2]),
                                            float(r2)), "bgk_lattice_set_sphere")

    def upload(self, state: np.ndarray) -> None:
        st = np.ascontiguousarray(state)
        check(self.L.bgk_lattice_load(self.h, st.ctypes.data, self._stream()), "bgk_lattice_load")
        torch.cuda.current_stream(self.device).synchronize()

    FLOWS = {"uniform": 0, "rest": 0, "tgv": 1, "kida": 2, "tgv_ref": 3, "tg2d_ref": 4}

    def init_flow(self, flow: str, params=(1.0, 0.0, 0.0, 0.0)) -> None:
        """Equilibrium state of an analytic flow computed on the device."""
        arr = (ctypes.c_double * 4)(*([float(v) for v in params] + [0.0] * (4 - len(params))))
        check(self.L.bgk_lattice_init(self.h, self.FLOWS[flow], arr, self._stream()), "bgk_lattice_init")

    def profile(self, axis: int, c1: int, c2: int) -> np.ndarray:
        """(len, 5): position (t - 0.5), u_x, u_y, u_z, rho along a grid line
        (bgk_lattice_profile; axis 0 = prof_i at (j, k) = (c1, c2), 1 = prof_j
        at (i, k), 2 = prof_k at (i, j))."""
        ln = (self.l, self.m, self.n)[axis] if axis in (0, 1, 2) else 1   # the library rejects bad axes
        out = torch.empty(4 * ln, dtype=torch.float64, device=self.device)
        check(self.L.bgk_lattice_profile(self.h, axis, c1, c2, out.data_ptr(), self._stream()),
              "bgk_lattice_profile")
        return np.column_stack([np.arange(1, ln + 1) - 0.5, out.cpu().numpy().reshape(ln, 4)])

    def probe(self, i: int, j: int, k: int) -> np.ndarray:
        """(u_x, u_y, u_z, rho) at one node (bgk_lattice_probe)."""
        out = torch.empty(4, dtype=torch.float64, device=self.device)
        check(self.L.bgk_lattice_probe(self.h, i, j, k, out.data_ptr(), self._stream()), "bgk_lattice_probe")
        return out.cpu().numpy()

    def slice(self, plane: int, index: int) -> np.ndarray:
        """(n2, n1, 3) float32 velocity over a plane (bgk_lattice_slice; plane 0
        = xy at k = index, 1 = xz at j = index, 2 = yz at i = index)."""
        n1 = self.m if plane == 2 else self.l
        n2 = self.m if plane == 0 else self.n    # (the library rejects planes other than 0, 1, 2)
        out = torch.empty(3 * n1 * n2, dtype=torch.float32, device=self.device)
        check(self.L.bgk_lattice_slice(self.h, plane, index, out.data_ptr(), self._stream()), "bgk_lattice_slice")
        return out.cpu().numpy().reshape(n2, n1, 3)

    def save(self, path, itime: int | None = None, file_bytes: int = 0) -> None:
        """Restart file in the reference's record format (bgk_lattice_save);
        itime defaults to the lattice's step count."""
        it = self.steps if itime is None else int(itime)
        check(self.L.bgk_lattice_save(self.h, os.fsencode(path), it, int(file_bytes), self._stream()),
              "bgk_lattice_save")

    def restore(self, path) -> int:
        """Load a restart file (bgk_lattice_restore); returns its time step."""
        it = ctypes.c_int(0)
        check(self.L.bgk_lattice_restore(self.h, os.fsencode(path), ctypes.byref(it), self._stream()),
              "bgk_lattice_restore")
        return int(it.value)

    def download(self) -> np.ndarray:
        dt = {0: np.float64, 1: np.float32, 2: np.uint16, 3: np.uint16, 4: np.float32}[self.kind]
        out = np.empty((19, self.n + 2, self.m + 2, self.l + 2), dt)
        check(self.L.bgk_lattice_store(self.h, out.ctypes.data, self._stream()), "bgk_lattice_store")
        torch.cuda.current_stream(self.device).synchronize()
        return out

    def step(self, nsteps=1) -> None:
        check(self.L.bgk_lattice_step(self.h, int(nsteps), self._stream()), "bgk_lattice_step")

    def prepare(self) -> None:
        """Capture the step graph now (nothing runs), so that the first long
        step run starts without the capture."""
        check(self.L.bgk_lattice_prepare(self.h), "bgk_lattice_prepare")

    def step_moments(self, nsteps: int, every: int = 1) -> np.ndarray:
        """Advance nsteps steps; FP64 moments of the state after every `every`-th
        step, computed in the same pass as that step: array (nsteps // every, 5)."""
        ns = nsteps // every
        out = torch.zeros(max(ns, 1) * 5, dtype=torch.float64, device=self.device)
        check(self.L.bgk_lattice_step_moments(self.h, int(nsteps), int(every), out.data_ptr(),
                                              self._stream()), "bgk_lattice_step_moments")
        return out[:ns * 5].view(ns, 5).cpu().numpy()

    @property
    def steps(self) -> int:
        return int(self.L.bgk_lattice_steps(self.h))

    def moments(self) -> np.ndarray:
        check(self.L.bgk_lattice_moments(self.h, self._out.data_ptr(), self._stream()), "moments")
        return self._out[:5].cpu().numpy().copy()

    def dissipation(self, nu: float) -> np.ndarray:
        """FP64 TKE, 2 nu Pi:Pi, mean squares, enstrophy and its node count
        (bgk_lattice_dissipation), 7 values."""
        check(self.L.bgk_lattice_dissipation(self.h, float(nu), self._out.data_ptr(), self._stream()),
              "dissipation")
        return self._out[:7].cpu().numpy().copy()

    def draglift(self, box) -> np.ndarray:
        check(self.L.bgk_lattice_draglift(self.h, *[int(v) for v in box], self._out.data_ptr(),
                                          self._stream()), "draglift")
        return self._out[:3].cpu().numpy().copy()


class Batch:
    """Many Lattice objects (AB pattern, one storage kind) advanced together
    (bgk_batch_*): by default one launch per group of members that share a
    boundary case, collision mode and obstacle logic, blocks taking chunks of
    one member's warp segments; or one persistent launch over a device tile
    queue (set_config)."""

    def __init__(self, lattices):
        self.L = lib()
        self.members = list(lattices)
        arr = (ctypes.c_void_p * len(self.members))(*[m.h.value for m in self.members])
        h = ctypes.c_void_p()
        check(self.L.bgk_batch_create(arr, len(self.members), ctypes.byref(h)), "bgk_batch_create")
        self.h = h
        self.device = self.members[0].device

    def close(self):
        if getattr(self, "h", None):
            self.L.bgk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _stream(self):
        return torch.cuda.current_stream(self.device).cuda_stream

    def step(self, nsteps: int = 1) -> None:
        check(self.L.bgk_batch_step(self.h, int(nsteps), self._stream()), "bgk_batch_step")

    def resync(self) -> None:
        """Accept members' states after they were loaded or stepped on their own."""
        check(self.L.bgk_batch_resync(self.h), "bgk_batch_resync")

    def tune(self, trial_steps: int = 4) -> int:
        used = ctypes.c_int()
        check(self.L.bgk_batch_tune(self.h, int(trial_steps), self._stream(), ctypes.byref(used)),
              "bgk_batch_tune")
        return used.value

    @property
    def config(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        check(self.L.bgk_batch_get_config(self.h, ctypes.byref(a), ctypes.byref(b)), "get_config")
        return a.value, b.value

    def set_config(self, tiles_per_grab: int, blocks_per_sm: int) -> None:
        """Select the tile-queue form with these parameters."""
        check(self.L.bgk_batch_set_chunk(self.h, 0), "set_chunk")
        check(self.L.bgk_batch_set_config(self.h, tiles_per_grab, blocks_per_sm), "set_config")

    @property
    def chunk(self) -> int:
        w = ctypes.c_int()
        check(self.L.bgk_batch_get_chunk(self.h, ctypes.byref(w)), "get_chunk")
        return w.value

    def set_chunk(self, warps_per_chunk: int) -> None:
        """Select the grouped form with this many warp segments per chunk (0: tile queue)."""
        check(self.L.bgk_batch_set_chunk(self.h, int(warps_per_chunk)), "set_chunk")

    @property
    def groups(self) -> int:
        """Launches per step of the grouped form (groups + solo members)."""
        return int(self.L.bgk_batch_groups(self.h))

    @property
    def solo(self) -> int:
        return int(self.L.bgk_batch_get_solo(self.h))

    def set_solo(self, min_nodes: int) -> None:
        """Members of min_nodes nodes or more step with their own launch (0: none)."""
        check(self.L.bgk_batch_set_solo(self.h, int(min_nodes)), "set_solo")

    @property
    def nodes(self) -> int:
        return int(self.L.bgk_batch_nodes(self.h))


class _DeviceRegion:
    """__cuda_array_interface__ of nbytes bytes of device memory at ptr."""

    def __init__(self, ptr: int, nbytes: int):
        self.__cuda_array_interface__ = {"shape": (nbytes,), "typestr": "|u1", "data": (ptr, False),
                                         "version": 3, "strides": None}


def _device_bytes(ptr: int, nbytes: int, device) -> torch.Tensor:
    """A uint8 tensor viewing device memory the library owns (no copy)."""
    return torch.as_tensor(_DeviceRegion(ptr, nbytes), device=device)


def set_retained_bytes(nbytes: int) -> None:
    """Bytes of freed lattice memory the current device's pool keeps for reuse
    (bgk_set_retained_bytes; 0, the default, gives it back at once)."""
    check(lib().bgk_set_retained_bytes(int(nbytes)), "bgk_set_retained_bytes")


def trim_memory() -> None:
    check(lib().bgk_trim_memory(), "bgk_trim_memory")


def save_name(itime: int) -> str:
    """The reference's restart file name for a time step (SRC/save_raw.F90:39-41)."""
    return f"save.{int(itime):08d}.bin"
