"""Case builders: the flows the reference's compile-time case flags select
(SRC/Makefile:328-361: LDC, TGV/HIT, VKS = inflow + obstacle, KVX, POF =
channel) with the parameters of the benchmark configurations, plus the
reference's own obstacle builder (SRC/build.obs.F90) and collision
parameters (SRC/hencol.F90).

A case is a dict of Lattice keyword arguments plus `init` (a function that
returns rho, ux, uy, uz device fields [k, j, i]), `flow` (the on-device
initial condition) and, for obstacle flows, `sphere` (centre, radius^2: the
mask is built on the device; obstacle_mask() builds it on the host) or
`obstacle` (int32 mask [k, j, i]), and `drag_box`.
"""
from __future__ import annotations

import math

import numpy as np

from . import fields as F


def tau_from_nu(nu: float) -> float:
    """tau = 3 nu + 0.5 (lattice units)."""
    return 3.0 * nu + 0.5


def omega_from_nu(nu: float) -> float:
    """SRC/hencol.F90:31: omega = 2 / (6 nu + 1) = 1 / tau."""
    return 2.0 / (6.0 * nu + 1.0)


def fgrad(u0: float, nu: float, m: int) -> float:
    """Channel forcing amplitude of SRC/hencol.F90:52: 4 u0 nu / (5 m^2)."""
    return 4.0 * u0 * nu / (5.0 * m * m)


# ------------------------------------------------------------------ obstacles
def reference_shell_obstacle(l: int, m: int, n: int, ly: int | None = None):
    """SRC/build.obs.F90:52-97: a spherical SHELL (R-2)^2 < d^2 < (R+2)^2,
    centre (2l/5, m/2, n/2) in integer division, R = 32 if m > 256 else ly/8.
    Returns (obs [k, j, i] int32, radius, bbox (imin, imax, jmin, jmax, kmin, kmax))."""
    ly = m if ly is None else ly
    ic, jc, kc = 2 * l // 5, m // 2, n // 2
    radius = 32 if m > 256 else ly // 8
    R = float(radius)
    r2a, r2b = (R - 2.0) ** 2, (R + 2.0) ** 2
    k, j, i = np.meshgrid(np.arange(1, n + 1), np.arange(1, m + 1), np.arange(1, l + 1), indexing="ij")
    d2 = ((ic - i) * (ic - i) + (jc - j) * (jc - j) + (kc - k) * (kc - k)).astype(np.float64)
    obs = ((d2 > r2a) & (d2 < r2b)).astype(np.int32)
    return obs, radius, _bbox(obs)


def solid_sphere_obstacle(l: int, m: int, n: int, diameter: float, center):
    """A solid sphere of the given diameter: nodes with |x - c|^2 <= (D/2)^2."""
    k, j, i = np.meshgrid(np.arange(1, n + 1), np.arange(1, m + 1), np.arange(1, l + 1), indexing="ij")
    r2 = (diameter / 2.0) ** 2
    d2 = (i - center[0]) ** 2 + (j - center[1]) ** 2 + (k - center[2]) ** 2
    obs = (d2 <= r2).astype(np.int32)
    return obs, _bbox(obs)


def sphere_bbox(l: int, m: int, n: int, diameter: float, center):
    """Bounding box (imin, imax, jmin, jmax, kmin, kmax) of the solid nodes of
    solid_sphere_obstacle, from the extents and the rule alone (no mask)."""
    r2 = (diameter / 2.0) ** 2
    ext = (l, m, n)

    def near(a, c):   # smallest (x - c)^2 over the integers 1..a
        x = min(max(int(round(c)), 1), a)
        return (x - c) ** 2

    lo, hi = [], []
    for ax in range(3):
        others = sum(near(ext[b], center[b]) for b in range(3) if b != ax)
        xs = [x for x in range(1, ext[ax] + 1) if (x - center[ax]) ** 2 + others <= r2]
        if not xs:
            return None
        lo.append(min(xs))
        hi.append(max(xs))
    return (lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])


def obstacle_mask(case: dict):
    """The case's int32 obstacle mask [k, j, i] (built on the host), or None."""
    if case.get("obstacle") is not None:
        return case["obstacle"]
    if case.get("sphere") is not None:
        center, r2 = case["sphere"]
        k, j, i = np.meshgrid(np.arange(1, case["n"] + 1), np.arange(1, case["m"] + 1),
                              np.arange(1, case["l"] + 1), indexing="ij")
        d2 = (i - center[0]) ** 2 + (j - center[1]) ** 2 + (k - center[2]) ** 2
        return (d2 <= r2).astype(np.int32)
    return None


def _bbox(obs):
    ks, js, is_ = np.nonzero(obs == 1)
    if len(is_) == 0:
        return None
    return (int(is_.min()) + 1, int(is_.max()) + 1, int(js.min()) + 1, int(js.max()) + 1,
            int(ks.min()) + 1, int(ks.max()) + 1)


def drag_box(bbox, delta: int = 3):
    """Box of SRC/draglift.F90:54-62: the obstacle extent grown by delta."""
    return (bbox[0] - delta, bbox[1] + delta, bbox[2] - delta, bbox[3] + delta, bbox[4] - delta,
            bbox[5] + delta)


# ---------------------------------------------------------------------- cases
def _rest(l, m, n):
    def init(device="cuda"):
        import torch
        z = torch.zeros((n, m, l), dtype=torch.float64, device=device)
        return z + 1.0, z.clone(), z.clone(), z.clone()
    return init


def lid_driven_cavity(n: int = 128, kind: str = "f64", re: float = 400.0, u_lid: float = 0.1, **kw):
    """3-D lid-driven cavity: n^3, bounce-back walls, lid u = (u_lid, 0, 0) at
    z = n+1 through the lid term force = u_lid / 6 (SRC/bcond.driven.F90:61),
    nu = u_lid n / Re, rest initial state."""
    nu = u_lid * n / re
    return dict(l=n, m=n, n=n, kind=kind, bcase="driven", omega=1.0 / tau_from_nu(nu),
                lid_force=u_lid / 6.0, init=_rest(n, n, n), flow=("rest", (1.0, 0.0, 0.0, 0.0)), nu=nu,
                name=f"ldc{n}_{kind}", **kw)


def taylor_green(n: int = 256, kind: str = "f32", u0: float = 0.05, re: float = 1600.0, **kw):
    """Periodic Taylor-Green vortex, nu = u0 n / Re (box length)."""
    nu = u0 * n / re

    def init(device="cuda"):
        return F.taylor_green_fields(n, n, n, u0, device=device)
    return dict(l=n, m=n, n=n, kind=kind, bcase="periodic", omega=1.0 / tau_from_nu(nu), init=init,
                flow=("tgv", (u0,)), nu=nu, u0=u0, name=f"tgv{n}_{kind}", **kw)


def kida(n: int, tau: float, kind: str = "f32", u0: float = 0.05, **kw):
    """Periodic Kida vortex, rho = 1."""
    def init(device="cuda"):
        return F.kida_fields(n, n, n, u0, device=device)
    return dict(l=n, m=n, n=n, kind=kind, bcase="periodic", omega=1.0 / tau, init=init,
                flow=("kida", (u0,)), name=f"kida{n}_{kind}", **kw)


def poiseuille(n: int, tau: float, kind: str = "f32", g: float = 1e-6, **kw):
    """Channel: x, y periodic, z bounce-back walls, body force g along x.
    The reference adds +-force to the 10 populations with c_x != 0
    (SRC/col_MC.F90:501-518), 10 force per node and step, with
    force = fgrad * rho (:482); g / 10 per population gives momentum g rho."""
    return dict(l=n, m=n, n=n, kind=kind, bcase="channel", omega=1.0 / tau, force_mode=1,
                force=(g / 10.0, 0.0, 0.0), init=_rest(n, n, n), flow=("rest", (1.0, 0.0, 0.0, 0.0)),
                name=f"pof{n}_{kind}", **kw)


def sphere(l: int = 512, m: int = 256, n: int = 256, kind: str = "f32", diameter: float = 40.0,
           center=(128, 128, 128), u_in: float = 0.05, re: float = 300.0, **kw):
    """Flow past a solid sphere: inflow u = (u_in, 0, 0) at x = 0, outflow at
    x = l+1 (equilibrium at rho = 1 with the momentum of node l, the
    reference's rule), periodic y/z, nu = u_in D / Re, rest initial state."""
    nu = u_in * diameter / re
    bbox = sphere_bbox(l, m, n, diameter, center)
    return dict(l=l, m=m, n=n, kind=kind, bcase="inflow", omega=1.0 / tau_from_nu(nu), u_inflow=u_in,
                init=_rest(l, m, n), flow=("rest", (1.0, 0.0, 0.0, 0.0)),
                sphere=(tuple(float(v) for v in center), (diameter / 2.0) ** 2),
                drag_box=drag_box(bbox) if bbox else None, radius=diameter / 2.0, nu=nu, name=f"sphere{l}x{m}x{n}_{kind}", **kw)


LATTICE_KEYS = ("kind", "bcase", "omega", "lid_force", "u_inflow", "force_mode", "force", "scale",
                "pattern", "fast")


def make_lattice(case: dict, pattern: str = "ab", scale: float | None = None, on_device: bool = True,
                 fast: bool | None = None):
    """Create a Lattice for the case, set its obstacle and its initial state:
    computed on the device for the analytic flows (default), else built with
    torch and loaded from the host."""
    import torch
    from .lattice import Lattice
    kw = {k: case[k] for k in LATTICE_KEYS if k in case}
    kw["pattern"] = pattern
    if fast is not None:
        kw["fast"] = fast
    if scale is not None:
        kw["scale"] = scale
    elif kw.get("kind") == "f16":
        kw["scale"] = 256.0
    lat = Lattice(case["l"], case["m"], case["n"], **kw)
    if case.get("sphere") is not None:
        lat.set_sphere(*case["sphere"])          # mask built on the device
    elif case.get("obstacle") is not None:
        lat.set_obstacle(case["obstacle"])
    if on_device and case.get("flow") is not None:
        lat.init_flow(*case["flow"])
    else:
        lat.upload(initial_state(case, lat.kind, kw.get("scale", 1.0)))
    return lat


def initial_state(case: dict, kind: int, scale: float = 1.0):
    """(19, n+2, m+2, l+2) equilibrium state of the case in the storage
    representation (built on the device, returned as a host numpy array)."""
    import torch
    l, m, n = case["l"], case["m"], case["n"]
    rho, ux, uy, uz = case["init"]("cuda")
    feq = F.equilibrium_shifted_torch(rho, ux, uy, uz, torch.float64)
    del rho, ux, uy, uz
    if kind in (0,):
        dt = torch.float64
    elif kind in (1, 4):
        dt = torch.float32
    else:
        dt = torch.float32
    full = torch.zeros((19, n + 2, m + 2, l + 2), dtype=dt, device="cuda")
    if kind in (2, 3):
        full[:, 1:n + 1, 1:m + 1, 1:l + 1] = (feq.float() * scale)
        full16 = full.to(torch.float16 if kind == 2 else torch.bfloat16)
        return full16.view(torch.int16).cpu().numpy().view(np.uint16)
    full[:, 1:n + 1, 1:m + 1, 1:l + 1] = feq.to(dt)
    return full.cpu().numpy()
