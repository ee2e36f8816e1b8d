"""Host-side helpers for population fields: equilibrium initial conditions,
the reference's collision parameters, and 16-bit storage views.

Population numbering and velocities are the reference's (SRC/alloca.F90:29-148);
populations are stored shifted by their weight, f_p - w_p (cte1 = 1,
SRC/col_MC.F90:139-144).
"""
from __future__ import annotations

import numpy as np

# c_x, c_y, c_z of populations 01..19 (SRC/alloca.F90:29-148)
CX = np.array([1, 1, 1, 1, 1, 0, 0, 0, 0, -1, -1, -1, -1, -1, 0, 0, 0, 0, 0])
CY = np.array([-1, 0, 1, 0, 0, 0, 1, 1, 1, -1, 0, 1, 0, 0, 0, -1, -1, -1, 0])
CZ = np.array([0, -1, 0, 1, 0, 1, 1, 0, -1, 0, -1, 0, 1, 0, -1, -1, 0, 1, 0])
# weights: 1/36 for the 12 diagonal links, 1/18 for the 6 axis links, 1/3 rest
W = np.where(np.abs(CX) + np.abs(CY) + np.abs(CZ) == 2, 1.0 / 36.0,
             np.where(np.abs(CX) + np.abs(CY) + np.abs(CZ) == 1, 1.0 / 18.0, 1.0 / 3.0))
OPP = np.array([11, 12, 9, 10, 13, 14, 15, 16, 17, 2, 3, 0, 1, 4, 5, 6, 7, 8, 18])

KIND_STORAGE = {0: np.float64, 1: np.float32, 2: np.float16, 3: "bfloat16", 4: np.float32}


def omega_from_tau(tau: float) -> float:
    return 1.0 / tau


def omega_hencol(svisc: float) -> float:
    """SRC/hencol.F90:31: omega = 2 / (6 nu + 1)."""
    return 2.0 / (6.0 * svisc + 1.0)


def equilibrium_shifted(rho, ux, uy, uz) -> np.ndarray:
    """f_p^eq - w_p for fields of any shape, in float64: shape (19, *rho.shape).

    f^eq_p = w_p rho (1 + 3 c.u + 4.5 (c.u)^2 - 1.5 u^2); the stored value
    subtracts w_p.  (The reference's init.F90 omits the w_p (rho - 1) term for
    shifted storage, SRC/init.F90:179-197 with cte1 = 0; this helper keeps it,
    so rho is represented exactly.)
    """
    rho = np.asarray(rho, np.float64)
    ux, uy, uz = (np.asarray(u, np.float64) for u in (ux, uy, uz))
    usq = ux * ux + uy * uy + uz * uz
    out = np.empty((19,) + rho.shape, np.float64)
    for p in range(19):
        cu = CX[p] * ux + CY[p] * uy + CZ[p] * uz
        out[p] = W[p] * (rho - 1.0) + W[p] * rho * (3.0 * cu + 4.5 * cu * cu - 1.5 * usq)
    return out


def to_storage_bits(x64: np.ndarray, kind: int, scale: float = 1.0) -> np.ndarray:
    """Round float64 values to the storage kind's representation.

    Returns float64/float32 arrays for native kinds and uint16 bit patterns
    for the 16-bit kinds (value stored = scale * x, round to nearest even,
    rounded through float32 first as the device does).
    """
    if kind == 0:
        return np.ascontiguousarray(x64, np.float64)
    if kind in (1, 4):
        return np.ascontiguousarray(x64, np.float32)
    x32 = (np.asarray(x64, np.float32) * np.float32(scale)).astype(np.float32)
    if kind == 2:
        return x32.astype(np.float16).view(np.uint16)
    if kind == 3:
        u = x32.view(np.uint32).astype(np.uint64)
        lsb = (u >> 16) & 1
        r = ((u + 0x7FFF + lsb) >> 16).astype(np.uint16)
        nan = np.isnan(x32)
        if nan.any():
            r[nan] = ((u[nan] >> 16) | 0x40).astype(np.uint16)
        return r
    raise ValueError(kind)


def from_storage_bits(s: np.ndarray, kind: int, scale: float = 1.0) -> np.ndarray:
    """Inverse of to_storage_bits, returning float64 values."""
    if kind in (0, 1, 4):
        return np.asarray(s, np.float64)
    if kind == 2:
        v = s.view(np.float16).astype(np.float32)
    else:
        v = (s.astype(np.uint32) << 16).view(np.float32)
    return (v * np.float32(1.0 / scale)).astype(np.float64)


def lattice_state(l, m, n, kind, rho=None, u=None, ipad=0, jpad=0, scale=1.0, fill_halo=True):
    """(19, n+2, m+2+jpad, l+2+ipad) storage-kind state at equilibrium.

    rho and u (3 arrays) are given on the interior (n, m, l) grid [k, j, i];
    defaults: rho = 1, u = 0.  With fill_halo the halo replicates the nearest
    interior node (the halo is rewritten by the boundary sweep anyway).
    """
    nz, ny, nx = n + 2, m + 2 + jpad, l + 2 + ipad
    if rho is None:
        rho = np.ones((n, m, l))
    if u is None:
        u = (np.zeros((n, m, l)),) * 3
    feq = equilibrium_shifted(rho, *u)
    full = np.zeros((19, nz, ny, nx))
    full[:, 1:n + 1, 1:m + 1, 1:l + 1] = feq
    if fill_halo:
        full[:, 0] = full[:, 1]
        full[:, n + 1] = full[:, n]
        full[:, :, 0] = full[:, :, 1]
        full[:, :, m + 1] = full[:, :, m]
        full[:, :, :, 0] = full[:, :, :, 1]
        full[:, :, :, l + 1] = full[:, :, :, l]
    return to_storage_bits(full, kind, scale)


def equilibrium_shifted_torch(rho, ux, uy, uz, dtype):
    """Device-side twin of equilibrium_shifted (torch ops, for set-up only):
    returns a (19, *rho.shape) tensor of f_p^eq - w_p in `dtype`, computed in
    float64 and rounded once."""
    import torch
    usq = ux * ux + uy * uy + uz * uz
    out = torch.empty((19,) + tuple(rho.shape), dtype=dtype, device=rho.device)
    for p in range(19):
        cu = float(CX[p]) * ux + float(CY[p]) * uy + float(CZ[p]) * uz
        w = float(W[p])
        out[p] = (w * (rho - 1.0) + w * rho * (3.0 * cu + 4.5 * cu * cu - 1.5 * usq)).to(dtype)
    return out


def taylor_green_fields(l, m, n, u0, device="cpu"):
    """Taylor-Green vortex on an l x m x n periodic box, x = 2 pi (i-1)/l etc.:
    u = u0 sin x cos y cos z, v = -u0 cos x sin y cos z, w = 0,
    rho = 1 + 3 (u0^2/16)(cos 2x + cos 2y)(cos 2z + 2).  Arrays are [k, j, i]."""
    import torch
    two_pi = 2.0 * np.pi
    x = torch.arange(l, dtype=torch.float64, device=device) * (two_pi / l)
    y = torch.arange(m, dtype=torch.float64, device=device) * (two_pi / m)
    z = torch.arange(n, dtype=torch.float64, device=device) * (two_pi / n)
    Z, Y, X = torch.meshgrid(z, y, x, indexing="ij")
    ux = u0 * torch.sin(X) * torch.cos(Y) * torch.cos(Z)
    uy = -u0 * torch.cos(X) * torch.sin(Y) * torch.cos(Z)
    uz = torch.zeros_like(ux)
    rho = 1.0 + 3.0 * (u0 * u0 / 16.0) * (torch.cos(2 * X) + torch.cos(2 * Y)) * (torch.cos(2 * Z) + 2.0)
    return rho, ux, uy, uz


def kida_fields(l, m, n, u0, device="cpu"):
    """Kida vortex: u = u0 sin x (cos 3y cos z - cos y cos 3z), v and w by
    cyclic permutation; rho = 1.  Arrays are [k, j, i]."""
    import torch
    two_pi = 2.0 * np.pi
    x = torch.arange(l, dtype=torch.float64, device=device) * (two_pi / l)
    y = torch.arange(m, dtype=torch.float64, device=device) * (two_pi / m)
    z = torch.arange(n, dtype=torch.float64, device=device) * (two_pi / n)
    Z, Y, X = torch.meshgrid(z, y, x, indexing="ij")
    ux = u0 * torch.sin(X) * (torch.cos(3 * Y) * torch.cos(Z) - torch.cos(Y) * torch.cos(3 * Z))
    uy = u0 * torch.sin(Y) * (torch.cos(3 * Z) * torch.cos(X) - torch.cos(Z) * torch.cos(3 * X))
    uz = u0 * torch.sin(Z) * (torch.cos(3 * X) * torch.cos(Y) - torch.cos(X) * torch.cos(3 * Y))
    return torch.ones_like(ux), ux, uy, uz
