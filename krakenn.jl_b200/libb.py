"""Host-side set-up of interpolated bounce-back (LI-BB) walls.

The fused LI-BB steps (`fused_trt_libb_v2_step_`, `fused_trt_libb_v2_step_3d_`)
read, per node and link, the wall-cut fraction q_wall in (0, 1] (0 = link not
cut) and the wall velocity at the cut.  These helpers compute them for the
reference's analytical geometries, as numpy arrays in the library's layout:
q_wall (9, Ny, Nx) / (19, Nz, Ny, Nx), is_solid (Ny, Nx) / (Nz, Ny, Nx).
Node (i, j[, k]) sits at x = i, y = j[, z = k] (0-based).
"""
from __future__ import annotations

import numpy as np

from . import lattice as L


def _cut_fraction(d, c, R2):
    """Smallest t in (0, 1] with |d + t c|^2 = R^2 for every node offset d
    (arrays, one per axis) and link c; 0 where the link is not cut.  The
    quadratic is solved as the reference does (li_bb_2d.jl:297-311)."""
    a = sum(float(ci) * float(ci) for ci in c)
    b = 2.0 * sum(di * float(ci) for di, ci in zip(d, c))
    cc = sum(di * di for di in d) - R2
    disc = b * b - 4.0 * a * cc
    ok = disc >= 0.0
    sd = np.sqrt(np.where(ok, disc, 0.0))
    t1 = (-b - sd) / (2.0 * a)
    t2 = (-b + sd) / (2.0 * a)
    t = np.where(t1 > 0.0, t1, t2)
    return np.where(ok & (t > 0.0) & (t <= 1.0), t, 0.0)


def precompute_q_wall_cylinder(Nx, Ny, cx, cy, R):
    """precompute_q_wall_cylinder -- src/kernels/li_bb_2d.jl:271-315: nodes
    inside the circle are solid; each fluid link whose end node is inside
    gets the analytical cut fraction."""
    x = np.arange(Nx, dtype=np.float64)[None, :] - float(cx) + np.zeros((Ny, 1))
    y = np.arange(Ny, dtype=np.float64)[:, None] - float(cy) + np.zeros((1, Nx))
    R2 = float(R) * float(R)
    solid = x * x + y * y <= R2
    qw = np.zeros((9, Ny, Nx))
    for q in range(1, 9):
        c = (L.D2Q9_CX[q], L.D2Q9_CY[q])
        xn, yn = x + c[0], y + c[1]
        crosses = (~solid) & (xn * xn + yn * yn <= R2)
        qw[q] = np.where(crosses, _cut_fraction((x, y), c, R2), 0.0)
    return qw, solid


def wall_velocity_rotating_cylinder(q_wall, cx, cy, Omega):
    """wall_velocity_rotating_cylinder -- src/kernels/li_bb_2d.jl:453-470:
    rigid rotation Omega about (cx, cy) evaluated at each cut point."""
    _, Ny, Nx = q_wall.shape
    i = np.arange(Nx, dtype=np.float64)[None, :]
    j = np.arange(Ny, dtype=np.float64)[:, None]
    ux = np.zeros_like(q_wall)
    uy = np.zeros_like(q_wall)
    for q in range(1, 9):
        cut = q_wall[q] != 0.0
        xw = i + q_wall[q] * float(L.D2Q9_CX[q])
        yw = j + q_wall[q] * float(L.D2Q9_CY[q])
        ux[q] = np.where(cut, -float(Omega) * (yw - float(cy)), 0.0)
        uy[q] = np.where(cut, float(Omega) * (xw - float(cx)), 0.0)
    return ux, uy


def precompute_q_wall_sphere_3d(Nx, Ny, Nz, cx, cy, cz, R):
    """precompute_q_wall_sphere_3d -- src/kernels/li_bb_3d_v2.jl:116-156."""
    shape = (Nz, Ny, Nx)
    x = np.broadcast_to(np.arange(Nx, dtype=np.float64)[None, None, :] - float(cx), shape)
    y = np.broadcast_to(np.arange(Ny, dtype=np.float64)[None, :, None] - float(cy), shape)
    z = np.broadcast_to(np.arange(Nz, dtype=np.float64)[:, None, None] - float(cz), shape)
    R2 = float(R) * float(R)
    solid = x * x + y * y + z * z <= R2
    qw = np.zeros((19,) + shape)
    for q in range(1, 19):
        c = (L.D3Q19_CX[q], L.D3Q19_CY[q], L.D3Q19_CZ[q])
        xn, yn, zn = x + c[0], y + c[1], z + c[2]
        crosses = (~solid) & (xn * xn + yn * yn + zn * zn <= R2)
        qw[q] = np.where(crosses, _cut_fraction((x, y, z), c, R2), 0.0)
    return qw, solid


def precompute_q_wall_sphere_3d_torch(Nx, Ny, Nz, cx, cy, cz, R, dtype=None, device="cuda"):
    """precompute_q_wall_sphere_3d evaluated with torch on `device` (float64
    arithmetic, the same operations as the numpy form), returned as tensors
    (q_wall in `dtype`, default float64; is_solid bool).  For grids whose
    per-link arrays are too large to build on the host."""
    import torch
    f64 = torch.float64
    shape = (Nz, Ny, Nx)
    x = (torch.arange(Nx, dtype=f64, device=device) - float(cx)).view(1, 1, Nx).expand(shape)
    y = (torch.arange(Ny, dtype=f64, device=device) - float(cy)).view(1, Ny, 1).expand(shape)
    z = (torch.arange(Nz, dtype=f64, device=device) - float(cz)).view(Nz, 1, 1).expand(shape)
    R2 = float(R) * float(R)
    solid = x * x + y * y + z * z <= R2
    qw = torch.zeros((19,) + shape, dtype=dtype or f64, device=device)
    for q in range(1, 19):
        c = (float(L.D3Q19_CX[q]), float(L.D3Q19_CY[q]), float(L.D3Q19_CZ[q]))
        xn, yn, zn = x + c[0], y + c[1], z + c[2]
        crosses = (~solid) & (xn * xn + yn * yn + zn * zn <= R2)
        a = c[0] * c[0] + c[1] * c[1] + c[2] * c[2]
        b = 2.0 * (x * c[0] + y * c[1] + z * c[2])
        cc = x * x + y * y + z * z - R2
        disc = b * b - 4.0 * a * cc
        ok = disc >= 0.0
        sd = torch.sqrt(torch.where(ok, disc, torch.zeros_like(disc)))
        den = torch.full_like(b, 2.0 * a)  # a true division, as the reference's
        t1 = (-b - sd) / den
        t2 = (-b + sd) / den
        t = torch.where(t1 > 0.0, t1, t2)
        keep = crosses & ok & (t > 0.0) & (t <= 1.0)
        qw[q] = torch.where(keep, t, torch.zeros_like(t)).to(qw.dtype)
        del xn, yn, zn, b, cc, disc, sd, t1, t2, t
    return qw, solid


class CutLinks:
    """Compact cut-link table on the device (kb_libb_links).

    Built once from the dense per-link arrays of a D3Q19 grid (torch CUDA
    tensors shaped like f, float64 or float32) and the solid mask; a step
    with it (`ops.fused_trt_libb_links_step_3d_`) reads one class byte per
    node and the link data of wall nodes only."""

    def __init__(self, is_solid, q_wall, uw_link_x, uw_link_y, uw_link_z):
        import ctypes as C

        import torch

        from . import ops
        from ._lib import call
        if q_wall.dim() != 4 or q_wall.shape[0] != 19:
            raise ValueError("q_wall must have shape (19, Nz, Ny, Nx)")
        for name, t in (("uw_link_x", uw_link_x), ("uw_link_y", uw_link_y),
                        ("uw_link_z", uw_link_z)):
            if t.dtype != q_wall.dtype or t.shape != q_wall.shape:
                raise ValueError(f"{name} must match q_wall in dtype and shape")
        if q_wall.dtype not in (torch.float64, torch.float32):
            raise ValueError("cut-link data must be float64 or float32")
        self.Nz, self.Ny, self.Nx = (int(n) for n in q_wall.shape[1:])
        self.dtype = ops.storage_dtype(q_wall)
        self._call = call
        self._h = C.c_void_p()
        call("kb_libb_links_create", C.byref(self._h), ops._mask(is_solid),
             ops._t(q_wall, "q_wall"), ops._t(uw_link_x, "uw_link_x"),
             ops._t(uw_link_y, "uw_link_y"), ops._t(uw_link_z, "uw_link_z"), self.Nx, self.Ny,
             self.Nz, self.dtype, ops._stream())

    @property
    def handle(self):
        return self._h

    def nodes_with_links(self) -> int:
        import ctypes as C
        n, dt = C.c_longlong(), C.c_int()
        self._call("kb_libb_links_info", self._h, C.byref(n), C.byref(dt))
        return int(n.value)

    def close(self):
        if self._h:
            self._call("kb_libb_links_destroy", self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
