"""FP64 numpy restatement of the consistent-initialisation iteration of the
MRT cavity (test infrastructure only).

No reference counterpart: Kraken.jl starts every run from rest.  The warm
start added beside it initialises f from a predicted (rho, u) and then
repeats the MRT cavity step with the collision's velocity held at u (the
iteration of Mei, Luo, Lallemand and d'Humieres 2006, "Consistent initial
conditions for lattice Boltzmann simulations").  The collision is
collide_mrt_2d! (src/kernels/collide_mrt_2d.jl:54-106) with u replaced by the
given field and the momentum reset to rho * u; the operation order follows
oracle/kb_oracle.c's or_collide_mrt_2d, so the FP64 kernel
(kb_cavity_mrt_init_step_2d) matches it bit for bit.
"""
from __future__ import annotations

import numpy as np

from . import oracle as orc


def mrt_collide_fixed_u(f, ux, uy, nu, s_e=1.4, s_eps=1.4, s_q=1.2):
    """MRT collision of f (9, Ny, Nx) with the equilibria at velocity (ux, uy)."""
    s_nu = 1.0 / (3.0 * nu + 0.5)
    f1, f2, f3, f4, f5, f6, f7, f8, f9 = (f[q] for q in range(9))
    rho = f1 + f2 + f3 + f4 + f5 + f6 + f7 + f8 + f9
    e = -4.0 * f1 - f2 - f3 - f4 - f5 + 2.0 * (f6 + f7 + f8 + f9)
    eps = 4.0 * f1 - 2.0 * (f2 + f3 + f4 + f5) + f6 + f7 + f8 + f9
    qx = -2.0 * f2 + 2.0 * f4 + f6 - f7 - f8 + f9
    qy = -2.0 * f3 + 2.0 * f5 + f6 + f7 - f8 - f9
    pxx = f2 - f3 + f4 - f5
    pxy = f6 - f7 + f8 - f9
    jx = rho * ux
    jy = rho * uy
    usq = ux * ux + uy * uy
    e_eq = -2.0 * rho + 3.0 * rho * usq
    eps_eq = rho - 3.0 * rho * usq
    qx_eq = -rho * ux
    qy_eq = -rho * uy
    pxx_eq = rho * (ux * ux - uy * uy)
    pxy_eq = rho * ux * uy
    es = e - s_e * (e - e_eq)
    ep = eps - s_eps * (eps - eps_eq)
    qxs = qx - s_q * (qx - qx_eq)
    qys = qy - s_q * (qy - qy_eq)
    ps = pxx - s_nu * (pxx - pxx_eq)
    pxys = pxy - s_nu * (pxy - pxy_eq)
    r, jxs, jys = rho, jx, jy
    c9, c36, c18, c6, c4, c12 = 1.0 / 9.0, 1.0 / 36.0, 1.0 / 18.0, 1.0 / 6.0, 1.0 / 4.0, 1.0 / 12.0
    out = np.empty_like(f)
    out[0] = c9 * r - c9 * es + c9 * ep
    out[1] = c9 * r - c36 * es - c18 * ep + c6 * jxs - c6 * qxs + c4 * ps
    out[2] = c9 * r - c36 * es - c18 * ep + c6 * jys - c6 * qys - c4 * ps
    out[3] = c9 * r - c36 * es - c18 * ep - c6 * jxs + c6 * qxs + c4 * ps
    out[4] = c9 * r - c36 * es - c18 * ep - c6 * jys + c6 * qys - c4 * ps
    out[5] = c9 * r + c18 * es + c36 * ep + c6 * jxs + c12 * qxs + c6 * jys + c12 * qys + c4 * pxys
    out[6] = c9 * r + c18 * es + c36 * ep - c6 * jxs - c12 * qxs + c6 * jys + c12 * qys - c4 * pxys
    out[7] = c9 * r + c18 * es + c36 * ep - c6 * jxs - c12 * qxs - c6 * jys - c12 * qys + c4 * pxys
    out[8] = c9 * r + c18 * es + c36 * ep + c6 * jxs + c12 * qxs - c6 * jys - c12 * qys - c4 * pxys
    return out


def cavity_mrt_init_step(f_in, ux, uy, nu, u_lid):
    """One iteration: pull with half-way bounce-back, Zou-He lid, fixed-u MRT."""
    fo = np.empty_like(f_in)
    orc.stream_2d(fo, f_in)
    orc.zou_he_north_2d(fo, u_lid)
    return mrt_collide_fixed_u(fo, ux, uy, nu)
