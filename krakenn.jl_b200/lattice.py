"""D2Q9 / D3Q19 constants and equilibrium on the host (numpy, FP64).

src/lattice/d2q9.jl:17-67 and src/lattice/d3q19.jl:11-75; population
indices are 0-based here (reference index minus one).
"""
from __future__ import annotations

import numpy as np

D2Q9_W = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
D2Q9_CX = np.array([0, 1, 0, -1, 0, 1, -1, -1, 1])
D2Q9_CY = np.array([0, 0, 1, 0, -1, 1, 1, -1, -1])
D2Q9_OPP = np.array([0, 3, 4, 1, 2, 7, 8, 5, 6])

D3Q19_W = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)
D3Q19_CX = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0])
D3Q19_CY = np.array([0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1])
D3Q19_CZ = np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1])
D3Q19_OPP = np.array([0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15])

CS2 = 1.0 / 3.0


def equilibrium_d2q9(rho, ux, uy, q):
    """equilibrium(::D2Q9, rho, ux, uy, q) -- src/lattice/d2q9.jl:60-67"""
    w = D2Q9_W[q]
    cu = float(D2Q9_CX[q]) * ux + float(D2Q9_CY[q]) * uy
    usq = ux * ux + uy * uy
    return w * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq)


def equilibrium_d3q19(rho, ux, uy, uz, q):
    """equilibrium(::D3Q19, rho, ux, uy, uz, q) -- src/lattice/d3q19.jl:67-75"""
    w = D3Q19_W[q]
    cu = float(D3Q19_CX[q]) * ux + float(D3Q19_CY[q]) * uy + float(D3Q19_CZ[q]) * uz
    usq = ux * ux + uy * uy + uz * uz
    return w * rho * (1.0 + 3.0 * cu + 4.5 * cu * cu - 1.5 * usq)
