"""CPU FP64 restatement of the reference's unfused thermal DDF drivers.

TEST INFRASTRUCTURE ONLY: the tests use these loops as the checker of the
B200 drivers; the product never calls them.

run_rayleigh_benard_2d follows src/drivers/thermal.jl:31-144 and
run_natural_convection_3d follows src/drivers/thermal.jl:455-537, step for
step, on the kernels of kb_oracle.c.  Arrays are (q, Ny, Nx) / (q, Nz, Ny, Nx).
"""
from __future__ import annotations

import math

import numpy as np

from . import oracle as orc

W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def rb_parameters(Nx, Ny, Ra, Pr, T_hot=1.0, T_cold=0.0, nu=None, alpha=None,
                  orientation="vertical"):
    """thermal.jl:41-64"""
    dT = T_hot - T_cold
    H = Ny if orientation == "vertical" else Nx
    nu_v = 0.05 if nu is None else float(nu)
    alpha_v = nu_v / Pr if alpha is None else float(alpha)
    return dict(nu=nu_v, alpha=alpha_v, beta_g=Ra * nu_v * alpha_v / (dT * H ** 3),
                omega_f=1.0 / (3.0 * nu_v + 0.5), omega_T=1.0 / (3.0 * alpha_v + 0.5),
                T_ref=(T_hot + T_cold) / 2)


def rb_initial_g(Nx, Ny, T_hot=1.0, T_cold=0.0, orientation="vertical"):
    """thermal.jl:76-98, node by node as the reference loop writes it."""
    dT = T_hot - T_cold
    g = np.empty((9, Ny, Nx))
    for j in range(1, Ny + 1):
        for i in range(1, Nx + 1):
            if orientation == "vertical":
                T0 = T_hot - dT * (j - 0.5) / Ny
                T0 += (0.01 * dT) * math.sin(2 * math.pi * i / Nx) * math.sin(math.pi * j / Ny)
            else:
                T0 = T_hot - dT * (i - 0.5) / Nx
            for q in range(9):
                g[q, j - 1, i - 1] = W9[q] * T0
    return g


def run_rayleigh_benard_2d(Nx, Ny, Ra, Pr=1.0, T_hot=1.0, T_cold=0.0, max_steps=20000, nu=None,
                           alpha=None, orientation="vertical"):
    p = rb_parameters(Nx, Ny, Ra, Pr, T_hot, T_cold, nu, alpha, orientation)
    f_in = np.empty((9, Ny, Nx))
    for q in range(9):
        f_in[q] = W9[q]
    f_out = f_in.copy()
    g_in = rb_initial_g(Nx, Ny, T_hot, T_cold, orientation)
    g_out = g_in.copy()
    solid = np.zeros((Ny, Nx), np.uint8)
    stream = orc.stream_periodic_x_wall_y_2d if orientation == "vertical" else orc.stream_2d
    for _ in range(max_steps):
        stream(f_out, f_in)
        stream(g_out, g_in)
        if orientation == "vertical":
            orc.fixed_temp_face_2d(g_out, "south", T_hot)
            orc.fixed_temp_face_2d(g_out, "north", T_cold)
        else:
            orc.fixed_temp_face_2d(g_out, "west", T_hot)
            orc.fixed_temp_face_2d(g_out, "east", T_cold)
        Temp = orc.temperature_2d(g_out)
        _, ux, uy = orc.macroscopic_2d(f_out)
        orc.collide_thermal_2d(g_out, ux, uy, p["omega_T"])
        orc.collide_boussinesq_2d(f_out, Temp, solid, p["omega_f"], p["beta_g"], p["T_ref"])
        f_in, f_out = f_out, f_in
        g_in, g_out = g_out, g_in
    rho, ux, uy = orc.macroscopic_2d(f_in)
    return dict(rho=rho, ux=ux, uy=uy, Temp=orc.temperature_2d(g_in), f=f_in, g=g_in)


def run_natural_convection_3d(N, Ra, Pr=0.71, T_hot=1.0, T_cold=0.0, max_steps=10000):
    dT = T_hot - T_cold
    nu = 0.05
    alpha = nu / Pr
    beta_g = Ra * nu * alpha / (dT * float(N) ** 3)
    w_f, w_T, T_ref = 1.0 / (3.0 * nu + 0.5), 1.0 / (3.0 * alpha + 0.5), (T_hot + T_cold) / 2
    f_in = np.empty((19, N, N, N))
    g_in = np.empty((19, N, N, N))
    for i in range(1, N + 1):
        T0 = T_hot - dT * (i - 0.5) / N
        for q in range(19):
            g_in[q, :, :, i - 1] = W19[q] * T0
    for q in range(19):
        f_in[q] = W19[q]
    f_out, g_out = f_in.copy(), g_in.copy()
    solid = np.zeros((N, N, N), np.uint8)
    for _ in range(max_steps):
        orc.stream_3d(f_out, f_in)
        orc.stream_3d(g_out, g_in)
        orc.fixed_temp_face_3d(g_out, "west", T_hot)
        orc.fixed_temp_face_3d(g_out, "east", T_cold)
        Temp = orc.temperature_3d(g_out)
        _, ux, uy, uz = orc.macroscopic_3d(f_out)
        orc.collide_thermal_3d(g_out, ux, uy, uz, w_T)
        orc.collide_boussinesq_3d(f_out, Temp, solid, w_f, beta_g, T_ref)
        f_in, f_out = f_out, f_in
        g_in, g_out = g_out, g_in
    rho, ux, uy, uz = orc.macroscopic_3d(f_in)
    Temp = orc.temperature_3d(g_in)
    # thermal.jl:524-533
    nu_arr = np.zeros((N, N))
    for k in range(N):
        for j in range(N):
            dTdx = (-8 * T_hot + 9 * Temp[k, j, 0] - Temp[k, j, 1]) / 3.0
            nu_arr[k, j] = -float(N) * dTdx / dT
    Nu = float(np.sum(nu_arr[1:-1, 1:-1]) / max((N - 2) * (N - 2), 1))
    return dict(rho=rho, ux=ux, uy=uy, uz=uz, Temp=Temp, Nu=Nu, f=f_in, g=g_in)
