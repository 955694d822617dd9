"""Pins of the oracle's unfused thermal DDF against the reference's own tests
(test/test_thermal.jl), run on the CPU restatement.  Each test names the
reference testset whose assertions it repeats."""
import numpy as np
import pytest

from oracle import thermal_drivers as td

W9 = td.W9
W19 = td.W19
C9 = (np.array([0, 1, 0, -1, 0, 1, -1, -1, 1]), np.array([0, 0, 1, 0, -1, 1, 1, -1, -1]))
OPP9 = [0, 3, 4, 1, 2, 7, 8, 5, 6]
C19 = (np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0]),
       np.array([0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1]),
       np.array([0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1]))
OPP19 = [0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15]


def test_heat_conduction_1d(orc):
    """"Heat conduction 1D" (test_thermal.jl:6-46): periodic x, hot south,
    cold north, u = 0; the half-way linear profile to 1e-7 after 5000 steps."""
    Nx, Ny, alpha = 4, 32, 0.1
    wT = 1.0 / (3.0 * alpha + 0.5)
    g_in = np.stack([np.full((Ny, Nx), W9[q] * 0.5) for q in range(9)])
    g_out = g_in.copy()
    u0 = np.zeros((Ny, Nx))
    for _ in range(5000):
        orc.stream_periodic_x_wall_y_2d(g_out, g_in)
        orc.fixed_temp_face_2d(g_out, "south", 1.0)
        orc.fixed_temp_face_2d(g_out, "north", 0.0)
        orc.collide_thermal_2d(g_out, u0, u0, wT)
        g_in, g_out = g_out, g_in
    T = orc.temperature_2d(g_in)[:, 1]
    ana = 1.0 - (np.arange(1, Ny + 1) - 0.5) / Ny
    assert np.max(np.abs(T - ana)) < 1e-7


def _stream_one_wall_axis(g_in, c, opp, wall_axis):
    """Pull streaming periodic on every axis but `wall_axis`, where a source
    outside the box is the node's own opposite population
    (test_thermal.jl:60-74).  Arrays are (q, ..., x) with the axes reversed."""
    D = g_in.ndim - 1
    g_out = np.empty_like(g_in)
    for q in range(g_in.shape[0]):
        src = g_in[q]
        for d in range(D):
            src = np.roll(src, c[d][q], axis=D - 1 - d)
        n = g_in.shape[D - wall_axis]
        idx = np.arange(n) - c[wall_axis][q]
        outside = (idx < 0) | (idx >= n)
        shape = [1] * D
        shape[D - 1 - wall_axis] = n
        outside = outside.reshape(shape)
        g_out[q] = np.where(outside, g_in[opp[q]], src)
    return g_out


@pytest.mark.parametrize("name,D,wall_axis,faces", [
    ("2D west/east", 2, 0, ("west", "east")),
    ("2D south/north", 2, 1, ("south", "north")),
    ("3D west/east", 3, 0, ("west", "east")),
    ("3D south/north", 3, 1, ("south", "north")),
    ("3D bottom/top", 3, 2, ("bottom", "top")),
])
def test_halfway_dirichlet_pure_conduction(orc, name, D, wall_axis, faces):
    """"Half-way Dirichlet walls: pure conduction to round-off"
    (test_thermal.jl:48-143): steady linear profile to 1e-12, Nu = 1 to 1e-10,
    wall value from linear extrapolation to 1e-12."""
    T_a, T_b = 0.8, 0.2
    wT = 1.0 / (3.0 * 0.1 + 0.5)
    N_wall, N_side, steps = 8, 3, 3000
    dims = [N_wall if d == wall_axis else N_side for d in range(D)]
    shape = tuple(reversed(dims))
    Q, W, c, opp = (9, W9, C9, OPP9) if D == 2 else (19, W19, C19, OPP19)
    g_in = np.stack([np.full(shape, W[q] * 0.5) for q in range(Q)])
    us = [np.zeros(shape) for _ in range(D)]
    face_fn = orc.fixed_temp_face_2d if D == 2 else orc.fixed_temp_face_3d
    for _ in range(steps):
        g_out = np.ascontiguousarray(_stream_one_wall_axis(g_in, c, opp, wall_axis))
        face_fn(g_out, faces[0], T_a)
        face_fn(g_out, faces[1], T_b)
        if D == 2:
            orc.collide_thermal_2d(g_out, *us, wT)
        else:
            orc.collide_thermal_3d(g_out, *us, wT)
        g_in = g_out
    Temp = orc.temperature_2d(g_in) if D == 2 else orc.temperature_3d(g_in)
    pos = np.arange(1, N_wall + 1)
    lin = T_a + (T_b - T_a) * (pos - 0.5) / N_wall
    prof = np.moveaxis(Temp, D - 1 - wall_axis, -1)
    assert np.max(np.abs(prof - lin)) < 1e-12, name
    line = prof.reshape(-1, N_wall)[0]
    T1, T2 = line[0], line[1]
    Nu = -N_wall * (-8 * T_a + 9 * T1 - T2) / 3 / (T_a - T_b)
    assert abs(Nu - 1) < 1e-10
    assert abs(1.5 * T1 - 0.5 * T2 - T_a) < 1e-12


FACES = (("west", 0, True), ("east", 0, False), ("south", 1, True), ("north", 1, False),
         ("bottom", 2, True), ("top", 2, False))


def expected_fixed_temp(g0, temps):
    """The reference's `_expected_fixed_temp` (test_thermal.jl:149-171), built
    from the lattice velocities alone: a slot whose link comes from outside
    the box through Dirichlet faces gets -g0 + 2 w_q mean(T of those faces)."""
    D = g0.ndim - 1
    Q = g0.shape[0]
    c, W = (C9, W9) if Q == 9 else (C19, W19)
    dims = list(reversed(g0.shape[1:]))
    g = g0.copy()
    for q in range(Q):
        for I in np.ndindex(*dims):
            crossed = []
            for face, d, low in FACES:
                if d >= D or temps.get(face) is None:
                    continue
                src = I[d] - c[d][q]
                if (src < 0) if low else (src > dims[d] - 1):
                    crossed.append(temps[face])
            if crossed:
                at = (q,) + tuple(reversed(I))
                g[at] = -g0[at] + 2 * W[q] * sum(crossed) / len(crossed)
    return g


def test_adjacent_dirichlet_faces_2d(orc):
    """"Adjacent Dirichlet faces ... 2D kernels against the reference"
    (test_thermal.jl:175-207)."""
    Nx, Ny = 5, 4
    g0 = np.random.default_rng(0).random((9, Ny, Nx))
    for face, t in (("west", 0.9), ("east", 0.1), ("south", 0.7), ("north", 0.3)):
        g_one = g0.copy()
        orc.fixed_temp_face_2d(g_one, face, t)
        g_all = g0.copy()
        orc.fixed_temp_2d(g_all, **{face: t})
        assert np.array_equal(g_all, g_one)
        assert np.max(np.abs(g_all - expected_fixed_temp(g0, {face: t}))) < 1e-15
    for temps in (dict(west=0.9, east=0.1, south=0.7, north=0.3), dict(west=0.9, south=0.7),
                  dict(east=0.1, north=0.3), dict(west=0.9, north=0.3, east=0.1)):
        g = g0.copy()
        orc.fixed_temp_2d(g, **temps)
        assert np.max(np.abs(g - expected_fixed_temp(g0, temps))) < 1e-15
    g = g0.copy()
    orc.fixed_temp_2d(g, west=0.9, east=0.1, south=0.7, north=0.3)
    assert abs(g[5, 0, 0] - (-g0[5, 0, 0] + (0.9 + 0.7) / 36)) < 1e-15
    assert abs(g[8, Ny - 1, 0] - (-g0[8, Ny - 1, 0] + (0.9 + 0.3) / 36)) < 1e-15
    assert abs(g[6, 0, Nx - 1] - (-g0[6, 0, Nx - 1] + (0.1 + 0.7) / 36)) < 1e-15
    assert abs(g[7, Ny - 1, Nx - 1] - (-g0[7, Ny - 1, Nx - 1] + (0.1 + 0.3) / 36)) < 1e-15


def test_adjacent_dirichlet_faces_3d(orc):
    """"Adjacent Dirichlet faces ... 3D kernels against the reference"
    (test_thermal.jl:209-238)."""
    Nx, Ny, Nz = 4, 5, 3
    g0 = np.random.default_rng(1).random((19, Nz, Ny, Nx))
    all_t = dict(west=0.9, east=0.1, south=0.7, north=0.3, bottom=0.6, top=0.2)
    for face, t in all_t.items():
        g_one = g0.copy()
        orc.fixed_temp_face_3d(g_one, face, t)
        g_all = g0.copy()
        orc.fixed_temp_3d(g_all, **{face: t})
        assert np.array_equal(g_all, g_one)
        assert np.max(np.abs(g_all - expected_fixed_temp(g0, {face: t}))) < 1e-15
    for temps in (all_t, dict(west=0.9, south=0.7, top=0.2), dict(east=0.1, north=0.3, bottom=0.6),
                  dict(south=0.7, bottom=0.6, top=0.2)):
        g = g0.copy()
        orc.fixed_temp_3d(g, **temps)
        assert np.max(np.abs(g - expected_fixed_temp(g0, temps))) < 1e-15


def test_square_hot_west_south(orc):
    """"2D square, hot west and south, cold east and north"
    (test_thermal.jl:243-274)."""
    T_w, T_c = 0.8, 0.2
    wT = 1.0 / (3.0 * 0.1 + 0.5)
    N = 12
    g_in = np.stack([np.full((N, N), W9[q] * 0.5) for q in range(9)])
    g_out = g_in.copy()
    u0 = np.zeros((N, N))
    bc = dict(west=T_w, south=T_w, east=T_c, north=T_c)
    for _ in range(6000):
        orc.stream_2d(g_out, g_in)
        orc.fixed_temp_2d(g_out, **bc)
        orc.collide_thermal_2d(g_out, u0, u0, wT)
        g_in, g_out = g_out, g_in
    T_prev = orc.temperature_2d(g_in)
    orc.stream_2d(g_out, g_in)
    orc.fixed_temp_2d(g_out, **bc)
    orc.collide_thermal_2d(g_out, u0, u0, wT)
    T = orc.temperature_2d(g_out)
    assert np.max(np.abs(T - T_prev)) < 1e-13
    assert np.max(np.abs(T - T.T)) < 1e-13
    assert T.min() >= T_c - 1e-13 and T.max() <= T_w + 1e-13
    assert abs(T[N - 1, 0] - 0.5 * (T_w + T_c)) < 1e-13


def test_cube_hot_west_south_bottom(orc):
    """"3D cube, hot west, south and bottom, cold east, north and top"
    (test_thermal.jl:276-308)."""
    T_w, T_c = 0.8, 0.2
    wT = 1.0 / (3.0 * 0.1 + 0.5)
    N = 6
    g_in = np.stack([np.full((N, N, N), W19[q] * 0.5) for q in range(19)])
    g_out = g_in.copy()
    u0 = np.zeros((N, N, N))
    bc = dict(west=T_w, south=T_w, bottom=T_w, east=T_c, north=T_c, top=T_c)
    for _ in range(3000):
        orc.stream_3d(g_out, g_in)
        orc.fixed_temp_3d(g_out, **bc)
        orc.collide_thermal_3d(g_out, u0, u0, u0, wT)
        g_in, g_out = g_out, g_in
    T_prev = orc.temperature_3d(g_in)
    orc.stream_3d(g_out, g_in)
    orc.fixed_temp_3d(g_out, **bc)
    orc.collide_thermal_3d(g_out, u0, u0, u0, wT)
    T = orc.temperature_3d(g_out)
    assert np.max(np.abs(T - T_prev)) < 1e-13
    for perm in ((0, 2, 1), (2, 1, 0), (1, 0, 2)):
        assert np.max(np.abs(T - np.transpose(T, perm))) < 1e-13
    assert T.min() >= T_c - 1e-13 and T.max() <= T_w + 1e-13


@pytest.mark.slow
def test_rayleigh_benard_onset(orc):
    """"Rayleigh-Benard onset" (test_thermal.jl:339-356): above Ra_c the
    vertical velocity grows far beyond the sub-critical one."""
    sub = td.run_rayleigh_benard_2d(64, 16, 1000.0, max_steps=10000)
    sup = td.run_rayleigh_benard_2d(64, 16, 5000.0, max_steps=20000)
    assert np.max(np.abs(sup["uy"])) > 5 * np.max(np.abs(sub["uy"]))
    assert np.all(np.isfinite(sub["Temp"])) and np.all(np.isfinite(sup["Temp"]))


def test_arrhenius_kernel_stable(orc):
    """"nu(T) Arrhenius kernel" (test_thermal.jl:358-385): 500 steps of
    periodic-x streaming and collide_boussinesq_vt_2d! stay finite."""
    Nx, Ny = 4, 32
    nu_ref, T_ref, A = 0.05, 1.0, 0.5
    f_in = np.stack([np.full((Ny, Nx), W9[q]) for q in range(9)])
    f_out = f_in.copy()
    Temp = np.repeat((1.2 - 0.4 * np.arange(Ny) / (Ny - 1))[:, None], Nx, axis=1)
    solid = np.zeros((Ny, Nx), np.uint8)
    for _ in range(500):
        orc.stream_periodic_x_wall_y_2d(f_out, f_in)
        orc.collide_boussinesq_vt_2d(f_out, Temp, solid, nu_ref, T_ref, A, 0.0)
        f_in, f_out = f_out, f_in
    rho, ux, _ = orc.macroscopic_2d(f_in)
    assert np.all(np.isfinite(rho)) and np.all(np.isfinite(ux))


@pytest.mark.slow
def test_box_pure_conduction_3d(orc):
    """"Pure conduction in the cavity drivers", 3D part (test_thermal.jl:330-336):
    run_natural_convection_3d at Ra = 0, N = 12: |Nu - 1| < 3e-3 and the
    mid-line within 4e-4 of the half-way linear profile."""
    r = td.run_natural_convection_3d(12, 0.0, max_steps=6000)
    d3 = max(abs(r["Temp"][5, 5, i] - (1 - (i + 0.5) / 12)) for i in range(12))
    assert abs(r["Nu"] - 1) < 3e-3
    assert d3 < 4e-4
