"""Pins of the oracle's Guo-forced collisions, force-corrected moments and the
x/z-periodic 3D stream against the reference's own tests
(test/test_poiseuille.jl, test/test_poiseuille_3d.jl, test/test_couette.jl)."""
import numpy as np

W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def oracle_poiseuille_2d(orc, Nx=4, Ny=32, nu=0.1, Fx=1e-5, steps=10000):
    """run_poiseuille_2d (src/drivers/basic.jl:185-203) on the oracle."""
    f_in = np.stack([np.full((Ny, Nx), W9[q]) for q in range(9)])
    f_out = np.empty_like(f_in)
    w = 1.0 / (3.0 * nu + 0.5)
    solid = np.zeros((Ny, Nx), np.uint8)
    for _ in range(steps):
        orc.stream_periodic_x_wall_y_2d(f_out, f_in)
        orc.collide_guo_2d(f_out, solid, w, Fx, 0.0)
        f_in, f_out = f_out, f_in
    rho, ux, uy = orc.macroscopic_2d(f_in)
    return rho, ux, uy, f_in


def oracle_couette_2d(orc, Nx=4, Ny=32, nu=0.1, u_wall=0.05, steps=30000):
    """run_couette_2d (src/drivers/basic.jl:213-234) on the oracle."""
    f_in = np.stack([np.full((Ny, Nx), W9[q]) for q in range(9)])
    f_out = np.empty_like(f_in)
    w = 1.0 / (3.0 * nu + 0.5)
    for _ in range(steps):
        orc.stream_periodic_x_wall_y_2d(f_out, f_in)
        orc.zou_he_south_2d(f_out, u_wall)
        orc.zou_he_north_2d(f_out, 0.0)
        orc.collide_2d(f_out, None, w)
        f_in, f_out = f_out, f_in
    rho, ux, uy = orc.macroscopic_2d(f_in)
    return rho, ux, uy, f_in


def poiseuille_err(ux_col, Ny, nu, Fx):
    """test_poiseuille.jl:10-20: L-inf error of the interior nodes relative to
    the peak of the half-way parabola."""
    u_ana = np.array([Fx / (2 * nu) * (j - 0.5) * (Ny + 0.5 - j) for j in range(1, Ny + 1)])
    return np.max(np.abs(ux_col[1:-1] - u_ana[1:-1])) / np.max(u_ana)


def test_poiseuille_2d(orc):
    """"Poiseuille 2D body force": 2 % L-inf, mass to 1e-3."""
    rho, ux, _, _ = oracle_poiseuille_2d(orc)
    assert poiseuille_err(ux[:, 1], 32, 0.1, 1e-5) < 0.02
    assert abs(rho.sum() - 4 * 32) / (4 * 32) < 1e-3


def test_couette_2d(orc):
    """"Couette 2D": the on-node Zou-He linear profile to 1e-10, u_y < 1e-6."""
    _, ux, uy, _ = oracle_couette_2d(orc)
    H = 31
    u_ana = np.array([0.05 * (1 - (j - 1) / H) for j in range(1, 33)])
    assert np.max(np.abs(ux[1:-1, 1] - u_ana[1:-1])) / 0.05 < 1e-10
    assert np.max(np.abs(uy)) < 1e-6


def oracle_poiseuille_3d(orc, Nx=4, Ny=32, Nz=4, nu=0.1, Fx=1e-5, steps=10000):
    """The loop of test_poiseuille_3d.jl:9-27 on the oracle."""
    f_in = np.stack([np.full((Nz, Ny, Nx), W19[q]) for q in range(19)])
    f_out = np.empty_like(f_in)
    w = 1.0 / (3.0 * nu + 0.5)
    solid = np.zeros((Nz, Ny, Nx), np.uint8)
    for _ in range(steps):
        orc.stream_periodic_xz_wall_y_3d(f_out, f_in)
        orc.collide_guo_3d(f_out, solid, w, Fx, 0.0, 0.0)
        m = orc.macroscopic_forced_3d(f_out, Fx, 0.0, 0.0)
        f_in, f_out = f_out, f_in
    return m, f_in


def test_poiseuille_3d(orc):
    """"Poiseuille 3D body force": 2 % L-inf, mass to 1e-3."""
    (rho, ux, _, _), _ = oracle_poiseuille_3d(orc)
    assert poiseuille_err(ux[1, :, 1], 32, 0.1, 1e-5) < 0.02
    assert abs(rho.sum() - 4 * 32 * 4) / (4 * 32 * 4) < 1e-3


def test_guo_field_equals_constant(orc):
    """A uniform force field gives the same bits as the constant-force kernel
    (2D and 3D), and the field moments equal the constant ones."""
    rng = np.random.default_rng(3)
    f = W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, 7, 5)))
    a, b = f.copy(), f.copy()
    orc.collide_guo_2d(a, None, 1.3, 2e-3, -1e-3)
    orc.collide_guo_field_2d(b, None, np.full((7, 5), 2e-3), np.full((7, 5), -1e-3), 1.3)
    assert np.array_equal(a, b)
    g = W19[:, None, None, None] * (1 + 0.05 * rng.standard_normal((19, 3, 4, 5)))
    a, b = g.copy(), g.copy()
    orc.collide_guo_3d(a, None, 1.2, 1e-3, 2e-3, -3e-3)
    F = [np.full((3, 4, 5), v) for v in (1e-3, 2e-3, -3e-3)]
    orc.collide_guo_field_3d(b, None, *F, 1.2)
    assert np.array_equal(a, b)
    m1 = orc.macroscopic_forced_3d(g, 1e-3, 2e-3, -3e-3)
    m2 = orc.macroscopic_forced_3d(g, *F)
    for x, y in zip(m1, m2):
        assert np.array_equal(x, y)


def test_guo_zero_force_is_bgk(orc):
    """With F = 0 the Guo collision is the plain BGK collide_2d! / collide_3d!."""
    rng = np.random.default_rng(4)
    f = W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, 6, 8)))
    a, b = f.copy(), f.copy()
    orc.collide_guo_2d(a, None, 1.4, 0.0, 0.0)
    orc.collide_2d(b, None, 1.4)
    assert np.max(np.abs(a - b)) < 1e-16
    g = W19[:, None, None, None] * (1 + 0.05 * rng.standard_normal((19, 3, 4, 5)))
    a, b = g.copy(), g.copy()
    orc.collide_guo_3d(a, None, 1.4, 0.0, 0.0, 0.0)
    orc.collide_3d(b, None, 1.4)
    assert np.max(np.abs(a - b)) < 1e-16
