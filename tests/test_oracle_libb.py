"""Pins of the oracle's TRT + interpolated bounce-back (LI-BB V2) steps and of
the host-side cut-fraction geometry against the reference's own tests
(test/test_couette_libb_canary.jl, test/test_couette_libb_canary_3d.jl,
test/test_li_bb_2d.jl)."""
import numpy as np
import pytest

W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def couette_2d_setup(Nx, Ny, u_top, q_w):
    """planar_couette_libb_setup (test_couette_libb_canary.jl:55-79): solid
    rows j = 0 and Ny-1; the links of the rows next to them that point into
    the walls are cut at q_w, the top wall moves at u_top."""
    solid = np.zeros((Ny, Nx), np.uint8)
    solid[0] = 1
    solid[Ny - 1] = 1
    qw = np.zeros((9, Ny, Nx))
    ux = np.zeros((9, Ny, Nx))
    uy = np.zeros((9, Ny, Nx))
    for q in (4, 7, 8):          # reference q = 5, 8, 9 (pointing -y)
        qw[q, 1] = q_w
    for q in (2, 5, 6):          # reference q = 3, 6, 7 (pointing +y)
        qw[q, Ny - 2] = q_w
        ux[q, Ny - 2] = u_top
    return solid, qw, ux, uy


def wrap_x_2d(f):
    """wrap_periodic_x! (test_couette_libb_canary.jl:83-90)."""
    f[:, :, 0] = f[:, :, -2]
    f[:, :, -1] = f[:, :, 1]


def run_couette_2d(step, Nx=8, Ny=33, nu=0.1, u_top=0.01, steps=5000, q_w=0.5):
    solid, qw, uwx, uwy = couette_2d_setup(Nx, Ny, u_top, q_w)
    f_in = np.stack([np.full((Ny, Nx), W9[q]) for q in range(9)])
    wrap_x_2d(f_in)
    f_out = np.empty_like(f_in)
    rho, ux, uy = (np.zeros((Ny, Nx)) for _ in range(3))
    for _ in range(steps):
        step(f_out, f_in, rho, ux, uy, solid, qw, uwx, uwy, nu)
        wrap_x_2d(f_out)
        f_in, f_out = f_out, f_in
    return rho, ux, uy, f_in


def oracle_step_2d(orc):
    def step(f_out, f_in, rho, ux, uy, solid, qw, uwx, uwy, nu):
        sp, sm = orc.trt_rates(nu, 3 / 16)
        orc.fused_trt_libb_2d(f_out, f_in, rho, ux, uy, solid, qw, uwx, uwy, sp, sm)
    return step


def couette_errors(ux, uy, u_top, q_w, Ny):
    """Profile errors at the interior column (test_couette_libb_canary.jl:183-200)."""
    Nx = ux.shape[1]
    H = (Ny - 3) + 2 * q_w
    u_ana = np.array([u_top * (j - 2 + q_w) / H for j in range(2, Ny)])
    u_num = ux[1:Ny - 1, Nx // 2 - 1]
    uy_num = uy[1:Ny - 1, Nx // 2 - 1]
    err = u_num - u_ana
    return (np.sqrt(np.sum(err ** 2) / np.sum(u_ana ** 2)), np.max(np.abs(err)) / u_top,
            np.max(np.abs(uy_num)) / u_top, np.min(u_num[:len(u_num) // 2]))


@pytest.mark.parametrize("q_w,steps", [(0.5, 20000), (0.3, 10000), (0.7, 10000)])
def test_couette_2d_libb_v2(orc, q_w, steps):
    """"Planar Couette -- LI-BB V2" and "V2 off-center" testsets: the linear
    profile to 1e-4 relative (Ginzburg-exact TRT, Lambda = 3/16)."""
    _, ux, uy, _ = run_couette_2d(oracle_step_2d(orc), steps=steps, q_w=q_w)
    L2, Linf, uy_max, umin = couette_errors(ux, uy, 0.01, q_w, 33)
    assert np.all(np.isfinite(ux)) and np.all(np.isfinite(uy))
    assert L2 < 1e-4 and Linf < 1e-4
    assert uy_max < 1e-4 and umin >= 0


def couette_3d_setup(Nx, Ny, Nz, u_top, q_w):
    """planar_couette_3d_setup (test_couette_libb_canary_3d.jl:5-33)."""
    solid = np.zeros((Nz, Ny, Nx), np.uint8)
    solid[0] = 1
    solid[Nz - 1] = 1
    qw, ux, uy, uz = (np.zeros((19, Nz, Ny, Nx)) for _ in range(4))
    for q in (6, 13, 14, 17, 18):    # reference q = 7, 14, 15, 18, 19 (-z)
        qw[q, 1] = q_w
    for q in (5, 11, 12, 15, 16):    # reference q = 6, 12, 13, 16, 17 (+z)
        qw[q, Nz - 2] = q_w
        ux[q, Nz - 2] = u_top
    return solid, qw, ux, uy, uz


def wrap_xy_3d(f):
    """wrap_periodic_xy_3d! (test_couette_libb_canary_3d.jl:37-49)."""
    f[:, :, :, 0] = f[:, :, :, -2]
    f[:, :, :, -1] = f[:, :, :, 1]
    f[:, :, 0, :] = f[:, :, -2, :]
    f[:, :, -1, :] = f[:, :, 1, :]


def run_couette_3d(step, Nx=4, Ny=4, Nz=33, nu=0.1, u_top=0.01, steps=10000, q_w=0.5):
    solid, qw, wx, wy, wz = couette_3d_setup(Nx, Ny, Nz, u_top, q_w)
    f_in = np.stack([np.full((Nz, Ny, Nx), W19[q]) for q in range(19)])
    wrap_xy_3d(f_in)
    f_out = np.empty_like(f_in)
    m = [np.zeros((Nz, Ny, Nx)) for _ in range(4)]
    for _ in range(steps):
        step(f_out, f_in, m, solid, qw, wx, wy, wz, nu)
        wrap_xy_3d(f_out)
        f_in, f_out = f_out, f_in
    return m, f_in


def oracle_step_3d(orc):
    def step(f_out, f_in, m, solid, qw, wx, wy, wz, nu):
        sp, sm = orc.trt_rates(nu, 3 / 16)
        orc.fused_trt_libb_3d(f_out, f_in, m, solid, qw, wx, wy, wz, sp, sm)
    return step


@pytest.mark.slow
@pytest.mark.parametrize("q_w", [0.3, 0.5, 0.7])
def test_couette_3d_libb_v2(orc, q_w):
    """"Planar Couette 3D -- LI-BB V2" (test_couette_libb_canary_3d.jl:80-110)."""
    (rho, ux, uy, uz), _ = run_couette_3d(oracle_step_3d(orc), q_w=q_w)
    Nz, u_top = 33, 0.01
    H = (Nz - 3) + 2 * q_w
    u_ana = np.array([u_top * (k - 2 + q_w) / H for k in range(2, Nz)])
    col = (slice(1, Nz - 1), 1, 1)
    err = ux[col] - u_ana
    assert np.sqrt(np.sum(err ** 2) / np.sum(u_ana ** 2)) < 1e-4
    assert np.max(np.abs(err)) / u_top < 1e-4
    assert np.max(np.abs(uy[col])) / u_top < 1e-4 and np.max(np.abs(uz[col])) / u_top < 1e-4


def test_cylinder_geometry(pkg):
    """"precompute_q_wall_cylinder -- analytical geometry" (test_li_bb_2d.jl:6-41)."""
    Nx = Ny = 32
    qw, solid = pkg.libb.precompute_q_wall_cylinder(Nx, Ny, 15.5, 15.5, 4.0)
    assert qw.shape == (9, Ny, Nx) and solid.shape == (Ny, Nx)
    assert np.all(qw[1:, 0, 0] == 0.0) and not solid[0, 0]
    assert solid[15, 15]
    assert np.any((~solid) & np.any(qw[1:] > 0, axis=0))
    cut = qw[qw > 0]
    assert np.all((cut > 0) & (cut <= 1))
    for j in range(Ny):
        for i in range(Nx - 1):
            q_e, q_w = qw[1, j, i], qw[3, j, i + 1]
            if q_e > 0 and q_w > 0 and not solid[j, i] and not solid[j, i + 1]:
                assert abs(q_e + q_w - 1.0) < 1e-10


def _scalar_cut(x, y, cx, cy, R, c):
    """The reference's per-link quadratic (li_bb_2d.jl:292-311), node by node."""
    R2 = R * R
    dx, dy = x - cx, y - cy
    if (x + c[0] - cx) ** 2 + (y + c[1] - cy) ** 2 > R2:
        return 0.0
    a = c[0] * c[0] + c[1] * c[1]
    b = 2.0 * (dx * c[0] + dy * c[1])
    cc = dx * dx + dy * dy - R2
    disc = b * b - 4.0 * a * cc
    if disc < 0:
        return 0.0
    sd = np.sqrt(disc)
    t1, t2 = (-b - sd) / (2.0 * a), (-b + sd) / (2.0 * a)
    t = t1 if t1 > 0 else t2
    return t if 0 < t <= 1 else 0.0


def test_cylinder_geometry_matches_scalar_formula(pkg):
    cx, cy, R = 10.3, 8.7, 3.4
    qw, solid = pkg.libb.precompute_q_wall_cylinder(21, 17, cx, cy, R)
    cxs, cys = [0, 1, 0, -1, 0, 1, -1, -1, 1], [0, 0, 1, 0, -1, 1, 1, -1, -1]
    for j in range(17):
        for i in range(21):
            if solid[j, i]:
                assert (i - cx) ** 2 + (j - cy) ** 2 <= R * R
                continue
            for q in range(1, 9):
                assert qw[q, j, i] == _scalar_cut(float(i), float(j), cx, cy, R, (cxs[q], cys[q]))


def test_zero_flow_cylinder(orc, pkg):
    """"Zero flow stays zero with cylinder obstacle" (test_li_bb_2d.jl:43-66),
    on the V2 step."""
    Nx = Ny = 32
    qw, solid = pkg.libb.precompute_q_wall_cylinder(Nx, Ny, 15.5, 15.5, 4.0)
    uwx, uwy = pkg.libb.wall_velocity_rotating_cylinder(qw, 15.5, 15.5, 0.0)
    f_in = np.stack([np.full((Ny, Nx), W9[q]) for q in range(9)])
    f_out = np.empty_like(f_in)
    rho, ux, uy = (np.zeros((Ny, Nx)) for _ in range(3))
    sp, sm = orc.trt_rates(0.1, 3 / 16)
    m = solid.astype(np.uint8)
    for _ in range(200):
        orc.fused_trt_libb_2d(f_out, f_in, rho, ux, uy, m, qw, uwx, uwy, sp, sm)
        f_in, f_out = f_out, f_in
    fl = ~solid
    assert np.max(np.abs(ux[fl])) < 1e-10 and np.max(np.abs(uy[fl])) < 1e-10
    assert np.max(np.abs(rho[fl] - 1.0)) < 1e-10


def swirl(ux, uy, solid, cx, cy, R):
    """Mean azimuthal velocity on the ring r = R + 2 (test_li_bb_2d.jl:95-108)."""
    Ny, Nx = ux.shape
    ut = []
    for th in np.arange(0, 2 * np.pi + 1e-12, np.pi / 8):
        i = int(round(cx + (R + 2) * np.cos(th)))
        j = int(round(cy + (R + 2) * np.sin(th)))
        if 0 <= i < Nx and 0 <= j < Ny and not solid[j, i]:
            X, Y = float(i) - cx, float(j) - cy
            ut.append((-Y * ux[j, i] + X * uy[j, i]) / np.hypot(X, Y))
    return float(np.mean(ut))


@pytest.mark.slow
def test_rotating_cylinder_swirl(orc, pkg):
    """"Rotating cylinder drives a swirl" (test_li_bb_2d.jl:68-114) on the V2
    step: positive mean azimuthal velocity, bounded speed."""
    Nx = Ny = 48
    cx = cy = 23.5
    R, Om = 4.0, 0.002
    qw, solid = pkg.libb.precompute_q_wall_cylinder(Nx, Ny, cx, cy, R)
    uwx, uwy = pkg.libb.wall_velocity_rotating_cylinder(qw, cx, cy, Om)
    f_in = np.stack([np.full((Ny, Nx), W9[q]) for q in range(9)])
    f_out = np.empty_like(f_in)
    rho, ux, uy = (np.zeros((Ny, Nx)) for _ in range(3))
    sp, sm = orc.trt_rates(0.1, 3 / 16)
    m = solid.astype(np.uint8)
    for _ in range(2000):
        orc.fused_trt_libb_2d(f_out, f_in, rho, ux, uy, m, qw, uwx, uwy, sp, sm)
        f_in, f_out = f_out, f_in
    assert np.all(np.isfinite(ux))
    assert swirl(ux, uy, solid, cx, cy, R) > 0
    assert np.max(np.hypot(ux, uy)) < 0.02


def test_sphere_geometry_torch_form(pkg):
    """The device form of precompute_q_wall_sphere_3d agrees with the numpy
    form (same arithmetic; torch's CPU sqrt may differ in the last bit, so
    a few ulp here; the GPU test holds it to equality)."""
    import torch
    for args in [(13, 11, 9, 6.2, 5.1, 4.3, 3.7), (32, 30, 28, 15.5, 14.2, 13.9, 9.3)]:
        a, sa = pkg.libb.precompute_q_wall_sphere_3d(*args)
        b, sb = pkg.libb.precompute_q_wall_sphere_3d_torch(*args, device="cpu")
        assert np.array_equal(sa, sb.numpy())
        assert np.array_equal(a > 0, b.numpy() > 0)
        assert np.max(np.abs(a - b.numpy())) < 1e-14
    assert b.dtype == torch.float64
