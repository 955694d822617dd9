"""Pin the CPU oracle against the reference's own known answers.

Each test restates one assertion of Kraken.jl's test suite (file:line in the
docstring) and runs it on the oracle, so the oracle is checked before any
GPU result is compared with it.
"""
import math

import numpy as np
import pytest


def _eq_f2(orc, rho, ux, uy, shape):
    Ny, Nx = shape
    f = np.empty((9, Ny, Nx))
    for q in range(9):
        f[q] = orc.equilibrium_d2q9(rho, ux, uy, q)
    return f


def test_lattice_constants(pkg):
    """test/test_lbm_basic.jl:6-36"""
    L = pkg.lattice
    assert abs(L.D2Q9_W.sum() - 1.0) < 1e-14
    assert abs(L.D3Q19_W.sum() - 1.0) < 1e-14
    assert np.all(L.D2Q9_OPP[L.D2Q9_OPP] == np.arange(9))
    assert np.all(L.D3Q19_OPP[L.D3Q19_OPP] == np.arange(19))
    for q in range(19):
        o = L.D3Q19_OPP[q]
        assert (L.D3Q19_CX[o], L.D3Q19_CY[o], L.D3Q19_CZ[o]) == \
            (-L.D3Q19_CX[q], -L.D3Q19_CY[q], -L.D3Q19_CZ[q])


def test_equilibrium_moments(orc, pkg):
    """test/test_lbm_basic.jl:38-77"""
    L = pkg.lattice
    for q in range(9):
        assert abs(orc.equilibrium_d2q9(1.0, 0.0, 0.0, q) - L.D2Q9_W[q]) < 1e-14
    rho, ux, uy = 2.5, 0.05, -0.03
    f = [orc.equilibrium_d2q9(rho, ux, uy, q) for q in range(9)]
    assert abs(sum(f) - rho) < 1e-12
    assert abs(sum(fq * c for fq, c in zip(f, L.D2Q9_CX)) - rho * ux) < 1e-12
    assert abs(sum(fq * c for fq, c in zip(f, L.D2Q9_CY)) - rho * uy) < 1e-12
    rho, ux, uy, uz = 1.8, 0.02, -0.01, 0.03
    f = [orc.equilibrium_d3q19(rho, ux, uy, uz, q) for q in range(19)]
    assert abs(sum(f) - rho) < 1e-12
    for c, u in ((L.D3Q19_CX, ux), (L.D3Q19_CY, uy), (L.D3Q19_CZ, uz)):
        assert abs(sum(fq * cq for fq, cq in zip(f, c)) - rho * u) < 1e-12


def test_trt_rates(orc, pkg):
    """test/test_fused_trt_2d.jl:6-27 (oracle and the library's host helper)."""
    for rates in (orc.trt_rates, pkg.trt_rates):
        sp, sm = rates(1 / 6, 3 / 16)
        assert abs(sp - 1.0) < 1e-12 and abs(sm - 8 / 7) < 1e-12
        nu = 0.01
        s = 1.0 / (3 * nu + 0.5)
        sp, sm = rates(nu, (1 / s - 0.5) ** 2)
        assert abs(sp - sm) < 1e-12 and abs(sm - s) < 1e-12


def test_trt_equals_bgk(orc):
    """test/test_fused_trt_2d.jl:29-65: TRT with Lambda=(1/s-1/2)^2 == BGK, 50 steps."""
    N, nu = 16, 0.02
    s = 1.0 / (3 * nu + 0.5)
    lam = (1 / s - 0.5) ** 2
    sp, sm = orc.trt_rates(nu, lam)
    f0 = np.empty((9, N, N))
    for i in range(N):
        u = 0.01 * math.sin(2 * math.pi * i / N)
        for q in range(9):
            f0[q, :, i] = orc.equilibrium_d2q9(1.0, u, 0.0, q)
    ft, fb = f0.copy(), f0.copy()
    ot, ob = np.empty_like(f0), np.empty_like(f0)
    mt = [np.zeros((N, N)) for _ in range(3)]
    mb = [np.zeros((N, N)) for _ in range(3)]
    solid = np.zeros((N, N), np.uint8)
    for _ in range(50):
        orc.fused_trt_2d(ot, ft, *mt, solid, sp, sm)
        orc.fused_bgk_2d(ob, fb, *mb, solid, s)
        ft, ot = ot, ft
        fb, ob = ob, fb
    assert np.max(np.abs(ft - fb)) < 1e-12
    assert np.max(np.abs(mt[1] - mb[1])) < 1e-12
    assert np.max(np.abs(mt[0] - mb[0])) < 1e-12


def test_trt_equilibrium_stationary(orc):
    """test/test_fused_trt_2d.jl:67-84"""
    N = 16
    f = _eq_f2(orc, 1.0, 0.0, 0.0, (N, N))
    f0, out = f.copy(), np.empty_like(f)
    m = [np.zeros((N, N)) for _ in range(3)]
    sp, sm = orc.trt_rates(0.02, 3 / 16)
    for _ in range(100):
        orc.fused_trt_2d(out, f, *m, None, sp, sm)
        f, out = out, f
    assert np.max(np.abs(f - f0)) < 1e-12
    assert np.max(np.abs(m[1])) < 1e-12 and np.max(np.abs(m[0] - 1)) < 1e-12


def test_trt_dissipates(orc):
    """test/test_fused_trt_2d.jl:86-110"""
    N, nu, u0 = 48, 0.02, 0.01
    k = 2 * math.pi / N
    f = np.empty((9, N, N))
    ux0 = np.empty((N, N)); uy0 = np.empty((N, N))
    for j in range(N):
        for i in range(N):
            a = -u0 * math.cos(k * i) * math.sin(k * j)
            b = u0 * math.sin(k * i) * math.cos(k * j)
            ux0[j, i], uy0[j, i] = a, b
            for q in range(9):
                f[q, j, i] = orc.equilibrium_d2q9(1.0, a, b, q)
    out = np.empty_like(f)
    m = [np.zeros((N, N)) for _ in range(3)]
    sp, sm = orc.trt_rates(nu, 3 / 16)
    ke0 = float(np.sum(ux0 ** 2 + uy0 ** 2))
    for _ in range(500):
        orc.fused_trt_2d(out, f, *m, None, sp, sm)
        f, out = out, f
    ke = float(np.sum(m[1] ** 2 + m[2] ** 2))
    assert np.all(np.isfinite(m[1])) and 0 < ke < ke0


def test_mass_conservation_2d(orc):
    """test/test_lbm_basic.jl:79-87: 16^2 cavity, 100 steps, < 1 %."""
    N, nu, u = 16, 0.1, 0.05
    f = _eq_f2(orc, 1.0, 0.0, 0.0, (N, N))
    rho, _, _ = orc.run_cavity_2d(f, N, N, 1 / (3 * nu + 0.5), u, 100)
    assert abs(rho.sum() - N * N) / (N * N) < 0.01


def test_mass_conservation_3d(orc, pkg):
    """test/test_lbm_basic.jl:89-98: 8^3 cavity, 50 steps, < 1 %."""
    N, nu = 8, 0.1
    f = np.empty((19, N, N, N))
    for q in range(19):
        f[q] = pkg.lattice.D3Q19_W[q]
    rho, *_ = orc.run_cavity_3d(f, 1 / (3 * nu + 0.5), 0.05, 50)
    assert abs(rho.sum() - N ** 3) / N ** 3 < 0.01


def _ghia_err(ux, pins_entry, u_lid):
    N = ux.shape[0]
    ic = N // 2 - 1  # Julia i_center = N ÷ 2 (1-based)
    err = 0.0
    for yg, ug in zip(pins_entry["y"], pins_entry["u"]):
        j = min(max(round(yg * (N - 1)) + 1, 1), N) - 1
        err = max(err, abs(ux[j, ic] / u_lid - ug))
    return err


@pytest.mark.slow
def test_cavity_ghia_re100(orc, pins):
    """test/test_cavity.jl:6-40: 128^2, Re=100, 30000 steps, max centreline error < 0.1."""
    N, u_lid = 128, 0.1
    nu = u_lid * N / 100.0
    f = _eq_f2(orc, 1.0, 0.0, 0.0, (N, N))
    _, ux, _ = orc.run_cavity_2d(f, N, N, 1 / (3 * nu + 0.5), u_lid, 30000)
    assert _ghia_err(ux, pins["ghia_re100"], u_lid) < 0.1


@pytest.mark.slow
def test_mrt_cavity_ghia(orc, pins):
    """test/test_mrt.jl:6-45: 64^2, Re=100, 15000 steps, error < 0.15."""
    N, u_lid = 64, 0.1
    nu = u_lid * N / 100.0
    f = _eq_f2(orc, 1.0, 0.0, 0.0, (N, N))
    fo = np.empty_like(f)
    for _ in range(15000):
        orc.stream_2d(fo, f)
        orc.zou_he_north_2d(fo, u_lid)
        orc.collide_mrt_2d(fo, None, nu)
        f, fo = fo, f
    _, ux, _ = orc.macroscopic_2d(f)
    assert np.all(np.isfinite(ux))
    assert _ghia_err(ux, pins["ghia_re100_mrt"], u_lid) < 0.15


def test_taylor_green_2d(orc, pkg):
    """test/test_taylor_green.jl:4-38: N=64, nu=0.01, 1000 steps, L2 < 5 %."""
    N, nu, u0, steps = 64, 0.01, 0.01, 1000
    f = pkg.drivers.taylor_green_2d_populations(N, u0)
    fo = np.empty_like(f)
    w = 1.0 / (3 * nu + 0.5)
    for _ in range(steps):
        orc.stream_fully_periodic_2d(fo, f)
        orc.collide_2d(fo, None, w)
        f, fo = fo, f
    _, ux, _ = orc.macroscopic_2d(f)
    k = 2 * math.pi / N
    x = np.arange(N)[None, :]; y = np.arange(N)[:, None]
    ua = -u0 * np.cos(k * x) * np.sin(k * y) * math.exp(-2 * nu * k * k * steps)
    l2 = math.sqrt(np.sum((ux - ua) ** 2) / np.sum(ua ** 2))
    assert l2 < 0.05
    assert np.max(np.abs(ux)) < u0


def test_cavity_3d_lid(orc, pkg):
    """test/test_cavity_3d.jl:7-44: 32^3, Re=100, 2000 steps; lid mean, no overshoot."""
    N, u_lid, nu = 32, 0.1, 0.032
    f = np.empty((19, N, N, N))
    for q in range(19):
        f[q] = pkg.lattice.D3Q19_W[q]
    rho, ux, uy, uz = orc.run_cavity_3d(f, 1 / (3 * nu + 0.5), u_lid, 2000)
    assert np.all(np.isfinite(rho)) and abs(rho.mean() - 1) < 0.05
    top = ux[N - 1, 1:N - 1, 1:N - 1]
    assert abs(top.mean() - u_lid) / u_lid < 0.1
    assert np.max(np.abs(ux)) <= 1.05 * u_lid


def test_zou_he_all_faces_rest(orc, pkg):
    """test/test_cavity_3d.jl:46-90: zero-velocity Zou-He on 6 faces keeps rest."""
    N, nu = 8, 0.1
    f = np.empty((19, N, N, N))
    for q in range(19):
        f[q] = pkg.lattice.D3Q19_W[q]
    fo = np.empty_like(f)
    w = 1 / (3 * nu + 0.5)
    for _ in range(500):
        orc.stream_3d(fo, f)
        for face in ("top", "bottom", "west", "east", "south", "north"):
            orc.zou_he_velocity_3d(fo, face, 0.0, 0.0, 0.0)
        orc.collide_3d(fo, None, w)
        f, fo = fo, f
    rho, ux, uy, uz = orc.macroscopic_3d(f)
    assert abs(rho.mean() - 1) < 1e-3
    assert max(np.max(np.abs(ux)), np.max(np.abs(uy)), np.max(np.abs(uz))) < 1e-10


def test_natconv_zero_buoyancy(orc, pkg):
    """With zero buoyancy the fused natural-convection step leaves the flow at
    rest to round-off (Guo source and velocity vanish) and the temperature
    relaxes to a profile that falls monotonically from the hot to the cold
    Dirichlet wall (fused_thermal_2d.jl:37-57 anti-bounce-back)."""
    N = 8
    p = pkg.drivers.natconv_parameters(N, 0.0, 0.71)
    f = _eq_f2(orc, 1.0, 0.0, 0.0, (N, N))
    f0 = f.copy()
    g = np.empty((9, N, N))
    for q in range(9):
        g[q] = pkg.lattice.D2Q9_W[q] * 0.5
    fo, go, T = np.empty_like(f), np.empty_like(g), np.empty((N, N))
    for _ in range(6000):
        orc.fused_natconv_2d(fo, f, go, g, T, p["omega_f"], p["omega_T"], 0.0, 0.5, 1.0, 0.0)
        f, fo = fo, f
        g, go = go, g
    assert np.max(np.abs(f - f0)) < 1e-14
    T = orc.temperature_2d(g)
    assert np.all(np.diff(T, axis=1) < 0) and 0.0 < T.min() and T.max() < 1.0
    assert abs(pkg.drivers.nusselt_hot_wall(T) - 1.0) < 0.05


@pytest.mark.slow
def test_natconv_de_vahl_davis(orc, pkg, pins):
    """test/test_thermal.jl:388-404: N=64, Ra=1e3, 30000 steps, Nu within 0.5 %."""
    N, Ra, steps = 64, 1e3, 30000
    p = pkg.drivers.natconv_parameters(N, Ra, 0.71)
    f = _eq_f2(orc, 1.0, 0.0, 0.0, (N, N))
    g = pkg.drivers.natconv_initial_g(N)
    fo, go, T = np.empty_like(f), np.empty_like(g), np.empty((N, N))
    for _ in range(steps):
        orc.fused_natconv_2d(fo, f, go, g, T, p["omega_f"], p["omega_T"], p["beta_g"], p["T_ref"],
                             1.0, 0.0)
        f, fo = fo, f
        g, go = go, g
    T = orc.temperature_2d(g)
    nu_ref = pins["natconv_ra1e3_nu_ref"]
    assert abs(pkg.drivers.nusselt_hot_wall(T) - nu_ref) / nu_ref < 0.005
