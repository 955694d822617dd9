"""Unfused thermal DDF parity (thermal_2d.jl / thermal_3d.jl kernels and the
Rayleigh-Benard and 3D natural-convection drivers) against the oracle.

FP64 kernels are bit-identical to the oracle, except the two nu(T) collisions
whose exp() comes from different math libraries (CUDA's on the GPU, the C
library's in the oracle): those are held to 1e-13 relative.  FP32 runs are
held to FP32 rounding bounds.
"""
import numpy as np
import pytest
import torch

from oracle import thermal_drivers as td

pytestmark = pytest.mark.gpu

SIZES2 = [(1, 1), (2, 3), (17, 13), (33, 7), (130, 9)]
SIZES3 = [(1, 1, 1), (3, 2, 5), (17, 5, 6), (33, 9, 4)]
W9 = td.W9
W19 = td.W19


def _g(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def _h(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _rand_pop(shape, W, seed, amp=0.05, base=1.0):
    rng = np.random.default_rng(seed)
    w = W.reshape((-1,) + (1,) * (len(shape) - 1))
    return w * base * (1.0 + amp * rng.standard_normal(shape))


def _field(shape, seed, scale=0.05):
    return scale * np.random.default_rng(seed).standard_normal(shape)


def _mask(shape, seed, frac=0.2):
    return (np.random.default_rng(seed + 77).random(shape) < frac).astype(np.uint8)


@pytest.mark.parametrize("Nx,Ny", SIZES2)
def test_collide_thermal_2d(cuda, pkg, orc, Nx, Ny):
    g = _rand_pop((9, Ny, Nx), W9, 1, base=0.7)
    ux, uy = _field((Ny, Nx), 2), _field((Ny, Nx), 3)
    ref = g.copy()
    orc.collide_thermal_2d(ref, ux, uy, 1.31)
    gt = _g(g)
    pkg.collide_thermal_2d_(gt, _g(ux), _g(uy), 1.31)
    assert np.array_equal(_h(gt), ref)
    # masked form: skipped nodes untouched, the rest as the oracle's loop form
    m = _mask((Ny, Nx), 4)
    ref = g.copy()
    orc.collide_thermal_masked_2d(ref, ux, uy, 1.31, m)
    gt = _g(g)
    pkg.collide_thermal_masked_2d_(gt, _g(ux), _g(uy), 1.31, _g(m, torch.uint8))
    out = _h(gt)
    assert np.array_equal(out, ref)
    assert np.array_equal(out[:, m.astype(bool)], g[:, m.astype(bool)])
    T = np.empty((Ny, Nx))
    Tt = _g(T)
    pkg.compute_temperature_2d_(Tt, _g(g))
    assert np.array_equal(_h(Tt), orc.temperature_2d(g))


@pytest.mark.parametrize("Nx,Ny", SIZES2)
def test_fixed_temp_2d(cuda, pkg, orc, Nx, Ny):
    g0 = np.random.default_rng(5).random((9, Ny, Nx))
    # every single face, with corner temperatures and skip flags
    for n, face in enumerate(("west", "east", "south", "north")):
        for skip in ((False, False), (True, False), (False, True), (True, True)):
            tc = (0.3 + 0.1 * n, 0.65 - 0.05 * n)
            ref = g0.copy()
            orc.fixed_temp_face_2d(ref, face, 0.9 - 0.2 * n, tc, skip)
            gt = _g(g0)
            pkg.ops._fixed_temp_face_2d_(gt, face, 0.9 - 0.2 * n, tc, skip)
            assert np.array_equal(_h(gt), ref), (face, skip)
    # the per-face public functions
    for face, fn in (("west", lambda t: pkg.apply_fixed_temp_west_2d_(t, 0.9, Ny)),
                     ("east", lambda t: pkg.apply_fixed_temp_east_2d_(t, 0.1, Nx, Ny)),
                     ("south", lambda t: pkg.apply_fixed_temp_south_2d_(t, 0.7, Nx)),
                     ("north", lambda t: pkg.apply_fixed_temp_north_2d_(t, 0.3, Nx, Ny))):
        ref = g0.copy()
        orc.fixed_temp_face_2d(ref, face, dict(west=0.9, east=0.1, south=0.7, north=0.3)[face])
        gt = _g(g0)
        fn(gt)
        assert np.array_equal(_h(gt), ref), face
    # all 16 Dirichlet face sets in one launch, corner rule
    temps = dict(west=0.9, east=0.1, south=0.7, north=0.3)
    for mask in range(16):
        sel = {k: v for n, (k, v) in enumerate(temps.items()) if mask >> n & 1}
        ref = g0.copy()
        orc.fixed_temp_2d(ref, **sel)
        gt = _g(g0)
        pkg.apply_fixed_temp_2d_(gt, Nx, Ny, **sel)
        assert np.array_equal(_h(gt), ref), sel


@pytest.mark.parametrize("Nx,Ny", SIZES2)
@pytest.mark.parametrize("with_mask", [False, True])
def test_collide_boussinesq_2d(cuda, pkg, orc, Nx, Ny, with_mask):
    f = _rand_pop((9, Ny, Nx), W9, 6)
    Temp = 0.5 + 0.3 * np.random.default_rng(7).random((Ny, Nx))
    m = _mask((Ny, Nx), 8) if with_mask else None
    mt = _g(m, torch.uint8) if m is not None else None
    ref = f.copy()
    orc.collide_boussinesq_2d(ref, Temp, m, 1.21, 3e-4, 0.5)
    ft = _g(f)
    pkg.collide_boussinesq_2d_(ft, _g(Temp), mt, 1.21, 3e-4, 0.5)
    assert np.array_equal(_h(ft), ref)
    # nu(T) forms: exp() of two math libraries, 1e-13 relative
    for o_fn, g_fn in (
            (lambda a: orc.collide_boussinesq_vt_2d(a, Temp, m, 0.05, 1.0, 0.5, 2e-4),
             lambda t: pkg.collide_boussinesq_vt_2d_(t, _g(Temp), mt, 0.05, 1.0, 0.5, 2e-4)),
            (lambda a: orc.collide_boussinesq_vt_modified_2d(a, Temp, m, 0.05, 0.0, -1.2, 2e-4, 0.5),
             lambda t: pkg.collide_boussinesq_vt_modified_2d_(t, _g(Temp), mt, 0.05, 0.0, -1.2,
                                                              2e-4, 0.5))):
        ref = f.copy()
        o_fn(ref)
        ft = _g(f)
        g_fn(ft)
        out = _h(ft)
        assert np.max(np.abs(out - ref) / np.abs(ref)) < 1e-13


@pytest.mark.parametrize("Nx,Ny,Nz", SIZES3)
def test_collide_thermal_3d(cuda, pkg, orc, Nx, Ny, Nz):
    shape = (Nz, Ny, Nx)
    g = _rand_pop((19,) + shape, W19, 11, base=0.6)
    u = [_field(shape, 12 + n) for n in range(3)]
    ref = g.copy()
    orc.collide_thermal_3d(ref, *u, 1.44)
    gt = _g(g)
    pkg.collide_thermal_3d_(gt, *[_g(a) for a in u], 1.44)
    assert np.array_equal(_h(gt), ref)
    Tt = torch.empty(shape, dtype=torch.float64, device=cuda)
    pkg.compute_temperature_3d_(Tt, _g(g))
    assert np.array_equal(_h(Tt), orc.temperature_3d(g))


@pytest.mark.parametrize("Nx,Ny,Nz", SIZES3)
def test_fixed_temp_3d(cuda, pkg, orc, Nx, Ny, Nz):
    g0 = np.random.default_rng(13).random((19, Nz, Ny, Nx))
    faces = ("west", "east", "south", "north", "bottom", "top")
    for n, face in enumerate(faces):
        for skip in (0, 5, 10, 15):
            te = [0.2 + 0.1 * n, 0.3, 0.45 - 0.02 * n, 0.8]
            ref = g0.copy()
            orc.fixed_temp_face_3d(ref, face, 0.9 - 0.1 * n, te, skip)
            gt = _g(g0)
            pkg.ops._fixed_temp_face_3d_(gt, face, 0.9 - 0.1 * n, te, skip)
            assert np.array_equal(_h(gt), ref), (face, skip)
    temps = dict(west=0.9, east=0.1, south=0.7, north=0.3, bottom=0.6, top=0.2)
    for mask in range(64):
        sel = {k: v for n, (k, v) in enumerate(temps.items()) if mask >> n & 1}
        ref = g0.copy()
        orc.fixed_temp_3d(ref, **sel)
        gt = _g(g0)
        pkg.apply_fixed_temp_3d_(gt, Nx, Ny, Nz, **sel)
        assert np.array_equal(_h(gt), ref), sel


@pytest.mark.parametrize("Nx,Ny,Nz", SIZES3)
@pytest.mark.parametrize("with_mask", [False, True])
def test_collide_boussinesq_3d(cuda, pkg, orc, Nx, Ny, Nz, with_mask):
    shape = (Nz, Ny, Nx)
    f = _rand_pop((19,) + shape, W19, 14)
    Temp = 0.5 + 0.3 * np.random.default_rng(15).random(shape)
    m = _mask(shape, 16) if with_mask else None
    ref = f.copy()
    orc.collide_boussinesq_3d(ref, Temp, m, 1.33, 4e-4, 0.5)
    ft = _g(f)
    pkg.collide_boussinesq_3d_(ft, _g(Temp), _g(m, torch.uint8) if m is not None else None,
                               1.33, 4e-4, 0.5)
    assert np.array_equal(_h(ft), ref)


def test_f32_kernels_within_rounding(cuda, pkg, orc):
    """Float32 storage runs the same arithmetic in single precision."""
    Nx, Ny = 40, 24
    f = _rand_pop((9, Ny, Nx), W9, 21)
    Temp = 0.5 + 0.3 * np.random.default_rng(22).random((Ny, Nx))
    ref = f.copy()
    orc.collide_boussinesq_2d(ref, Temp, None, 1.21, 3e-4, 0.5)
    ft = _g(f, torch.float32)
    pkg.collide_boussinesq_2d_(ft, _g(Temp, torch.float32), None, 1.21, 3e-4, 0.5)
    assert np.max(np.abs(_h(ft) - ref)) < 2e-7
    g = _rand_pop((19, 6, 7, 9), W19, 23, base=0.6)
    u = [_field((6, 7, 9), 24 + n) for n in range(3)]
    ref = g.copy()
    orc.collide_thermal_3d(ref, *u, 1.44)
    gt = _g(g, torch.float32)
    pkg.collide_thermal_3d_(gt, *[_g(a, torch.float32) for a in u], 1.44)
    assert np.max(np.abs(_h(gt) - ref)) < 2e-7


@pytest.mark.parametrize("orientation", ["vertical", "horizontal"])
@pytest.mark.parametrize("graph", [False, True])
def test_rayleigh_benard_driver_matches_oracle(cuda, pkg, orientation, graph):
    """run_rayleigh_benard_2d on the B200 kernels equals the oracle's
    restatement of the reference driver bit for bit (301 steps: the graph
    path replays 150 two-step cycles, then one eager step)."""
    Nx, Ny, steps = 32, 12, 301
    r = pkg.run_rayleigh_benard_2d(Nx=Nx, Ny=Ny, Ra=5000.0, max_steps=steps,
                                   orientation=orientation, graph=graph)
    o = td.run_rayleigh_benard_2d(Nx, Ny, 5000.0, max_steps=steps, orientation=orientation)
    for k in ("rho", "ux", "uy", "Temp"):
        assert np.array_equal(r[k], o[k]), k
    assert np.array_equal(_h(r["g"]), o["g"])


def test_rayleigh_benard_onset_gpu(cuda, pkg):
    """Reference pin "Rayleigh-Benard onset" (test_thermal.jl:339-356) through
    the B200 driver."""
    sub = pkg.run_rayleigh_benard_2d(Nx=64, Ny=16, Ra=1000.0, max_steps=10000)
    sup = pkg.run_rayleigh_benard_2d(Nx=64, Ny=16, Ra=5000.0, max_steps=20000)
    assert np.max(np.abs(sup["uy"])) > 5 * np.max(np.abs(sub["uy"]))
    assert np.all(np.isfinite(sup["Temp"]))


def test_natural_convection_3d_driver_matches_oracle(cuda, pkg):
    N, steps = 8, 121
    r = pkg.run_natural_convection_3d(N=N, Ra=2e4, max_steps=steps)
    o = td.run_natural_convection_3d(N, 2e4, max_steps=steps)
    for k in ("rho", "ux", "uy", "uz", "Temp"):
        assert np.array_equal(r[k], o[k]), k
    assert r["Nu"] == o["Nu"]


def test_box_pure_conduction_3d_gpu(cuda, pkg):
    """Reference pin (test_thermal.jl:330-336) through the B200 driver."""
    r = pkg.run_natural_convection_3d(N=12, Ra=0.0, max_steps=6000)
    d3 = max(abs(r["Temp"][5, 5, i] - (1 - (i + 0.5) / 12)) for i in range(12))
    assert abs(r["Nu"] - 1) < 3e-3 and d3 < 4e-4


@pytest.mark.parametrize("with_mask", [False, True])
def test_f32_forced_collisions_two_lanes_match_one_node_kernel(cuda, pkg, with_mask):
    """FP32 forced BGK in 3D (Boussinesq, constant and per-node Guo force):
    the two-node kernel (even Nx, 8-byte aligned fields, packed FP32x2
    arithmetic) and the one-node kernel (the same populations one element
    off the 8-byte boundary) agree to 4 ulp, solid nodes (pairs with one or
    two solid nodes) and the rest population bit for bit."""
    Nx, Ny, Nz = 34, 6, 5
    shape = (Nz, Ny, Nx)
    rng = np.random.default_rng(31)
    f = (W19[:, None, None, None] * (1 + 0.05 * rng.standard_normal((19,) + shape))).astype(np.float32)
    Temp = torch.from_numpy((0.5 + 0.3 * rng.random(shape)).astype(np.float32)).to(cuda)
    F = [torch.from_numpy((1e-3 * rng.standard_normal(shape)).astype(np.float32)).to(cuda) for _ in range(3)]
    m = _g(_mask(shape, 16), torch.uint8) if with_mask else None
    n = f.size

    def pair():
        a = torch.from_numpy(f.copy()).to(cuda)
        buf = torch.empty(n + 1, dtype=torch.float32, device=cuda)
        b = buf[1:].view(f.shape)
        b.copy_(a)
        assert a.data_ptr() % 8 == 0 and b.data_ptr() % 8 == 4
        return a, b

    for run in (lambda x: pkg.collide_boussinesq_3d_(x, Temp, m, 1.33, 4e-4, 0.5),
                lambda x: pkg.collide_guo_3d_(x, m, 1.27, 2e-4, 1e-4, -3e-4),
                lambda x: pkg.collide_guo_field_3d_(x, m, *F, 1.27)):
        a, b = pair()
        run(a)
        run(b)
        A, B = _h(a), _h(b)
        ulp = np.spacing(np.maximum(np.abs(A), np.abs(B)).astype(np.float32))
        assert np.all(np.abs(A - B) <= 4 * ulp)
        assert np.array_equal(A[0], B[0])
        if m is not None:
            s = _h(m).astype(bool)
            assert np.array_equal(A[:, s], B[:, s])


@pytest.mark.parametrize("with_mask", [False, True])
def test_f32_forced_collisions_2d_two_lanes_match_one_node_kernel(cuda, pkg, with_mask):
    """FP32 forced BGK in 2D (Boussinesq, constant and per-node Guo force):
    the two-node kernel (even Nx, 8-byte aligned fields, packed FP32x2
    arithmetic) and the one-node kernel (the same populations one element off
    the 8-byte boundary) agree to 4 ulp, solid nodes (pairs with one or two
    solid nodes) bit for bit."""
    Nx, Ny = 66, 24
    shape = (Ny, Nx)
    rng = np.random.default_rng(41)
    f = (W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9,) + shape))).astype(np.float32)
    Temp = torch.from_numpy((0.5 + 0.3 * rng.random(shape)).astype(np.float32)).to(cuda)
    F = [torch.from_numpy((1e-3 * rng.standard_normal(shape)).astype(np.float32)).to(cuda) for _ in range(2)]
    m = _g(_mask(shape, 17), torch.uint8) if with_mask else None

    def pair():
        a = torch.from_numpy(f.copy()).to(cuda)
        buf = torch.empty(f.size + 1, dtype=torch.float32, device=cuda)
        b = buf[1:].view(f.shape)
        b.copy_(a)
        assert a.data_ptr() % 8 == 0 and b.data_ptr() % 8 == 4
        return a, b

    for run in (lambda x: pkg.collide_boussinesq_2d_(x, Temp, m, 1.33, 4e-4, 0.5),
                lambda x: pkg.collide_guo_2d_(x, m, 1.27, 2e-4, -1e-4),
                lambda x: pkg.collide_guo_field_2d_(x, m, *F, 1.27)):
        a, b = pair()
        run(a)
        run(b)
        A, B = _h(a), _h(b)
        ulp = np.spacing(np.maximum(np.abs(A), np.abs(B)).astype(np.float32))
        assert np.all(np.abs(A - B) <= 4 * ulp)
        if m is not None:
            s = _h(m).astype(bool)
            assert np.array_equal(A[:, s], B[:, s])
