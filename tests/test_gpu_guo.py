"""Guo-forced collisions, force-corrected moments, the x/z-periodic 3D stream
and the Poiseuille / Couette drivers on the B200 against the oracle (FP64
bit for bit)."""
import numpy as np
import pytest
import torch

from test_oracle_guo import (W9, W19, oracle_couette_2d, oracle_poiseuille_2d,
                             oracle_poiseuille_3d, poiseuille_err)

pytestmark = pytest.mark.gpu


def _g(a, dtype=torch.float64):
    return torch.from_numpy(np.ascontiguousarray(a)).to("cuda", dtype)


def _h(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def _mask(shape, seed):
    return (np.random.default_rng(seed).random(shape) < 0.2).astype(np.uint8)


@pytest.mark.parametrize("Nx,Ny", [(1, 1), (2, 3), (17, 13), (33, 7), (130, 9)])
@pytest.mark.parametrize("with_mask", [False, True])
def test_guo_2d(cuda, pkg, orc, Nx, Ny, with_mask):
    rng = np.random.default_rng(Nx + Ny)
    f = W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, Ny, Nx)))
    m = _mask((Ny, Nx), 2) if with_mask else None
    mt = _g(m, torch.uint8) if m is not None else None
    ref = f.copy()
    orc.collide_guo_2d(ref, m, 1.31, 3e-4, -2e-4)
    ft = _g(f)
    pkg.collide_guo_2d_(ft, mt, 1.31, 3e-4, -2e-4)
    assert np.array_equal(_h(ft), ref)
    Fx, Fy = 1e-3 * rng.standard_normal((2, Ny, Nx))
    ref = f.copy()
    orc.collide_guo_field_2d(ref, m, Fx, Fy, 1.31)
    ft = _g(f)
    pkg.collide_guo_field_2d_(ft, mt, _g(Fx), _g(Fy), 1.31)
    assert np.array_equal(_h(ft), ref)
    r = [torch.empty((Ny, Nx), dtype=torch.float64, device=cuda) for _ in range(3)]
    pkg.compute_macroscopic_forced_2d_(*r, _g(f), 3e-4, -2e-4)
    for t, a in zip(r, orc.macroscopic_forced_2d(f, 3e-4, -2e-4)):
        assert np.array_equal(_h(t), a)


@pytest.mark.parametrize("Nx,Ny,Nz", [(1, 1, 1), (3, 2, 5), (17, 5, 6), (33, 9, 4)])
@pytest.mark.parametrize("with_mask", [False, True])
def test_guo_3d(cuda, pkg, orc, Nx, Ny, Nz, with_mask):
    shape = (Nz, Ny, Nx)
    rng = np.random.default_rng(Nx + 7 * Nz)
    f = W19[:, None, None, None] * (1 + 0.05 * rng.standard_normal((19,) + shape))
    m = _mask(shape, 3) if with_mask else None
    mt = _g(m, torch.uint8) if m is not None else None
    ref = f.copy()
    orc.collide_guo_3d(ref, m, 1.27, 2e-4, 1e-4, -3e-4)
    ft = _g(f)
    pkg.collide_guo_3d_(ft, mt, 1.27, 2e-4, 1e-4, -3e-4)
    assert np.array_equal(_h(ft), ref)
    F = 1e-3 * rng.standard_normal((3,) + shape)
    ref = f.copy()
    orc.collide_guo_field_3d(ref, m, *F, 1.27)
    ft = _g(f)
    pkg.collide_guo_field_3d_(ft, mt, *[_g(a) for a in F], 1.27)
    assert np.array_equal(_h(ft), ref)
    r = [torch.empty(shape, dtype=torch.float64, device=cuda) for _ in range(4)]
    pkg.compute_macroscopic_forced_3d_(*r, _g(f), *[_g(a) for a in F])
    for t, a in zip(r, orc.macroscopic_forced_3d(f, *F)):
        assert np.array_equal(_h(t), a)
    pkg.compute_macroscopic_forced_3d_(*r, _g(f), 2e-4, 1e-4, -3e-4)
    for t, a in zip(r, orc.macroscopic_forced_3d(f, 2e-4, 1e-4, -3e-4)):
        assert np.array_equal(_h(t), a)
    out = np.empty_like(f)
    orc.stream_periodic_xz_wall_y_3d(out, f)
    fo = torch.empty_like(_g(f))
    pkg.stream_periodic_xz_wall_y_3d_(fo, _g(f), Nx, Ny, Nz)
    assert np.array_equal(_h(fo), out)


@pytest.mark.parametrize("graph", [False, True])
def test_poiseuille_2d_driver(cuda, pkg, orc, graph):
    """run_poiseuille_2d == the oracle's restatement (501 steps), and the
    reference pin after 10 000 steps."""
    r = pkg.run_poiseuille_2d(Nx=4, Ny=32, nu=0.1, Fx=1e-5, max_steps=501, graph=graph)
    rho, ux, uy, f = oracle_poiseuille_2d(orc, steps=501)
    assert np.array_equal(r["ux"], ux) and np.array_equal(r["rho"], rho)
    assert np.array_equal(_h(r["f"]), f)
    r = pkg.run_poiseuille_2d(max_steps=10000)
    assert poiseuille_err(r["ux"][:, 1], 32, 0.1, 1e-5) < 0.02


def test_couette_2d_driver(cuda, pkg, orc):
    r = pkg.run_couette_2d(max_steps=30000)
    _, ux, uy, _ = oracle_couette_2d(orc, steps=30000)
    assert np.array_equal(r["ux"], ux) and np.array_equal(r["uy"], uy)
    u_ana = np.array([0.05 * (1 - (j - 1) / 31) for j in range(1, 33)])
    assert np.max(np.abs(r["ux"][1:-1, 1] - u_ana[1:-1])) / 0.05 < 1e-10


def test_poiseuille_3d_loop(cuda, pkg, orc):
    """The loop of test_poiseuille_3d.jl on the B200 kernels == the oracle."""
    Nx, Ny, Nz, steps = 4, 32, 4, 2000
    f = np.stack([np.full((Nz, Ny, Nx), W19[q]) for q in range(19)])
    fi, fo = _g(f), _g(f)
    m = [torch.zeros((Nz, Ny, Nx), dtype=torch.float64, device=cuda) for _ in range(4)]
    w = 1.0 / (3.0 * 0.1 + 0.5)
    for _ in range(steps):
        pkg.stream_periodic_xz_wall_y_3d_(fo, fi, Nx, Ny, Nz)
        pkg.collide_guo_3d_(fo, None, w, 1e-5, 0.0, 0.0)
        pkg.compute_macroscopic_forced_3d_(*m, fo, 1e-5, 0.0, 0.0)
        fi, fo = fo, fi
    om, of = oracle_poiseuille_3d(orc, steps=steps)
    assert np.array_equal(_h(fi), of)
    for t, a in zip(m, om):
        assert np.array_equal(_h(t), a)
