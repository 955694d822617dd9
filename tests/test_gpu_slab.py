"""Slab decomposition on the GPU: the CUDA step on each slab's local array
(ghost planes included, z non-periodic) plus the ghost exchange reproduces
the full-grid CUDA step bit for bit for the round-to-nearest storages --
including the staged row-tile kernel (Nx = 256) and the x / x+32 pair kernel
(Nx = 96) of the 16-bit storages -- with periodic or walled z and solid
nodes.  The slabs live in one process; between GPUs the same planes travel
by NCCL point-to-point (the exchange order is covered by the gloo test)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def _setup(pkg, Nx, Ny, Nz, dtype, deviation, seed=5):
    rng = np.random.default_rng(seed)
    f = W19[:, None, None, None] * (1 + 0.05 * rng.standard_normal((19, Nz, Ny, Nx)))
    m = (rng.random((Nz, Ny, Nx)) < 0.08).astype(np.uint8)
    full = torch.empty((19, Nz, Ny, Nx), dtype=dtype, device="cuda")
    pkg.convert_populations(full, torch.from_numpy(f).cuda(), dst_deviation=deviation)
    return full, torch.from_numpy(m).cuda().bool()


@pytest.mark.parametrize("dtype,deviation", [(torch.float64, False), (torch.float32, False),
                                             (torch.float16, True), (torch.bfloat16, True),
                                             (torch.float32, True)])
@pytest.mark.parametrize("shape,per,R", [((256, 4, 9), (1, 1, 1), 3), ((256, 3, 8), (0, 1, 0), 2),
                                         ((96, 5, 7), (1, 0, 1), 2), ((96, 4, 10), (0, 0, 0), 4)])
def test_slabs_match_full_grid_on_gpu(cuda, pkg, dtype, deviation, shape, per, R):
    Nx, Ny, Nz = shape
    steps = 3
    full, mask = _setup(pkg, Nx, Ny, Nz, dtype, deviation)
    slabs = [pkg.slab.Slab(Nz, R, r, bool(per[2])) for r in range(R)]
    a = [s.local_from_global(full).contiguous() for s in slabs]
    b = [torch.empty_like(x) for x in a]
    masks = [s.local_from_global(mask).contiguous() for s in slabs]
    fd = torch.float64 if dtype == torch.float64 else torch.float32
    steppers = [pkg.slab.SlabTRT3D(s, Nx, Ny, nu=0.02, Lambda=0.25, periodic_xy=per[:2],
                                   deviation=deviation, mask=mk) for s, mk in zip(slabs, masks)]
    mom = [[torch.zeros((s.nz_alloc, Ny, Nx), dtype=fd, device="cuda") for _ in range(4)]
           for s in slabs]
    g = torch.empty_like(full)
    fm = [torch.zeros((Nz, Ny, Nx), dtype=fd, device="cuda") for _ in range(4)]
    for s in range(steps):
        last = s == steps - 1
        pkg.fused_trt_step_3d_(g, full, *(fm if last else (None,) * 4), mask, Nx, Ny, Nz, 0.02, 0.25,
                               periodic=per, deviation=deviation)
        full, g = g, full
        # one process holds every slab: step them all, then exchange in process
        for st, x, y, mm in zip(steppers, a, b, mom):
            st.step_fn(y, x, mm if last else None, st.mask)
        pkg.slab.exchange_in_process(b, slabs)
        a, b = b, a
    torch.cuda.synchronize()
    for s, x, mm in zip(slabs, a, mom):
        assert torch.equal(s.real(x), full[:, s.z0:s.z1])
        for t, u in zip(mm, fm):
            assert torch.equal(s.real(t), u[s.z0:s.z1])


def test_single_slab_periodic_ring_on_gpu(cuda, pkg):
    """One rank on a periodic z axis: the ghosts are the slab's own end planes
    (SlabTRT3D.step with the CUDA step and the one-rank exchange)."""
    Nx, Ny, Nz = 256, 4, 6
    full, _ = _setup(pkg, Nx, Ny, Nz, torch.float16, True, seed=9)
    s = pkg.slab.Slab(Nz, 1, 0, True)
    st = pkg.slab.SlabTRT3D(s, Nx, Ny, nu=0.01, Lambda=0.25, periodic_xy=(1, 1), deviation=True)
    a = s.local_from_global(full).contiguous()
    b = torch.empty_like(a)
    g = torch.empty_like(full)
    for _ in range(4):
        pkg.fused_trt_step_3d_(g, full, None, None, None, None, None, Nx, Ny, Nz, 0.01, 0.25,
                               periodic=(1, 1, 1), deviation=True)
        full, g = g, full
        st.step(b, a)
        a, b = b, a
    assert torch.equal(s.real(a), full)


def _range_cases():
    out = []
    for dtype, dev in [(torch.float64, False), (torch.float32, False), (torch.float32, True)]:
        out.append((dtype, dev, 0))
    for dtype in (torch.float16, torch.bfloat16):
        for v in range(6):
            out.append((dtype, True, v))
    return out


@pytest.mark.parametrize("dtype,deviation,variant", _range_cases())
@pytest.mark.parametrize("Nx,per_xy", [(256, (1, 1)), (96, (0, 1)), (64, (1, 0))])
def test_zrange_steps_match_whole_local_step(cuda, pkg, dtype, deviation, variant, Nx, per_xy):
    """kb_fused_trt_step_3d_zrange over [1, 2), [Nz-2, Nz-1) and the planes
    between equals one step of the whole local array (z non-periodic) on
    every plane but the two halo planes, bit for bit, for every kernel
    variant of the 16-bit storages (the staged row tiles need Nx % 8 == 0
    and 16-byte rows: every Nx here runs them)."""
    Ny, Nz = 5, 10
    full, mask = _setup(pkg, Nx, Ny, Nz, dtype, deviation, seed=21)
    fd = torch.float64 if dtype == torch.float64 else torch.float32
    ref = torch.zeros_like(full)
    got = torch.zeros_like(full)
    rm = [torch.zeros((Nz, Ny, Nx), dtype=fd, device="cuda") for _ in range(4)]
    gm = [torch.zeros((Nz, Ny, Nx), dtype=fd, device="cuda") for _ in range(4)]
    pkg.set_trt3d_variant(variant)
    try:
        for m in (mask, None):
            pkg.fused_trt_step_3d_(ref, full, *rm, m, Nx, Ny, Nz, 0.02, 0.25,
                                   periodic=(*per_xy, 0), deviation=deviation)
            for kb, ke in ((1, 2), (Nz - 2, Nz - 1), (2, Nz - 2)):
                pkg.fused_trt_step_3d_zrange_(got, full, *gm, m, Nx, Ny, Nz, kb, ke, 0.02, 0.25,
                                              periodic_xy=per_xy, deviation=deviation)
            torch.cuda.synchronize()
            assert torch.equal(got[:, 1:Nz - 1], ref[:, 1:Nz - 1])
            for a, b in zip(gm, rm):
                assert torch.equal(a[1:Nz - 1], b[1:Nz - 1])
            # only the range is written
            assert not got[:, 0].any() and not got[:, Nz - 1].any()
    finally:
        pkg.set_trt3d_variant(0)


def test_zrange_rejects_halo_planes(cuda, pkg):
    Nx, Ny, Nz = 64, 4, 6
    f = torch.zeros((19, Nz, Ny, Nx), dtype=torch.float32, device="cuda")
    g = torch.zeros_like(f)
    for kb, ke in ((0, 3), (1, Nz), (3, 3), (4, 2)):
        with pytest.raises(ValueError):
            pkg.fused_trt_step_3d_zrange_(g, f, None, None, None, None, None, Nx, Ny, Nz, kb, ke,
                                          0.02, 0.25)


@pytest.mark.parametrize("dtype,deviation", [(torch.float64, False), (torch.float16, True),
                                             (torch.float32, True)])
@pytest.mark.parametrize("R", [1, 2, 3])
def test_overlapped_slab_steps_match_full_grid_on_gpu(cuda, pkg, dtype, deviation, R):
    """Each slab of a periodic z ring steps its two face planes, then its
    interior, with range steps (the order of step_overlapped); the exchange
    in one process then gives the full-grid CUDA step bit for bit.  With one
    slab, step_overlapped itself runs (its exchange is the one-rank ghost
    fill)."""
    Nx, Ny, Nz = 256, 4, 12
    full, mask = _setup(pkg, Nx, Ny, Nz, dtype, deviation, seed=17)
    slabs = [pkg.slab.Slab(Nz, R, r, True) for r in range(R)]
    a = [s.local_from_global(full).contiguous() for s in slabs]
    b = [torch.zeros_like(x) for x in a]
    masks = [s.local_from_global(mask).contiguous() for s in slabs]
    steppers = [pkg.slab.SlabTRT3D(s, Nx, Ny, nu=0.02, Lambda=0.25, periodic_xy=(1, 0),
                                   deviation=deviation, mask=mk) for s, mk in zip(slabs, masks)]
    assert all(st.overlapped() for st in steppers)
    g = torch.empty_like(full)
    for _ in range(3):
        pkg.fused_trt_step_3d_(g, full, None, None, None, None, mask, Nx, Ny, Nz, 0.02, 0.25,
                               periodic=(1, 0, 1), deviation=deviation)
        full, g = g, full
        if R == 1:
            steppers[0].step_overlapped(b[0], a[0])
        else:
            for st, x, y in zip(steppers, a, b):
                s = st.slab
                bot, top = s.k0, s.k0 + s.nz - 1
                st.range_fn(y, x, None, st.mask, bot, bot + 1)
                st.range_fn(y, x, None, st.mask, top, top + 1)
                st.range_fn(y, x, None, st.mask, bot + 1, top)
            pkg.slab.exchange_in_process(b, slabs)
        a, b = b, a
    torch.cuda.synchronize()
    for s, x in zip(slabs, a):
        assert torch.equal(s.real(x), full[:, s.z0:s.z1])


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("kind", ["bgk", "trt", "cavity", "movingwall"])
@pytest.mark.parametrize("R", [2, 3])
def test_d2q9_y_slabs_match_full_grid_on_gpu(cuda, pkg, dtype, kind, R):
    """D2Q9 y-slabs (SlabD2Q9) with the CUDA fused 2D steps, in one process,
    against the full-grid CUDA step bit for bit: populations and moments,
    walled grid with solid nodes, the lid on the top slab."""
    Nx, Ny, steps = 200, 37, 4
    rng = np.random.default_rng(3)
    w9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)
    f = torch.from_numpy(w9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, Ny, Nx))))
    m = torch.from_numpy(rng.random((Ny, Nx)) < 0.08)
    full, mask = f.to("cuda", dtype), m.cuda()
    slabs = [pkg.slab.Slab(Ny, R, r, False) for r in range(R)]
    kw = dict(omega=1.0 / (3 * 0.02 + 0.5), nu=0.02, Lambda=0.25, u_lid=0.1)
    steppers = [pkg.slab.SlabD2Q9(s, Nx, kind, mask=s.local_from_global(mask, axis=-2).contiguous(),
                                  **kw) for s in slabs]
    a = [s.local_from_global(full, axis=-2).contiguous() for s in slabs]
    b = [torch.zeros_like(x) for x in a]
    mom = [[torch.zeros((s.nz_alloc, Nx), dtype=dtype, device="cuda") for _ in range(3)]
           for s in slabs]
    ref = pkg.slab.SlabD2Q9(pkg.slab.Slab(Ny, 1, 0, False), Nx, kind, mask=mask, **kw)
    g = torch.zeros_like(full)
    fm = [torch.zeros((Ny, Nx), dtype=dtype, device="cuda") for _ in range(3)]
    for _ in range(steps):
        ref.step(g, full, fm)
        full, g = g, full
        for st, x, y, mm in zip(steppers, a, b, mom):
            st.step_fn(y, x, mm, st.mask)
        pkg.slab.exchange_in_process(b, slabs, (pkg.slab.CYP, pkg.slab.CYM))
        a, b = b, a
    torch.cuda.synchronize()
    for s, x, mm in zip(slabs, a, mom):
        assert torch.equal(s.real(x, axis=-2), full[:, s.z0:s.z1])
        for t, u in zip(mm, fm):
            assert torch.equal(s.real(t, axis=-2), u[s.z0:s.z1])
