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
