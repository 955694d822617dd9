"""Slab decomposition of one D3Q19 grid along z, host logic on CPU.

The decomposition splits the planes evenly and places ghost planes where a
neighbouring slab exists.  With gloo ranks (world size 2 and 3) and the
oracle's fused TRT step as the local step, the slabs exchange their
crossing populations after every step and reproduce the full-grid oracle
run bit for bit: periodic and walled z, walls or wraps in x and y, solid
nodes, moments."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT

W19 = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fields(Nx, Ny, Nz, with_mask):
    rng = np.random.default_rng(11)
    f = W19[:, None, None, None] * (1 + 0.05 * rng.standard_normal((19, Nz, Ny, Nx)))
    m = (rng.random((Nz, Ny, Nx)) < 0.1).astype(np.uint8) if with_mask else None
    return f, m


def _oracle_step(orc, sp, sm, per_xy):
    def step(f_out, f_in, moments, mask):
        m = tuple(t.numpy() for t in moments) if moments is not None else None
        orc.fused_trt_3d(f_out.numpy(), f_in.numpy(), m, mask, sp, sm,
                         (per_xy[0], per_xy[1], 0))
    return step


def _oracle_range(orc, sp, sm, per_xy):
    """A z-range step from the oracle: the whole local array is stepped into
    scratch (z non-periodic) and only the planes [k_begin, k_end) are kept,
    which is what the range step computes when planes k_begin - 1 and k_end
    exist."""
    whole = _oracle_step(orc, sp, sm, per_xy)

    def step(f_out, f_in, moments, mask, k_begin, k_end):
        tmp = torch.empty_like(f_in)
        tm = [torch.zeros_like(t) for t in moments] if moments is not None else None
        whole(tmp, f_in, tm, mask)
        f_out[:, k_begin:k_end] = tmp[:, k_begin:k_end]
        if moments is not None:
            for t, u in zip(moments, tm):
                t[k_begin:k_end] = u[k_begin:k_end]
    return step


def _run_slab(pkg, orc, slab, cfg, group=None, fs=None, overlap=False):
    Nx, Ny, Nz, per, steps, with_mask = cfg
    f, m = _fields(Nx, Ny, Nz, with_mask)
    sp, sm = orc.trt_rates(0.02, 0.25)
    ml = np.ascontiguousarray(slab.local_from_global(m)) if m is not None else None
    st = pkg.slab.SlabTRT3D(slab, Nx, Ny, mask=ml, group=group,
                            step_fn=_oracle_step(orc, sp, sm, per[:2]),
                            range_fn=_oracle_range(orc, sp, sm, per[:2]) if overlap else None)
    a = torch.from_numpy(np.ascontiguousarray(slab.local_from_global(f)))
    b = torch.zeros_like(a)
    mom = [torch.zeros((slab.nz_alloc, Ny, Nx), dtype=torch.float64) for _ in range(4)]
    for s in range(steps):
        (st.step_overlapped if overlap else st.step)(b, a, mom if s == steps - 1 else None)
        a, b = b, a
    return slab.real(a).numpy().copy(), [slab.real(t).numpy().copy() for t in mom]


def _worker(rank, world, port, cfg, out, overlap=False):
    import sys
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as graft
    pkg, orc = graft.load_package(), graft.load_oracle()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        slab = pkg.slab.Slab(cfg[2], world, rank, bool(cfg[3][2]))
        got, mom = _run_slab(pkg, orc, slab, cfg, overlap=overlap)
        out.put((rank, slab.z0, slab.z1, got, mom))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def _full(orc, cfg):
    Nx, Ny, Nz, per, steps, with_mask = cfg
    f, m = _fields(Nx, Ny, Nz, with_mask)
    sp, sm = orc.trt_rates(0.02, 0.25)
    g = np.empty_like(f)
    mom = [np.zeros((Nz, Ny, Nx)) for _ in range(4)]
    for s in range(steps):
        orc.fused_trt_3d(g, f, mom if s == steps - 1 else None, m, sp, sm, per)
        f, g = g, f
    return f, mom


@pytest.mark.parametrize("world,cfg,overlap", [
    (2, (6, 5, 8, (1, 1, 1), 3, False), False),
    (2, (7, 4, 9, (0, 1, 0), 3, True), False),
    (3, (5, 6, 10, (1, 0, 1), 4, True), False),
    (3, (6, 3, 7, (0, 0, 0), 3, False), False),
    # the exchange overlapped with the interior planes (step_overlapped);
    # on a walled z axis the two end slabs fall back to the plain step
    (2, (6, 5, 8, (1, 1, 1), 3, True), True),
    (3, (5, 6, 10, (1, 0, 1), 4, True), True),
    (3, (6, 4, 9, (0, 1, 0), 3, True), True),
])
def test_slabs_over_gloo_ranks_match_full_grid(orc, world, cfg, overlap):
    ref, ref_mom = _full(orc, cfg)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, cfg, q, overlap))
             for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    covered = []
    for rank, z0, z1, got, mom in res:
        assert np.array_equal(got, ref[:, z0:z1]), rank
        for a, b in zip(mom, ref_mom):
            assert np.array_equal(a, b[z0:z1]), rank
        covered += list(range(z0, z1))
    assert sorted(covered) == list(range(cfg[2]))


@pytest.mark.parametrize("R,per_z", [(1, True), (2, False), (4, True), (5, False)])
def test_slabs_in_one_process_match_full_grid(pkg, orc, R, per_z):
    """exchange_in_process over R slabs held by one process, oracle steps."""
    cfg = (5, 4, 11, (1, 0, int(per_z)), 3, True)
    Nx, Ny, Nz, per, steps, _ = cfg
    ref, _ = _full(orc, cfg)
    f, m = _fields(Nx, Ny, Nz, True)
    sp, sm = orc.trt_rates(0.02, 0.25)
    slabs = [pkg.slab.Slab(Nz, R, r, per_z) for r in range(R)]
    a = [torch.from_numpy(np.ascontiguousarray(s.local_from_global(f))) for s in slabs]
    b = [torch.empty_like(x) for x in a]
    masks = [np.ascontiguousarray(s.local_from_global(m)) for s in slabs]
    step = _oracle_step(orc, sp, sm, per[:2])
    for _ in range(steps):
        for x, y, mk in zip(a, b, masks):
            step(y, x, None, mk)
        pkg.slab.exchange_in_process(b, slabs)
        a, b = b, a
    for s, x in zip(slabs, a):
        assert np.array_equal(s.real(x).numpy(), ref[:, s.z0:s.z1])


@pytest.mark.parametrize("Nz,world", [(8, 3), (10, 4), (7, 7), (256, 8)])
def test_slab_split_and_ghosts(pkg, Nz, world):
    for per_z in (False, True):
        slabs = [pkg.slab.Slab(Nz, world, r, per_z) for r in range(world)]
        assert slabs[0].z0 == 0 and slabs[-1].z1 == Nz
        assert all(a.z1 == b.z0 for a, b in zip(slabs, slabs[1:]))
        assert max(s.nz for s in slabs) - min(s.nz for s in slabs) <= 1
        assert slabs[0].lo == per_z and slabs[-1].hi == per_z
        assert all(s.lo and s.hi for s in slabs[1:-1])
        for s in slabs:
            g = s.global_planes()
            assert g[s.k0:s.k0 + s.nz] == list(range(s.z0, s.z1))
            if s.lo:
                assert g[0] == (s.z0 - 1) % Nz
            if s.hi:
                assert g[-1] == s.z1 % Nz
    with pytest.raises(ValueError):
        pkg.slab.Slab(3, 4, 0, True)
    with pytest.raises(ValueError):
        pkg.slab.Slab(8, 2, 2, True)


def _worker_peer_gone(rank, world, port, out):
    import sys
    from datetime import timedelta
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as graft
    pkg = graft.load_package()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=5))
    slab = pkg.slab.Slab(8, world, rank, True)
    f = torch.zeros((19, slab.nz_alloc, 3, 4), dtype=torch.float64)
    if rank == 1:
        out.put((rank, "left"))
        return  # leaves between steps, before its exchange
    try:
        pkg.slab.exchange(f, slab)
        out.put((rank, "no error"))
    except Exception as e:  # the surviving rank learns of it from the process group
        out.put((rank, type(e).__name__))


def test_slab_exchange_reports_a_missing_peer(pkg):
    """A rank that leaves between steps makes its neighbour's next exchange
    end with an error within the process-group timeout, not hang."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker_peer_gone, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert res[1] == "left"
    assert res[0] != "no error", res


# ------------------------------------------------------------ D2Q9 y-slabs

W9 = np.array([4 / 9] + [1 / 9] * 4 + [1 / 36] * 4)


def _fields2(Nx, Ny, with_mask, seed=13):
    rng = np.random.default_rng(seed)
    f = W9[:, None, None] * (1 + 0.05 * rng.standard_normal((9, Ny, Nx)))
    m = (rng.random((Ny, Nx)) < 0.1).astype(np.uint8) if with_mask else None
    return f, m


def _oracle_step2(orc, kind):
    om, u_lid = 1.0 / (3 * 0.02 + 0.5), 0.1
    sp, sm = orc.trt_rates(0.02, 0.25)

    def step(f_out, f_in, moments, mask):
        a, b = f_out.numpy(), f_in.numpy()
        rho, ux, uy = (t.numpy() for t in moments)
        if kind == "bgk":
            orc.fused_bgk_2d(a, b, rho, ux, uy, mask, om)
        elif kind == "trt":
            orc.fused_trt_2d(a, b, rho, ux, uy, mask, sp, sm)
        else:
            orc.cavity_movingwall_bgk_2d(a, b, rho, ux, uy, mask, om, u_lid)
    return step


def _full2(orc, Nx, Ny, kind, steps, with_mask):
    f, m = _fields2(Nx, Ny, with_mask)
    g = np.empty_like(f)
    mom = [torch.zeros((Ny, Nx), dtype=torch.float64) for _ in range(3)]
    step = _oracle_step2(orc, kind)
    a, b = torch.from_numpy(f), torch.from_numpy(g)
    for _ in range(steps):
        step(b, a, mom, m)
        a, b = b, a
    return a.numpy(), [t.numpy() for t in mom]


def _worker2(rank, world, port, cfg, out):
    import sys
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as graft
    pkg, orc = graft.load_package(), graft.load_oracle()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        Nx, Ny, kind, steps, with_mask = cfg
        slab = pkg.slab.Slab(Ny, world, rank, False)
        f, m = _fields2(Nx, Ny, with_mask)
        ml = np.ascontiguousarray(slab.local_from_global(m, axis=-2)) if m is not None else None
        st = pkg.slab.SlabD2Q9(slab, Nx, kind, mask=ml, step_fn=_oracle_step2(orc, kind))
        a = torch.from_numpy(np.ascontiguousarray(slab.local_from_global(f, axis=-2)))
        b = torch.zeros_like(a)
        mom = [torch.zeros((slab.nz_alloc, Nx), dtype=torch.float64) for _ in range(3)]
        for _ in range(steps):
            st.step(b, a, mom)
            a, b = b, a
        out.put((rank, slab.z0, slab.z1, slab.real(a, axis=-2).numpy().copy(),
                 [slab.real(t, axis=-2).numpy().copy() for t in mom]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,cfg", [
    (2, (7, 10, "bgk", 4, True)),
    (3, (6, 11, "trt", 3, True)),
    (3, (8, 9, "movingwall", 4, False)),
])
def test_d2q9_y_slabs_over_gloo_ranks_match_full_grid(orc, world, cfg):
    """D2Q9 y-slabs on gloo ranks, the oracle's fused step as the local step,
    against the full-grid oracle bit for bit (populations and moments)."""
    Nx, Ny, kind, steps, with_mask = cfg
    ref, ref_mom = _full2(orc, Nx, Ny, kind, steps, with_mask)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker2, args=(r, world, port, cfg, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=180) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    covered = []
    for rank, y0, y1, got, mom in res:
        assert np.array_equal(got, ref[:, y0:y1]), rank
        for a, b in zip(mom, ref_mom):
            assert np.array_equal(a, b[y0:y1]), rank
        covered += list(range(y0, y1))
    assert sorted(covered) == list(range(Ny))


@pytest.mark.parametrize("R", [1, 2, 4])
@pytest.mark.parametrize("kind", ["bgk", "trt", "movingwall"])
def test_d2q9_y_slabs_in_one_process_match_full_grid(pkg, orc, R, kind):
    Nx, Ny, steps = 6, 12, 3
    ref, _ = _full2(orc, Nx, Ny, kind, steps, True)
    f, m = _fields2(Nx, Ny, True)
    slabs = [pkg.slab.Slab(Ny, R, r, False) for r in range(R)]
    a = [torch.from_numpy(np.ascontiguousarray(s.local_from_global(f, axis=-2))) for s in slabs]
    b = [torch.zeros_like(x) for x in a]
    masks = [np.ascontiguousarray(s.local_from_global(m, axis=-2)) for s in slabs]
    step = _oracle_step2(orc, kind)
    mom = [[torch.zeros((s.nz_alloc, Nx), dtype=torch.float64) for _ in range(3)] for s in slabs]
    for _ in range(steps):
        for x, y, mk, mm in zip(a, b, masks, mom):
            step(y, x, mm, mk)
        pkg.slab.exchange_in_process(b, slabs, (pkg.slab.CYP, pkg.slab.CYM))
        a, b = b, a
    for s, x in zip(slabs, a):
        assert np.array_equal(s.real(x, axis=-2).numpy(), ref[:, s.z0:s.z1])


def test_d2q9_slab_rejects_periodic_split(pkg):
    with pytest.raises(ValueError):
        pkg.slab.SlabD2Q9(pkg.slab.Slab(8, 2, 0, True), 4, "bgk", omega=1.0)
