"""Multi-rank host logic on CPU (gloo, world size 2): sweep cases shard across
ranks with no data exchange, every case runs exactly once, loads balance,
and the max-over-ranks timing reduction matches the single-process one."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, N, out):
    import sys
    sys.path.insert(0, str(ROOT))
    import __graft_entry__ as graft
    pkg = graft.load_package()
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = pkg.sharding.shard_cases(N, world, rank)
    sizes = [None] * world
    dist.all_gather_object(sizes, mine.tolist())
    # each rank "times" its shard as its node total; the job time is the max
    t = torch.tensor([float(np.sum(np.asarray(N)[mine] ** 2))], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        out.put((sizes, float(t.item())))
    dist.barrier()
    dist.destroy_process_group()


def test_shard_cases_two_ranks_gloo(pkg):
    N, _, _, _ = pkg.sweep_cases(256, seed=0)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, N, q)) for r in range(2)]
    for p in procs:
        p.start()
    sizes, tmax = q.get(timeout=120)
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    allc = sorted(sizes[0] + sizes[1])
    assert allc == list(range(256))
    loads = pkg.sharding.shard_loads(N, 2)
    assert tmax == max(loads)
    assert max(loads) - min(loads) <= int(np.max(N.astype(np.int64)) ** 2)


@pytest.mark.parametrize("world", [1, 3, 8])
def test_shard_cases_partition(pkg, world):
    N = np.array([64, 512, 96, 480, 128, 64, 256, 320, 512, 96])
    seen = np.concatenate([pkg.sharding.shard_cases(N, world, r) for r in range(world)])
    assert sorted(seen.tolist()) == list(range(len(N)))
    loads = pkg.sharding.shard_loads(N, world)
    assert max(loads) - min(loads) <= 512 ** 2
    with pytest.raises(ValueError):
        pkg.sharding.shard_cases(N, world, world)
