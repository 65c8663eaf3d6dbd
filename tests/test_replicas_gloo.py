"""The multi-rank host logic (dclaw_b200/replicas.py) with two gloo ranks on
the CPU: timings combine as the maximum over ranks, ensemble shards cover
every member once with balanced cell counts, replicas get distinct seeds."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from dclaw_b200.replicas import max_over_ranks, replica_seed, shard_members


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = 10.0 + 5.0 * rank
        out[rank] = max_over_ranks(ms)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    assert out[0] == 15.0 and out[1] == 15.0


def test_single_process_max_is_identity():
    assert max_over_ranks(3.5) == 3.5


def test_shards_cover_members_once_and_balance_cells():
    rng = np.random.default_rng(0)
    cells = rng.integers(32 * 1024, 128 * 4096, size=256)
    for world in (1, 2, 4, 8):
        shards = [shard_members(cells, r, world) for r in range(world)]
        flat = sorted(k for s in shards for k in s)
        assert flat == list(range(len(cells)))
        loads = np.array([cells[s].sum() for s in shards])
        assert loads.max() <= loads.mean() + cells.max()


def test_replica_seeds_differ():
    assert len({replica_seed(0, r) for r in range(8)}) == 8
