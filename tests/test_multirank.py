"""The N > 1 host logic of bench.py on CPU: two gloo ranks on 127.0.0.1. The
batched scenes are split between ranks with no overlap and no gap, and the
timing reduction gives every rank the slowest rank's time."""
import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import sys
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    mine = bench.shard(list(range(256)), rank, world)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    t = bench.max_reducer(world, "cpu")(1.5 * (rank + 1))
    out.put((rank, gathered, t))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_shard_scenes_and_reduce_the_time():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, gathered, t in res:
        assert t == 3.0
        flat = [i for part in gathered for i in part]
        assert sorted(flat) == list(range(256))
        assert len(set(gathered[0]) & set(gathered[1])) == 0
