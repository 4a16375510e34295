"""The N > 1 host logic of bench.py on CPU: two gloo ranks on 127.0.0.1. The
batched scenes are split between ranks with no overlap and no gap, by
estimated cost (longest processing time first) so that the ranks' totals
stay within a stated bound of each other, and the timing reduction gives
every rank the slowest rank's time."""
import math
import os
import socket

import numpy as np
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
    # uneven scenes (fluid counts log-uniform in [2,000, 60,000], as the batched dams)
    rng = np.random.default_rng(6)
    sizes = [int(x) for x in np.exp(rng.uniform(math.log(2000), math.log(60000), 256))]
    costed = bench.shard(list(range(256)), rank, world, cost=lambda i: bench.scene_cost(sizes[i], sizes[i] // 4))
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    gathered_costed = [None] * world
    dist.all_gather_object(gathered_costed, costed)
    t = bench.max_reducer(world, "cpu")(1.5 * (rank + 1))
    loads = [sum(bench.scene_cost(sizes[i], sizes[i] // 4) for i in part) for part in gathered_costed]
    biggest = max(bench.scene_cost(s, s // 4) for s in sizes)
    out.put((rank, gathered, gathered_costed, loads, biggest, t))
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
    for rank, gathered, costed, loads, biggest, t in res:
        assert t == 3.0
        for split in (gathered, costed):
            flat = [i for part in split for i in part]
            assert sorted(flat) == list(range(256))
            assert len(set(split[0]) & set(split[1])) == 0
        # longest processing time first: no rank above the mean plus the largest scene
        mean = sum(loads) / world
        assert max(loads) <= mean + biggest
        # and in practice within 1 % of the mean for 256 scenes on 2 ranks
        assert max(loads) <= 1.01 * mean
