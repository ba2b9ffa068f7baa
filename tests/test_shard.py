"""Work-list sharding of independent problems (cedar_b200.shard): the split
every rank computes, and the statistics gather over a two-rank gloo group on
the CPU (the path that bench.py --gpus N takes for the batched solves)."""
import os
import socket

import numpy as np
import pytest

from cedar_b200 import problems as P
from cedar_b200 import shard


def test_partition_covers_once_and_balances():
    sizes = P.batch_sizes(512)
    for world in (1, 2, 3, 4, 8):
        parts = shard.partition(sizes, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(sizes)))
        ld = shard.loads(sizes, parts)
        # longest processing time first: within one largest problem of even
        assert max(ld) - min(ld) <= int(sizes.max()) ** 2
        assert shard.partition(sizes, world) == parts  # deterministic


def test_partition_rejects_bad_world():
    with pytest.raises(ValueError):
        shard.partition([63, 127], 0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        sizes = P.batch_sizes(64)
        parts = shard.partition(sizes, world)
        ids = np.array(parts[rank], dtype=np.int64)
        vals = np.stack([ids * 2.0, sizes[ids].astype(float)], axis=1)
        table = shard.gather_stats(ids, vals, dist)
        ok = table.shape == (64, 2) and np.array_equal(table[:, 0], np.arange(64) * 2.0) \
            and np.array_equal(table[:, 1], sizes.astype(float))
        q.put((rank, bool(ok)))
    finally:
        dist.destroy_process_group()


def test_gather_stats_two_ranks_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    res = sorted(q.get(timeout=5) for _ in procs)
    assert res == [(0, True), (1, True)]
    assert all(p.exitcode == 0 for p in procs)
