"""Replica sharding across ranks (world_size 2, gloo on CPU): every chunk is owned by exactly one
rank, and the max-over-ranks timing reduction the benchmark uses agrees on every rank."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, n_items, out):
    import torch
    import torch.distributed as dist
    from petakit5d_b200.chunking import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=__import__("datetime").timedelta(seconds=60))
    mine = shard(n_items, rank, world)
    mask = torch.zeros(n_items, dtype=torch.int64)
    mask[mine] = 1
    dist.all_reduce(mask)                          # each chunk counted once over all ranks
    t = torch.tensor([1.5 + rank])                 # per-rank step time
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    out[rank] = (mask.tolist(), float(t.item()), len(mine))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("n_items", [96, 7, 1])
def test_two_replicas_cover_every_chunk_once(n_items):
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(world, _free_port(), n_items, out), nprocs=world, join=True)
    for r in range(world):
        mask, tmax, cnt = out[r]
        assert mask == [1] * n_items
        assert tmax == 2.5
    assert out[0][2] + out[1][2] == n_items


def test_shard_rejects_bad_rank():
    from petakit5d_b200.chunking import shard
    with pytest.raises(ValueError):
        shard(10, 2, 2)
