"""Multi-rank host logic on CPU: world_size 2 over gloo."""
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


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from sseqs_b200 import shard
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # shard r holds hits with scores r + 0.5*k; ties across shards on 1.5
        rows = [(float(rank) + 0.5 * k, 0, 10 * rank + k, 100 + k, 50, f"S{rank}{k}")
                for k in range(4)]
        rows.sort(key=lambda x: (-x[0], x[1], x[2]))
        merged = shard.gather_hits(rows, num_msas=5)
        out[rank] = merged
    finally:
        dist.destroy_process_group()


def test_gather_hits_two_ranks():
    world = 2
    port = _free_port()
    manager = mp.get_context("spawn").Manager()   # no fork after torch has started threads
    out = manager.dict()
    mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
    assert out[0] == out[1]
    merged = out[0]
    assert [round(r[0], 1) for r in merged] == [2.5, 2.0, 1.5, 1.5, 1.0]
    # tie at 1.5: shard 0 before shard 1
    assert merged[2][1] == 0 and merged[3][1] == 1
    assert merged[0][6] == "S13"


def test_merge_single_process():
    from sseqs_b200 import shard
    rows = [(3.0, 0, 1, 9, 9, "a"), (1.0, 1, 2, 9, 9, "b")]
    assert shard.gather_hits(rows, 1) == [(3.0, 0, 0, 1, 9, 9, "a")]
