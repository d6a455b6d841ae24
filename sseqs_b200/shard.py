"""Database sharding across GPUs: one process per GPU, each holding its own
shard of the database resident in HBM (the reference's multi-GPU mode runs
independent per-GPU threads over shared host RAM, sseqs/msa.py:87-104).

A search runs on every shard independently; the only exchange is the merge
of each shard's ranked hits (a few thousand small records per query), done
with one ``all_gather_object`` over the process group.  Merged order: score
descending, then shard rank, batch and segment position ascending -- the
same canonical order ``msa.rank_hits`` uses inside one shard.
"""
from __future__ import annotations

import torch.distributed as dist


def merge_ranked(per_rank: list, num_msas: int) -> list:
    """Merge lists of ranked rows (score, batch, segment, ...) from shards."""
    rows = []
    for r, lst in enumerate(per_rank):
        for row in lst:
            rows.append((row[0], r) + tuple(row[1:]))
    rows.sort(key=lambda x: (-x[0], x[1], x[2], x[3]))
    return rows[:num_msas]


def gather_hits(rows: list, num_msas: int, group=None) -> list:
    """All ranks receive the merged top ``num_msas`` rows; each row gains the
    shard rank as its second field."""
    if not dist.is_available() or not dist.is_initialized():
        return merge_ranked([rows], num_msas)
    world = dist.get_world_size(group)
    per = [None] * world
    dist.all_gather_object(per, rows, group=group)
    return merge_ranked(per, num_msas)
