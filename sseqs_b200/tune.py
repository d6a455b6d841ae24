"""Autotuner of the score kernel's lane layout.

For every stripe width tpt = ceil(query_len/32) <= 16 the score kernel exists
in two layouts (see ``sseqs_sw_set_variant``): fewer, longer rows per lane
group, or more targets per warp with twice the columns per lane.  Both give
identical scores; which is faster depends on the width and on register
pressure, so it is measured: each candidate scores a sample of database
segments, timed with CUDA events on the current stream, and the faster one is
selected for that (gap model, width).  Choices are kept for the process.
"""
from __future__ import annotations

import importlib

import torch

from ._lib import check, lib

_chosen: dict = {}


def tpt_of(query_len: int) -> int:
    return (query_len + 31) // 32


def set_variant(affine: bool, tpt: int, wide: int) -> None:
    check(lib().sseqs_sw_set_variant(1 if affine else 0, int(tpt), int(wide)), "set_variant")


def _time(q, batch, affine, n, reps):
    sw = importlib.import_module("sseqs_b200.sw")
    kw = dict(affine=affine, g0=1, n_targets=n, skip=1 if affine else 0,
              gap_a=11 if affine else -1, gap_b=1)
    out = sw.sw_scan(q, batch.ascii, batch.delim, **kw)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        sw.sw_scan(q, batch.ascii, batch.delim, out=out, **kw)
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(query_lengths, batch, max_segments: int = 200_000, reps: int = 2) -> dict:
    """Pick the faster layout for every width the given query lengths need.

    ``batch`` is a resident database batch whose first ``max_segments``
    segments serve as the timing sample.  Returns {(affine, tpt): wide}.
    """
    n = min(max_segments, batch.n_segments - 2)
    if n <= 0:
        return dict(_chosen)
    gen = torch.Generator(device="cpu")
    gen.manual_seed(1)
    for tpt in sorted({tpt_of(L) for L in query_lengths if 0 < L}):
        if tpt > 16:
            continue
        q = torch.randint(0, 20, (tpt * 32,), generator=gen, dtype=torch.uint8).cuda()
        for affine in (False, True):
            if (affine, tpt) in _chosen:
                continue
            t = []
            for wide in (0, 1):
                set_variant(affine, tpt, wide)
                t.append(_time(q, batch, affine, n, reps))
            best = 0 if t[0] <= t[1] else 1
            set_variant(affine, tpt, best)
            _chosen[(affine, tpt)] = best
    return dict(_chosen)


def chosen() -> dict:
    return dict(_chosen)
