"""Autotuner of the score kernel's lane layout.

For every stripe width tpt = ceil(query_len/32) <= 16 (linear kernel: <= 29)
the score kernel exists in two layouts (see ``sseqs_sw_set_variant``): fewer,
longer rows per lane group, or more targets per warp with twice the columns
per lane.  Both give
identical scores; which is faster depends on the width and on register
pressure, so it is measured: each candidate scores a sample of database
segments, timed with CUDA events on the current stream, and the faster one is
selected for that kernel (linear, affine, or the fused pass computing both)
and width.  The batched affine launch can also score two queries per launch
row (the query-pair kernel, ``sseqs_sw_set_query_pairing``); whether that is
faster depends on the width as well (it shares the per-row work, but doubles
the profile in shared memory), so ``autotune_pairing`` times it against one
query per row.  Choices are kept for the process.
"""
from __future__ import annotations

import importlib

import torch

from ._lib import check, lib

_chosen: dict = {}


def tpt_of(query_len: int) -> int:
    return (query_len + 31) // 32


MODES = ("linear", "affine", "both", "pair")
MAX_FUSED_TPT = 23      # widths scored by the fused pass (wider: the two kernels)


def set_variant(affine, tpt: int, wide: int) -> None:
    """``affine``: False/0 linear, True/1 affine, 2 the fused pass."""
    check(lib().sseqs_sw_set_variant(int(affine), int(tpt), int(wide)), "set_variant")


def get_variant(affine, tpt: int) -> int:
    """The layout selected for (kernel, tpt): 0 narrow, 1 wide."""
    v = lib().sseqs_sw_get_variant(int(affine), int(tpt))
    if v < 0:
        raise ValueError(f"no score kernel for mode {affine}, width {tpt}")
    return v


def has_wide(mode: int, tpt: int) -> bool:
    """Whether the kernel of ``mode`` has a wide layout of its own at ``tpt``."""
    words = [lib().sseqs_sw_variant_words(int(mode), int(tpt), w) for w in (0, 1)]
    return words[0] > 0 and words[1] != words[0]


def fused(query_len: int) -> bool:
    """Whether ``sw_scan_both`` runs the fused kernel for this query length."""
    return 0 < tpt_of(query_len) <= MAX_FUSED_TPT


def _time(q, batch, mode, n, reps):
    sw = importlib.import_module("sseqs_b200.sw")
    if mode == 2:
        def run():
            sw.sw_scan_both(q, batch.ascii, batch.delim, g0=1, n_targets=n, affine_skip=1)
    else:
        kw = dict(affine=mode == 1, g0=1, n_targets=n, skip=mode, gap_a=11 if mode else -1,
                  gap_b=1)
        out = torch.empty(n, dtype=torch.int32, device=batch.ascii.device)

        def run():
            sw.sw_scan(q, batch.ascii, batch.delim, out=out, **kw)
    run()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        run()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def autotune(query_lengths, batch, max_segments: int = 200_000, reps: int = 2) -> dict:
    """Pick the faster layout for every kernel and width the given query
    lengths need.

    ``batch`` is a resident database batch whose first ``max_segments``
    segments serve as the timing sample.  Returns {(mode name, tpt): wide}.
    """
    n = min(max_segments, batch.n_segments - 2)
    if n <= 0:
        return dict(_chosen)
    gen = torch.Generator(device="cpu")
    gen.manual_seed(1)
    for tpt in sorted({tpt_of(L) for L in query_lengths if 0 < L}):
        q = None
        for mode, name in enumerate(MODES):
            if (name, tpt) in _chosen or (mode == 2 and tpt > MAX_FUSED_TPT) or name == "pair":
                continue                 # the query-pair kernel: autotune_pairing
            if not has_wide(mode, tpt):
                continue
            if q is None:
                q = torch.randint(0, 20, (tpt * 32,), generator=gen, dtype=torch.uint8).cuda()
            t = []
            for wide in (0, 1):
                set_variant(mode, tpt, wide)
                t.append(_time(q, batch, mode, n, reps))
            best = 0 if t[0] <= t[1] else 1
            set_variant(mode, tpt, best)
            _chosen[(name, tpt)] = best
    return dict(_chosen)


def set_query_pairing(tpt: int, on: bool) -> None:
    """Score affine queries of width ``tpt`` (0: all widths) that share their
    targets two per launch row in the batched launch."""
    check(lib().sseqs_sw_set_query_pairing(int(tpt), 1 if on else 0), "set_query_pairing")


def get_query_pairing(tpt: int) -> bool:
    v = lib().sseqs_sw_get_query_pairing(int(tpt))
    if v < 0:
        raise ValueError(f"no width {tpt}")
    return bool(v)


def autotune_pairing(query_lengths, batch, max_segments: int = 200_000, reps: int = 2,
                     n_queries: int = 4) -> dict:
    """For every width the given lengths need, time the batched affine launch
    of ``n_queries`` queries one per launch row against two per row (the
    query-pair kernel, in each of its lane layouts) on a sample of
    ``batch``, and keep the faster.  Returns {("pairing", tpt): 0 off, 1 on}."""
    from . import batched
    n = min(max_segments, batch.n_segments - 2)
    if n <= 0:
        return dict(_chosen)
    gen = torch.Generator(device="cpu")
    gen.manual_seed(2)
    dev = batch.ascii.device
    for tpt in sorted({tpt_of(L) for L in query_lengths if 0 < L}):
        if ("pairing", tpt) in _chosen:
            continue
        q = torch.randint(0, 20, (n_queries, tpt * 32), generator=gen, dtype=torch.uint8).to(dev)
        lens = torch.full((n_queries,), tpt * 32, dtype=torch.int32, device=dev)
        out = torch.empty((n_queries, n), dtype=torch.int32, device=dev)
        tickets = torch.empty(n_queries, dtype=torch.int32, device=dev)

        def run():
            batched.sw_scan_queries(q, lens, tpt, batch.ascii, batch.delim, affine=True, g0=1,
                                    n_targets=n, skip=1, gap_a=11, gap_b=1, out=out,
                                    tickets=tickets)

        def time_it():
            run()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            for _ in range(reps):
                run()
            e1.record()
            torch.cuda.synchronize()
            return e0.elapsed_time(e1) / reps

        set_query_pairing(tpt, False)
        best_t, best = time_it(), (False, get_variant(3, tpt))
        for wide in ((0, 1) if has_wide(3, tpt) else (0,)):
            set_query_pairing(tpt, True)
            set_variant(3, tpt, wide)
            t = time_it()
            if t < best_t:
                best_t, best = t, (True, wide)
        set_query_pairing(tpt, best[0])
        set_variant(3, tpt, best[1])
        _chosen[("pairing", tpt)] = int(best[0])
        if best[0]:
            _chosen[("pair", tpt)] = best[1]
    return dict(_chosen)


def chosen() -> dict:
    return dict(_chosen)
