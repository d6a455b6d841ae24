"""Autotuner of the score kernel's lane layout.

For every stripe width tpt = ceil(query_len/32) <= 16 (linear kernel: <= 29)
the score kernel exists in two layouts (see ``sseqs_sw_set_variant``): fewer,
longer rows per lane group, or more targets per warp with twice the columns
per lane.  Both give
identical scores; which is faster depends on the width and on register
pressure, so it is measured: each candidate scores a sample of database
segments, timed with CUDA events on the current stream, and the faster one is
selected for that kernel (linear, affine, or the fused pass computing both)
and width.  Choices are kept for the process.
"""
from __future__ import annotations

import importlib

import torch

from ._lib import check, lib

_chosen: dict = {}


def tpt_of(query_len: int) -> int:
    return (query_len + 31) // 32


MODES = ("linear", "affine", "both")
MAX_FUSED_TPT = 21      # widths scored by the fused pass (wider: the two kernels)


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
            if (name, tpt) in _chosen or (mode == 2 and tpt > MAX_FUSED_TPT):
                continue
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


def chosen() -> dict:
    return dict(_chosen)
