"""Selection operators: delimiter scan, segment table and top-k.

Device-resident replacements for the torch ops on the reference path:
``arange[ascii == 64]`` (sseqs/msa.py:227), the lengths/offsets arithmetic
(sseqs/msa.py:237-267) and ``torch.topk`` + ``torch.sort`` (sseqs/msa.py:297,
307, 324, 335).  Top-k returns indices in increasing order and breaks ties at
the k-th value by taking lower indices first (torch.topk leaves that order
unspecified); like torch's radix select, -0.0 ranks below +0.0.
"""
from __future__ import annotations

import torch

from ._lib import check, lib, ptr, stream_ptr, workspace


def find_delims(ascii: torch.Tensor, count: torch.Tensor | None = None,
                max_out: int | None = None, sync: bool = True):
    """Positions (int32) of every '@' byte of ``ascii``.

    With ``sync`` the result is copied out at its exact size (one host
    read), so a resident table does not pin the ``max_out``-sized scratch
    (four bytes per input byte); otherwise ``(positions[max_out],
    count_dev)`` is returned.
    """
    n = ascii.numel()
    L = lib()
    if max_out is None:
        max_out = n
    out = torch.empty(max(max_out, 1), dtype=torch.int32, device=ascii.device)
    cnt = count if count is not None else torch.zeros(1, dtype=torch.int64, device=ascii.device)
    ws = workspace(L.sseqs_find_delims_workspace_bytes(n), ascii.device)
    check(L.sseqs_find_delims(ptr(ascii), n, ptr(out), max_out, ptr(cnt), ptr(ws), ws.numel(),
                              stream_ptr()), "find_delims")
    if not sync:
        return out, cnt
    c = int(cnt.item())
    return out[:c].clone() if c < out.numel() else out


def segment_table(ascii: torch.Tensor, delim: torch.Tensor) -> dict:
    """Non-empty segments of one decoded batch (sseqs/msa.py:237-267).

    Returns ``seg_index`` (segment number of each non-empty segment, i.e.
    the reference's filtered ``lengths`` positions), ``lengths``, ``offsets``
    (exclusive running sum of lengths+1, the reference's ``_offsets``) and
    ``maxlen``.
    """
    n = ascii.numel()
    nd = torch.tensor([delim.numel()], dtype=torch.int64, device=ascii.device)
    max_seg = delim.numel() + 1
    dev = ascii.device
    seg_index = torch.empty(max_seg, dtype=torch.int32, device=dev)
    lengths = torch.empty(max_seg, dtype=torch.int32, device=dev)
    offsets = torch.empty(max_seg, dtype=torch.int64, device=dev)
    nseg = torch.zeros(1, dtype=torch.int64, device=dev)
    maxlen = torch.zeros(1, dtype=torch.int32, device=dev)
    L = lib()
    ws = workspace(L.sseqs_segment_table_workspace_bytes(max_seg), dev)
    d = delim if delim.numel() else torch.zeros(1, dtype=torch.int32, device=dev)
    check(L.sseqs_segment_table(ptr(ascii), n, ptr(d), ptr(nd), max_seg, ptr(seg_index),
                                ptr(lengths), ptr(offsets), ptr(nseg), ptr(maxlen), ptr(ws),
                                ws.numel(), stream_ptr()), "segment_table")
    m = int(nseg.item())
    return {"seg_index": seg_index[:m], "lengths": lengths[:m], "offsets": offsets[:m],
            "maxlen": int(maxlen.item()), "n_segments": m}


def topk_indices(values: torch.Tensor, k: int, out: torch.Tensor | None = None,
                 ws: torch.Tensor | None = None) -> torch.Tensor:
    """Increasing indices of the k largest values (int32 or float16)."""
    if values.dtype == torch.int32:
        kt = 0
    elif values.dtype == torch.float16:
        kt = 1
    else:
        raise TypeError("topk_indices takes int32 or float16 values")
    values = values.contiguous()
    n = values.numel()
    k = int(k)
    if k < 0 or k > n:
        raise ValueError(f"selected index k out of range (k={k}, n={n})")
    L = lib()
    if out is None:
        out = torch.empty(max(k, 1), dtype=torch.int32, device=values.device)
    need = L.sseqs_topk_workspace_bytes(n)
    if ws is None or ws.numel() < need:
        ws = workspace(need, values.device)
    check(L.sseqs_topk(ptr(values), kt, n, k, ptr(out), ptr(ws), ws.numel(), stream_ptr()),
          "topk")
    return out[:k]
