"""xbit 5-bit codec -- the operators of the reference's ``xbit`` extension.

Same names, argument meaning and return values as sseqs/xbit_bind.cpp:11-35:
``compress(u8[n]) -> u8[(5n+7)//8]`` and ``decompress(packed, n, lo) -> u8[n]``
(decodes the stream starting at packed byte ``lo``).  Work runs on the current
torch CUDA stream.
"""
from __future__ import annotations

import torch

from ._lib import check, lib, ptr, stream_ptr


def compress(input: torch.Tensor) -> torch.Tensor:
    """sseqs/xbit_bind.cpp:11-18."""
    inp = input.contiguous().to(device="cuda", dtype=torch.uint8)
    n = inp.numel()
    out = torch.zeros((n * 5 + 7) // 8, dtype=torch.uint8, device=inp.device)
    check(lib().sseqs_xbit_compress(ptr(inp), ptr(out), n, stream_ptr()), "xbit.compress")
    return out


def decompress(input: torch.Tensor, n: int, lo: int) -> torch.Tensor:
    """sseqs/xbit_bind.cpp:23-28."""
    inp = input.to(device="cuda", dtype=torch.uint8)
    if not inp.is_contiguous():
        inp = inp.contiguous()
    n, lo = int(n), int(lo)
    need = lo + (5 * n + 7) // 8      # the reference reads past the end here
    if n and need > inp.numel():
        raise ValueError(f"decompress: {n} symbols from byte {lo} need {need} bytes, "
                         f"input has {inp.numel()}")
    out = torch.empty(n, dtype=torch.uint8, device=inp.device)
    check(lib().sseqs_xbit_decompress(ptr(inp), ptr(out), n, lo, stream_ptr()), "xbit.decompress")
    return out
