"""Gapless FFT prefilter -- the reference's ``conv`` extension and its LUTs.

``prefilter_luts`` is the query-weighted SVD of BLOSUM62 of
sseqs/msa.py:110-145 (same numpy calls, so the same tables); the scores come
from ``csrc/prefilter.cu`` (fp32 FFTs, fp16 output).  ``warp_corr`` keeps the
call shape of sseqs/filter_bind.cpp:20-81 and fills ``corr`` in place.

Supported transform lengths are 64..2048.  The reference computes no scores
(leaves zeros) for N < 64 and N = 2048 (sseqs/filter.cu:182-320); here N < 64
is computed at 64 and N = 2048 is computed.
"""
from __future__ import annotations

import numpy as np
import torch

from ._lib import check, lib, ptr, stream_ptr, workspace

AA = "ARNDCQEGHILKMFPSTWYV"
AA_TO_POS = {a: i for i, a in enumerate(AA)}
AA_TO_POS.update({"X": 20, "-": 20, "*": 20})

_B62_FLAT = [4, -1, -2, -2, 0, -1, -1, 0, -2, -1, -1, -1, -1, -2, -1, 1, 0, -3, -2, 0, -1, 5, 0, -2,
             -3, 1, 0, -2, 0, -3, -2, 2, -1, -3, -2, -1, -1, -3, -2, -3, -2, 0, 6, 1, -3, 0, 0, 0,
             1, -3, -3, 0, -2, -3, -2, 1, 0, -4, -2, -3, -2, -2, 1, 6, -3, 0, 2, -1, -1, -3, -4,
             -1, -3, -3, -1, 0, -1, -4, -3, -3, 0, -3, -3, -3, 9, -3, -4, -3, -3, -1, -1, -3, -1,
             -2, -3, -1, -1, -2, -2, -1, -1, 1, 0, 0, -3, 5, 2, -2, 0, -3, -2, 1, 0, -3, -1, 0,
             -1, -2, -1, -2, -1, 0, 0, 2, -4, 2, 5, -2, 0, -3, -3, 1, -2, -3, -1, 0, -1, -3, -2,
             -2, 0, -2, 0, -1, -3, -2, -2, 6, -2, -4, -4, -2, -3, -3, -2, 0, -2, -2, -3, -3, -2, 0,
             1, -1, -3, 0, 0, -2, 8, -3, -3, -1, -2, -1, -2, -1, -2, -2, 2, -3, -1, -3, -3, -3, -1,
             -3, -3, -4, -3, 4, 2, -3, 1, 0, -3, -2, -1, -3, -1, 3, -1, -2, -3, -4, -1, -2, -3, -4,
             -3, 2, 4, -2, 2, 0, -3, -2, -1, -2, -1, 1, -1, 2, 0, -1, -3, 1, 1, -2, -1, -3, -2, 5,
             -1, -3, -1, 0, -1, -3, -2, -2, -1, -1, -2, -3, -1, 0, -2, -3, -2, 1, 2, -1, 5, 0, -2,
             -1, -1, -1, -1, 1, -2, -3, -3, -3, -2, -3, -3, -3, -1, 0, 0, -3, 0, 6, -4, -2, -2, 1,
             3, -1, -1, -2, -2, -1, -3, -1, -1, -2, -2, -3, -3, -1, -2, -4, 7, -1, -1, -4, -3, -2,
             1, -1, 1, 0, -1, 0, 0, 0, -1, -2, -2, 0, -1, -2, -1, 4, 1, -3, -2, -2, 0, -1, 0, -1,
             -1, -1, -1, -2, -2, -1, -1, -1, -1, -2, -1, 1, 5, -2, -2, 0, -3, -3, -4, -4, -2, -2,
             -3, -2, -2, -3, -2, -3, -1, 1, -4, -3, -2, 11, 2, -3, -2, -2, -2, -3, -2, -1, -2, -3,
             2, -1, -1, -2, -1, 3, -3, -2, -2, 2, 7, -1, 0, -3, -3, -3, -1, -2, -2, -3, -3, 3, 1,
             -2, 1, -1, -2, -2, 0, -3, -1, 4]


class Luts:
    def __init__(self, A: torch.Tensor, B: torch.Tensor, qrev: torch.Tensor, query_len: int):
        self.A, self.B, self.qrev, self.query_len = A, B, qrev, query_len

    @property
    def rank(self):
        return self.A.shape[0]


def prefilter_luts(query: str, fft_rank: int = 4, device="cuda") -> Luts:
    """sseqs/msa.py:125-145 and :157 -> tables A, B (float32 [20, 21]) and the
    reversed query mapped to 0..20."""
    b62 = np.array(_B62_FLAT).reshape(20, 20)
    if fft_rank == 1:
        b62[b62 < 0] = 0
    w = np.sqrt(np.array([query.count(a) for a in AA]) / len(query))
    U, S, Vt = np.linalg.svd(w[:, None] * b62)
    A = np.stack([np.append(np.sqrt(s) * u, 0.0) for s, u in zip(S, U.T)]).astype(np.float32)
    B = np.stack([np.append(np.sqrt(s) * v, 0.0) for s, v in zip(S, Vt)]).astype(np.float32)
    qrev = np.array([AA_TO_POS.get(c, 20) for c in query[::-1]], dtype=np.uint8)
    return Luts(torch.from_numpy(A).to(device), torch.from_numpy(B).to(device),
                torch.from_numpy(qrev).to(device), len(query))


def transform_length(query_len: int, maxlen: int) -> int:
    """N = next power of two of max(len(query), longest segment) (msa.py:261)."""
    n = 1 << (max(query_len, maxlen) - 1).bit_length()
    return max(n, 64)


def prefilter_scores(luts: Luts, ascii, offsets, lengths, n_segments: int, n: int, k: int,
                     out: torch.Tensor | None = None) -> torch.Tensor:
    k = max(1, min(k, luts.rank))
    if out is None:
        out = torch.zeros(max(n_segments, 1), dtype=torch.float16, device=ascii.device)
    L = lib()
    ws = workspace(L.sseqs_prefilter_workspace_bytes(n, k), ascii.device)
    A = luts.A[:k].contiguous()
    B = luts.B[:k].contiguous()
    check(L.sseqs_prefilter(ptr(ascii), ptr(offsets), ptr(lengths), n_segments, ptr(luts.qrev),
                            luts.query_len, ptr(A), ptr(B), k, n, ptr(out), ptr(ws), ws.numel(),
                            stream_ptr()), "prefilter")
    return out[:n_segments]


def prefilter_batch(query: str, batch, luts: Luts, fft_rank: int = 4) -> torch.Tensor:
    n = transform_length(len(query), batch.maxlen)
    return prefilter_scores(luts, batch.ascii, batch.offsets, batch.lengths, batch.n_segments,
                            n, fft_rank)


def warp_corr(corr, query_reversed_indices, weight_LUTS_A, W, flat, offsets, lengths, k,
              query_length, maxlen, n, query_rfft_tensor=None):
    """sseqs/filter_bind.cpp:20-64: fills ``corr`` (float16 [B]) in place.

    ``query_rfft_tensor`` was scratch space in the reference and is not used;
    the returned (B, 2) tensor is, as in the reference, uninitialised.
    """
    B = lengths.numel()
    luts = Luts(weight_LUTS_A.float().contiguous(), W.float().contiguous(),
                query_reversed_indices.to(torch.uint8).contiguous(), int(query_length))
    off = offsets.to(torch.int64).contiguous()
    ln = lengths.to(torch.int32).contiguous()
    target = corr if corr.dtype == torch.float16 else torch.empty_like(corr, dtype=torch.float16)
    prefilter_scores(luts, flat, off, ln, B, max(int(n), 64), int(k), out=target)
    if target is not corr:
        corr.copy_(target)
    return torch.empty((B, 2), dtype=torch.float32, device=corr.device)
